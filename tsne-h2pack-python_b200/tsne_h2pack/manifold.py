"""scikit-learn style TSNE estimator over the B200 engine.

Mirrors the reference's tsne_h2pack.manifold (tsne_h2pack/manifold.py of the reference
project): same constructor arguments and defaults, per-dimension H2 defaults, parameter
mapping onto tsne_params_t, PCA / random / array initialisation, the 'precomputed' k-NN
graph path and the fitted attributes. The optimisation itself runs in the native engine.
"""
import os
import warnings
from typing import Optional, Union

import numpy as np

from ._backend import NP_DTYPE, TSNEParams, get_backend


def _resolve_n_jobs(n_jobs: Optional[int]) -> int:
    """joblib convention: None -> 1, -1 -> all cores, -2 -> all but one, 0 -> 1."""
    if n_jobs is None or n_jobs == 0:
        return 1
    if n_jobs < 0:
        return max(1, (os.cpu_count() or 1) + 1 + n_jobs)
    return n_jobs


# Per-dimension H2 settings (reference manifold.py:44-47): 2D tolerance 1e-2, 3D 3e-2;
# rebuild every 3 iterations (every 10 during early exaggeration); 100 points per leaf.
H2_DEFAULTS = {
    2: dict(h2_tol=1e-2, h2_rebuild_freq=3, h2_rebuild_freq_early=10, h2_leaf_size=100),
    3: dict(h2_tol=3e-2, h2_rebuild_freq=3, h2_rebuild_freq_early=10, h2_leaf_size=100),
}


def h2_defaults(n_components: int) -> dict:
    """H2 defaults for an embedding dimension (3 and more share the 3D row)."""
    return dict(H2_DEFAULTS[2 if n_components <= 2 else 3])


class TSNE:
    """t-SNE with the repulsive force from a device H2 matrix (method='h2pack') or exact
    O(N^2) device sums (method='exact').

    Parameters and attributes follow the reference estimator: n_components, perplexity,
    early_exaggeration, learning_rate ('auto' = max(N / 12, 200)), max_iter,
    n_iter_without_progress, min_grad_norm, metric ('euclidean' or 'precomputed' k-NN
    distance graph), init ('pca', 'random' or an (n_samples, n_components) array), verbose,
    random_state, method ('h2pack' or 'exact'), n_jobs, h2_tol, h2_rebuild_freq,
    enable_profiling, profiling_output_file, knn_method, knn_params, h2_rebuild_freq_early,
    h2_leaf_size. After fit_transform: embedding_, kl_divergence_, n_iter_, knn_time_.
    """

    def __init__(self, n_components: int = 2, perplexity: float = 30.0, early_exaggeration: float = 12.0,
                 learning_rate: Union[float, str] = "auto", max_iter: int = 1000,
                 n_iter_without_progress: int = 300, min_grad_norm: float = 1e-7, metric: str = "euclidean",
                 init: Union[str, np.ndarray] = "pca", verbose: int = 0, random_state: Optional[int] = None,
                 method: str = "h2pack", n_jobs: Optional[int] = None, h2_tol: Optional[float] = None,
                 h2_rebuild_freq: Optional[int] = None, enable_profiling: bool = False,
                 profiling_output_file: Optional[str] = None, knn_method: str = "pynndescent",
                 knn_params: Optional[dict] = None, h2_rebuild_freq_early: Optional[int] = None,
                 h2_leaf_size: Optional[int] = None):
        self.n_components = n_components
        self.perplexity = perplexity
        self.early_exaggeration = early_exaggeration
        self.learning_rate = learning_rate
        self.max_iter = max_iter
        self.n_iter_without_progress = n_iter_without_progress
        self.min_grad_norm = min_grad_norm
        self.metric = metric
        self.init = init
        self.verbose = verbose
        self.random_state = random_state
        self.method = method
        self.n_jobs = _resolve_n_jobs(n_jobs)
        dflt = h2_defaults(n_components if isinstance(n_components, int) and n_components >= 1 else 2)
        self.h2_tol = dflt["h2_tol"] if h2_tol is None else h2_tol
        self.h2_rebuild_freq = dflt["h2_rebuild_freq"] if h2_rebuild_freq is None else h2_rebuild_freq
        self.enable_profiling = enable_profiling
        self.profiling_output_file = profiling_output_file
        self.knn_method = knn_method
        self.knn_params = knn_params or {}
        self.h2_rebuild_freq_early = (dflt["h2_rebuild_freq_early"] if h2_rebuild_freq_early is None
                                      else h2_rebuild_freq_early)
        self.h2_leaf_size = dflt["h2_leaf_size"] if h2_leaf_size is None else h2_leaf_size
        self.embedding_: Optional[np.ndarray] = None
        self.kl_divergence_: Optional[float] = None
        self.n_iter_: Optional[int] = None
        self._validate_params()

    def _validate_params(self):
        if self.metric not in ("euclidean", "precomputed"):
            raise ValueError(f"metric='{self.metric}' not supported. Use 'euclidean' or 'precomputed'.")
        if isinstance(self.init, str):
            if self.init not in ("random", "pca"):
                raise ValueError(f"init='{self.init}' not supported. Must be 'random', 'pca' or an ndarray of "
                                 "shape (n_samples, n_components).")
        else:
            init = np.asarray(self.init)
            if init.ndim != 2 or init.shape[1] != self.n_components:
                what = "an array of shape " + str(init.shape) if init.ndim else repr(self.init)
                raise ValueError("init not supported: must be 'random', 'pca' or an ndarray of shape "
                                 f"(n_samples, n_components={self.n_components}), got {what}")
            if not np.issubdtype(init.dtype, np.number) or not np.isfinite(init).all():
                raise ValueError("init array must contain only finite numbers")
        if self.method not in ("h2pack", "exact"):
            raise ValueError(f"method='{self.method}' not supported. Must be 'h2pack' or 'exact'.")
        if self.n_components < 1:
            raise ValueError("n_components must be >= 1")
        if self.perplexity <= 0:
            raise ValueError("perplexity must be > 0")
        if isinstance(self.learning_rate, str):
            if self.learning_rate != "auto":
                raise ValueError("learning_rate must be a positive number or 'auto'")
        elif self.learning_rate <= 0:
            raise ValueError("learning_rate must be > 0")
        if self.h2_rebuild_freq < 1 or self.h2_rebuild_freq_early < 1:
            raise ValueError("h2_rebuild_freq and h2_rebuild_freq_early must be >= 1")
        if self.h2_leaf_size < 1:
            raise ValueError("h2_leaf_size must be >= 1")
        if self.max_iter < 1:
            raise ValueError("max_iter must be >= 1")

    def _map_params_to_c_struct(self, n_samples: Optional[int] = None) -> TSNEParams:
        """tsne_params_t for this estimator (reference manifold.py:319-378): method='exact'
        disables the H2 matrix (rebuild frequency 999999); the early rebuild frequency is never
        below the late one."""
        p = get_backend().create_default_params()
        p.n_iter = self.max_iter
        p.perplexity = self.perplexity
        if self.learning_rate == "auto":
            p.learning_rate = max((n_samples or 0) / 12.0, 200.0)
        else:
            p.learning_rate = self.learning_rate
        p.early_exag = self.early_exaggeration
        p.early_exag_iter = 250
        p.initial_momentum = 0.5
        p.momentum = 0.8
        p.momentum_switch_iter = 250
        p.verbose = 1 if self.verbose > 0 else 0
        p.print_freq = 50
        if self.method == "exact":
            p.h2_rebuild_freq = 999999
            p.h2_tol = 1e-4
        else:
            p.h2_rebuild_freq = self.h2_rebuild_freq
            p.h2_tol = self.h2_tol
        p.h2_rebuild_freq_early = max(self.h2_rebuild_freq_early, self.h2_rebuild_freq)
        p.h2_leaf_size = self.h2_leaf_size
        p.enable_profiling = 1 if self.enable_profiling else 0
        if self.profiling_output_file is not None:
            p.profiling_output_file = self.profiling_output_file.encode("utf-8")
        if self.random_state is not None:
            p.random_seed = self.random_state
        p.num_threads = self.n_jobs
        p.convergence_patience = self.n_iter_without_progress
        p.min_iter = 250
        p.sklearn_compatible = 1
        return p

    def _initial_embedding(self, X, n_samples: int) -> Optional[np.ndarray]:
        """(n_samples, n_components) initial Y, or None for 'random' (drawn by the engine from
        random_state). 'pca' is the exact PCA projection computed on the device, scaled to a
        first-coordinate standard deviation of 1e-4 (the reference uses scikit-learn's randomized
        approximation of the same projection)."""
        self._validate_params()
        if isinstance(self.init, str):
            if self.init == "random":
                return None
            if X is None:
                warnings.warn("init='pca' needs the input features, which metric='precomputed' does not "
                              "provide; using init='random' instead. Pass init='random' (or an ndarray) to "
                              "silence this warning.", UserWarning, stacklevel=4)
                return None
            n_features = X.shape[1]
            if self.n_components > min(n_samples, n_features):
                raise ValueError(f"init='pca' needs n_components={self.n_components} <= "
                                 f"min(n_samples, n_features)={min(n_samples, n_features)}")
            return get_backend().pca_init(np.asarray(X, dtype=np.float64), self.n_components)
        Y = np.array(self.init, dtype=np.float64)
        if Y.shape != (n_samples, self.n_components):
            raise ValueError(f"init array has shape {Y.shape}, expected (n_samples, n_components)="
                             f"{(n_samples, self.n_components)}")
        return Y

    def _fit_transform_precomputed(self, X):
        from scipy.sparse import csr_matrix, issparse
        if not issparse(X):
            raise ValueError("metric='precomputed' expects a sparse matrix of k-NN distances, e.g. "
                             "kneighbors_graph(X, n_neighbors=90, mode='distance')")
        if X.shape[0] != X.shape[1]:
            raise ValueError(f"precomputed k-NN graph must be square, got {X.shape}")
        graph = csr_matrix(X, copy=True)
        graph.setdiag(0)
        graph.eliminate_zeros()
        graph.sort_indices()
        if not np.isfinite(graph.data).all() or (graph.data < 0).any():
            raise ValueError("precomputed distances must be finite and non-negative")
        min_neighbors = int(np.diff(graph.indptr).min())
        if min_neighbors <= self.perplexity:
            raise ValueError(f"every row needs more than perplexity={self.perplexity} neighbors, but one row "
                             f"has {min_neighbors}")
        backend = get_backend()
        params = self._map_params_to_c_struct(n_samples=graph.shape[0])
        if self.verbose:
            print(f"Running t-SNE with backend: {backend.backend_type}")
            print(f"Precomputed k-NN graph: {graph.shape[0]} points, {graph.nnz} distances")
        init_Y = self._initial_embedding(None, graph.shape[0])
        self.knn_time_ = 0.0
        Y, metrics = backend.fit_transform_with_knn_distances(None, graph, self.n_components, params,
                                                              init_Y=init_Y)
        self.embedding_ = Y
        self.n_iter_ = metrics.get("n_iter", params.n_iter)
        self.kl_divergence_ = metrics.get("kl_divergence", 0.0)
        return self.embedding_

    def fit(self, X, y=None):
        raise NotImplementedError("fit() is not implemented. Use fit_transform() instead.")

    def fit_transform(self, X, y=None) -> np.ndarray:
        """Embed X (features, or a sparse k-NN distance graph with metric='precomputed')."""
        if self.metric == "precomputed":
            return self._fit_transform_precomputed(X)
        # the device k-NN reads single precision: a float32 X stays float32 (the float64 copy the
        # other k-NN methods read would round back to the same values), which saves a conversion
        # of the whole matrix each way; PCA initialisation converts on its own
        keep32 = self.knn_method == "cuda" and isinstance(X, np.ndarray) and X.dtype == np.float32
        X = self._validate_data(X, dtype=np.float32 if keep32 else NP_DTYPE)
        init_Y = self._initial_embedding(X, X.shape[0])
        backend = get_backend()
        params = self._map_params_to_c_struct(n_samples=X.shape[0])
        if self.verbose:
            print(f"Running t-SNE with backend: {backend.backend_type}")
            print(f"Input shape: {X.shape}")
            print(f"Perplexity: {self.perplexity}, max_iter: {self.max_iter}")
            print(f"k-NN method: {self.knn_method}")
        from ._knn_methods import get_knn_method
        knn = get_knn_method(self.knn_method)
        k = min(X.shape[0] - 1, int(3 * self.perplexity))
        if self.verbose:
            print(f"Computing {k} nearest neighbors using {self.knn_method}...")
        G = knn.compute(X, k=k, n_jobs=self.n_jobs, verbose=(self.verbose > 0), **self.knn_params)
        self.knn_time_ = getattr(G, "knn_time", 0.0)
        Y, metrics = backend.fit_transform_with_knn_distances(X, G, self.n_components, params, init_Y=init_Y)
        self.embedding_ = Y
        self.n_iter_ = metrics.get("n_iter", params.n_iter)
        self.kl_divergence_ = metrics.get("kl_divergence", 0.0)
        return self.embedding_

    def _validate_data(self, X, dtype=NP_DTYPE) -> np.ndarray:
        X = np.asarray(X, dtype=dtype)
        if X.ndim != 2:
            raise ValueError(f"X must be 2-dimensional array, got {X.ndim} dimensions")
        n_samples = X.shape[0]
        if n_samples < 2:
            raise ValueError(f"n_samples={n_samples} should be >= 2")
        if self.perplexity >= n_samples:
            raise ValueError(f"perplexity={self.perplexity} must be less than n_samples={n_samples}")
        if not np.isfinite(X).all():
            raise ValueError("X contains NaN or inf values")
        return X
