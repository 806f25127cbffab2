"""tsne_h2pack: t-SNE whose optimisation phase runs on a B200 (sm_100a) through the engine's
C ABI (include/tsne_h2pack.h); a drop-in for the reference package's public names.

    >>> from tsne_h2pack import TSNE
    >>> Y = TSNE(n_components=2, perplexity=30).fit_transform(X)
"""

__version__ = "3.3.1"

from .manifold import H2_DEFAULTS, TSNE, h2_defaults  # noqa: E402

__all__ = ["TSNE", "H2_DEFAULTS", "h2_defaults", "__version__"]
