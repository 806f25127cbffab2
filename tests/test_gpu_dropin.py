"""The drop-in, through the reference's own Python package: its unmodified tsne_h2pack
package (_backend.py's loader, ctypes signatures and marshalling, manifold.py's TSNE) loads
this engine's libtsne_h2pack.so from its _lib/ directory and runs method='h2pack' and
method='exact' on a precomputed graph. The results must equal, bit for bit, those of this
repository's own package on the same input (the same library underneath, the same
parameters mapped onto tsne_params_t, the same host-side P: this package's own default builds
P on the device instead, so the test selects its host path with TSNE_HOST_P=1).

The reference package is staged by build() in baseline/_ref/tsne_h2pack (a copy of the
reference checkout's package, as `pip install --target` would place it); the test copies it
to a temporary directory, adds the library, and imports it in a child process so that its
module name does not collide with this repository's package.
"""
import json
import shutil
import subprocess
import sys
import textwrap
from pathlib import Path

import numpy as np
import pytest

from helpers import problem

ROOT = Path(__file__).resolve().parent.parent
REF_PKG = ROOT / "baseline" / "_ref" / "tsne_h2pack"
LIB = ROOT / "tsne-h2pack-python_b200" / "tsne_h2pack" / "_lib" / "libtsne_h2pack.so"

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not REF_PKG.is_dir(), reason="the reference package was not staged by build()")]

CASES = [dict(method="h2pack", init="random", random_state=3, max_iter=300),
         dict(method="exact", init="random", random_state=4, max_iter=60),
         dict(method="h2pack", init="pca", random_state=5, max_iter=120, n_components=3)]


def test_reference_package_drives_this_library(tmp_path, monkeypatch):
    pkg = tmp_path / "tsne_h2pack"
    shutil.copytree(REF_PKG, pkg)
    (pkg / "_lib").mkdir(exist_ok=True)
    shutil.copy(LIB, pkg / "_lib" / "libtsne_h2pack.so")
    X, G, P, _ = problem(4000, seed=6, dim=30)
    G = G.tocsr()
    np.savez(tmp_path / "in.npz", X=X, gd=G.data, gi=G.indices, gp=G.indptr)
    script = textwrap.dedent(f"""
        import json, sys
        import numpy as np
        from scipy.sparse import csr_matrix
        sys.path.insert(0, {str(tmp_path)!r})
        import tsne_h2pack
        from tsne_h2pack import TSNE
        assert tsne_h2pack.__file__.startswith({str(tmp_path)!r}), tsne_h2pack.__file__
        z = np.load({str(tmp_path / 'in.npz')!r})
        n = z["X"].shape[0]
        G = csr_matrix((z["gd"], z["gi"], z["gp"]), shape=(n, n))
        cases = json.loads({json.dumps(json.dumps(CASES))})
        out = {{}}
        for i, c in enumerate(cases):
            init = c.pop("init")
            if init == "pca":
                # the reference's PCA init needs the features; with a precomputed graph it
                # takes an array: the same array is given to both packages
                from sklearn.decomposition import PCA
                Y0 = PCA(n_components=c.get("n_components", 2), random_state=0).fit_transform(z["X"])
                init = Y0 / np.std(Y0[:, 0]) * 1e-4
            t = TSNE(metric="precomputed", init=init, **c)
            out[f"Y{{i}}"] = t.fit_transform(G)
            out[f"kl{{i}}"] = np.array(t.kl_divergence_)
        np.savez({str(tmp_path / 'out.npz')!r}, **out)
        print("loaded", tsne_h2pack._backend.get_backend()._lib._name)
    """)
    r = subprocess.run([sys.executable, "-c", script], capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-3000:]
    assert str(pkg / "_lib" / "libtsne_h2pack.so") in r.stdout
    ref = np.load(tmp_path / "out.npz")

    from sklearn.decomposition import PCA
    from tsne_h2pack import TSNE
    monkeypatch.setenv("TSNE_HOST_P", "1")     # P symmetrised on the host, as the reference package does
    for i, c in enumerate(CASES):
        c = dict(c)
        init = c.pop("init")
        if init == "pca":
            Y0 = PCA(n_components=c.get("n_components", 2), random_state=0).fit_transform(X)
            init = Y0 / np.std(Y0[:, 0]) * 1e-4
        t = TSNE(metric="precomputed", init=init, **c)
        Y = t.fit_transform(G)
        assert np.isfinite(Y).all()
        np.testing.assert_array_equal(Y, ref[f"Y{i}"], err_msg=str(c))
        assert float(t.kl_divergence_) == float(ref[f"kl{i}"]), c
