"""The C ABI library without a GPU: it loads, exports every entry point declared in
include/tsne_h2pack.h, and its structs have the reference's layout."""
import ctypes
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
HEADER = ROOT / "include" / "tsne_h2pack.h"


def declared():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"^TSNE_API[^(]*?\b([a-z_0-9]+)\(", text, flags=re.M)))


def test_library_exports_every_declared_symbol():
    from tsne_h2pack._backend import get_backend
    lib = get_backend()._lib
    names = declared()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_backend_binds_reference_entry_points():
    """Every function the reference's Python loader configures (_backend.py:345-448)."""
    from tsne_h2pack._backend import get_backend
    lib = get_backend()._lib
    for n in ("tsne_create_default_params", "tsne_init", "tsne_init_with_P", "tsne_run", "tsne_get_embedding",
              "tsne_destroy", "tsne_fit_transform", "tsne_fit_transform_with_P", "compute_P_from_knn_distances",
              "sparse_matrix_destroy", "sparse_matrix_create", "tsne_set_init_profiling_times",
              "compute_kl_divergence"):
        fn = getattr(lib, n)
        assert fn.argtypes is not None or n == "tsne_create_default_params"


def test_params_layout_matches_header(tmp_path):
    """offsetof() of every tsne_params_t field, compiled from the header, equals the ctypes
    layout (160 bytes, reference _backend.py:51-96)."""
    from tsne_h2pack._backend import TSNEParams
    fields = [f for f, _ in TSNEParams._fields_ if not f.startswith("_pad")]
    src = tmp_path / "off.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "tsne_h2pack.h"\nint main(void){\n'
                   + "".join(f'printf("{f} %zu\\n", offsetof(tsne_params_t, {f}));\n' for f in fields)
                   + 'printf("sizeof %zu\\n", sizeof(tsne_params_t));\nprintf("csr %zu\\n", sizeof(sparse_matrix_t));\nreturn 0;}\n')
    exe = tmp_path / "off"
    subprocess.run(["gcc", "-I", str(HEADER.parent), str(src), "-o", str(exe)], check=True)
    out = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split("\n") if line)
    for f in fields:
        assert int(out[f]) == getattr(TSNEParams, f).offset, f
    assert int(out["sizeof"]) == ctypes.sizeof(TSNEParams) == 160
    from tsne_h2pack._backend import SparseMatrix
    assert int(out["csr"]) == ctypes.sizeof(SparseMatrix)


def test_default_params_from_library():
    from tsne_h2pack._backend import get_backend
    be = get_backend()
    p = be._lib.tsne_create_default_params()
    q = be.create_default_params()
    for f in ("n_iter", "perplexity", "momentum", "initial_momentum", "momentum_switch_iter", "early_exag",
              "early_exag_iter", "h2_tol", "h2_rebuild_freq", "h2_leaf_size", "h2_rebuild_freq_early",
              "min_iter", "sklearn_compatible", "convergence_patience"):
        assert getattr(p, f) == getattr(q, f), f
    assert p.h2_leaf_size == 100 and p.h2_rebuild_freq_early == 10


def test_sparse_matrix_roundtrip_on_host():
    """sparse_matrix_create / sparse_matvec / sparse_matrix_destroy are host functions."""
    import numpy as np
    from scipy.sparse import random as sprandom
    from tsne_h2pack._backend import SparseMatrix, get_backend, scipy_csr_to_c_sparse_matrix
    lib = get_backend()._lib
    lib.sparse_matvec.argtypes = [ctypes.POINTER(SparseMatrix), np.ctypeslib.ndpointer(np.float64),
                                  np.ctypeslib.ndpointer(np.float64)]
    A = sprandom(50, 50, density=0.2, random_state=0, format="csr")
    m = scipy_csr_to_c_sparse_matrix(A, lib)
    x = np.arange(50, dtype=np.float64)
    y = np.zeros(50)
    lib.sparse_matvec(m, x, y)
    np.testing.assert_allclose(y, A @ x, rtol=1e-12)
    lib.sparse_matrix_destroy(m)


def test_device_constants_match_oracle():
    """The H2 design constants of the device build and of the oracle are the same numbers."""
    cu = (ROOT / "tsne-h2pack-python_b200" / "csrc" / "common.cuh").read_text()
    ora = (ROOT / "oracle" / "tsne_oracle.c").read_text()
    def dev(name):
        return re.search(rf"constexpr \w+ {name} = ([0-9.e+-]+);", cu).group(1)
    def orc(name):
        return re.search(rf"#define ORA_{name} ([0-9.e+-]+)", ora).group(1)
    assert float(dev("KEY_DEPTH_2D")) == float(orc("KEY_DEPTH_2D"))
    assert float(dev("KEY_DEPTH_3D")) == float(orc("KEY_DEPTH_3D"))
    assert float(dev("MIN_HALF_WIDTH")) == float(orc("MIN_HALF_WIDTH"))
    assert float(dev("MIN_ADM_LEVEL")) == float(orc("MIN_ADM_LEVEL"))
    assert float(dev("ID_TOL_FACTOR")) == float(orc("ID_TOL_FACTOR"))
    assert float(dev("MAX_RANK_2D")) == float(orc("MAX_RANK_2D"))
    assert float(dev("ADM_EXTRA")) == float(orc("ADM_EXTRA"))
    assert float(dev("SHELL_PTS_2D")) == float(orc("SHELL_PTS_2D"))
    assert float(dev("SHELL_GRID_3D")) == float(orc("SHELL_GRID_3D"))
    rho = re.search(r"#define ORA_SHELL_RHO_LIST ([0-9., ]+)", ora).group(1)
    assert [float(x) for x in rho.split(",")] == [3.0, 4.5, 7.0, 12.0]
    assert "k == 0 ? 3.0 : k == 1 ? 4.5 : k == 2 ? 7.0 : 12.0" in cu


def test_job_info_layout_matches_header(tmp_path):
    """tsne_job_info_t of the batched/served entry points: ctypes layout = compiled header."""
    from tsne_h2pack.serving import JobInfo
    fields = [f for f, _ in JobInfo._fields_]
    src = tmp_path / "job.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "tsne_h2pack.h"\nint main(void){\n'
                   + "".join(f'printf("{f} %zu\\n", offsetof(tsne_job_info_t, {f}));\n' for f in fields)
                   + 'printf("sizeof %zu\\n", sizeof(tsne_job_info_t));\nreturn 0;}\n')
    exe = tmp_path / "job"
    subprocess.run(["gcc", "-I", str(HEADER.parent), str(src), "-o", str(exe)], check=True)
    out = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True).stdout.split("\n") if line)
    for f in fields:
        assert int(out[f]) == getattr(JobInfo, f).offset, f
    assert int(out["sizeof"]) == ctypes.sizeof(JobInfo)


def test_server_rejects_bad_arguments_without_a_device():
    """tsne_server_create validates its arguments before touching the device."""
    from tsne_h2pack.serving import _bind
    from tsne_h2pack._backend import get_backend
    lib = get_backend()._lib
    _bind(lib)
    assert not lib.tsne_server_create(0, 10.0)
    assert not lib.tsne_server_create(2, 0.0)
    assert lib.tsne_server_submit(None, 10, 2, None, None) == -1
    assert lib.tsne_server_pending(None) == -1


def test_embedding_server_fails_loudly_without_a_device():
    """The Python server wrapper raises when the engine cannot create a server (here: no CUDA
    device), rather than falling back to anything."""
    import torch
    from tsne_h2pack.serving import EmbeddingServer
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(RuntimeError):
        EmbeddingServer(max_concurrent=2, hbm_budget_gb=1.0)


@pytest.mark.parametrize("case", ["first_not_zero", "decreasing"])
def test_init_rejects_bad_row_pointers_before_the_device(case, capfd):
    """tsne_init_with_P checks P's row pointers on the host before it creates any device state
    (NULL, P left with the caller, as on a wrong shape)."""
    import numpy as np
    from scipy.sparse import csr_matrix
    from tsne_h2pack._backend import get_backend, scipy_csr_to_c_sparse_matrix
    be = get_backend()
    lib = be._lib
    n = 50
    P = csr_matrix(np.eye(n, k=1) + np.eye(n, k=-1))
    Pc = scipy_csr_to_c_sparse_matrix(P, lib)
    rp = Pc.contents.row_ptr
    if case == "first_not_zero":
        rp[0] = 1
    else:
        rp[10], rp[11] = rp[11], rp[10]
    params = be.create_default_params()
    params.verbose = 0
    ws = lib.tsne_init_with_P(None, n, 0, 2, ctypes.byref(params), Pc)
    ctypes.CDLL(None).fflush(None)
    assert not ws
    assert "row pointers" in capfd.readouterr().out
    lib.sparse_matrix_destroy(Pc)
