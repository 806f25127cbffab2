"""Build recipe of the engine: compiles csrc/*.cu for sm_100a into tsne_h2pack/_lib/libtsne_h2pack.so.

    python tsne-h2pack-python_b200/build.py [--jobs N]

nvcc cross-compiles without a GPU. The library links the CUDA runtime statically, so the
in-tree .so is all the reference's Python loader needs (tsne_h2pack/_backend.py searches
tsne_h2pack/_lib/libtsne_h2pack.so).
"""
import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
OUT_DIR = HERE / "tsne_h2pack" / "_lib"
OUT = OUT_DIR / "libtsne_h2pack.so"
BUILD = HERE / "_build"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-std=c++17", "-O3", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
         "-Xptxas", "-warn-spills", "--expt-relaxed-constexpr"]


def nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(exe).exists():
        raise RuntimeError("nvcc not found")
    return exe


def sources():
    return sorted(CSRC.glob("*.cu"))


def headers():
    return sorted(list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh")) + [HERE.parent / "include" / "tsne_h2pack.h"])


def _compile(src, obj, verbose):
    cmd = [nvcc()] + ARCH + FLAGS + ["-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name}:\n{r.stdout}\n{r.stderr}")
    return r.stderr


def build(jobs=None, verbose=False, force=False):
    BUILD.mkdir(exist_ok=True)
    OUT_DIR.mkdir(parents=True, exist_ok=True)
    hdr_mtime = max(p.stat().st_mtime for p in headers())
    todo = []
    objs = []
    for src in sources():
        obj = BUILD / (src.stem + ".o")
        objs.append(obj)
        if force or not obj.exists() or obj.stat().st_mtime < max(src.stat().st_mtime, hdr_mtime):
            todo.append((src, obj))
    with cf.ThreadPoolExecutor(max_workers=jobs or os.cpu_count() or 4) as ex:
        for msg in ex.map(lambda a: _compile(a[0], a[1], verbose), todo):
            if msg and verbose:
                print(msg)
    if todo or not OUT.exists():
        cmd = [nvcc()] + ARCH + ["-shared", "-cudart=static", "-o", str(OUT)] + [str(o) for o in objs]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    return OUT


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    a = ap.parse_args()
    print(build(a.jobs, a.verbose, a.force))
