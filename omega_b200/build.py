"""Build recipe of the native library ``omega_b200/lib/libomega_b200.so``.

Compiles every ``omega_b200/csrc/*.cu`` for sm_100a with nvcc and links one
shared library exporting the C-ABI of ``include/omega_b200.h``.  Runs without
a GPU (nvcc cross-compiles).  ``python -m omega_b200.build`` rebuilds when a
source is newer than the library.
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "omega_b200", "csrc")
INCLUDE = os.path.join(ROOT, "include")
OUT_DIR = os.path.join(ROOT, "omega_b200", "lib")
OBJ_DIR = os.path.join(ROOT, "_build")
LIB = os.path.join(OUT_DIR, "libomega_b200.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O3", "--expt-relaxed-constexpr",
         "-Xptxas", "-O3", "-I", INCLUDE, "-I", CSRC]
# Per-file flags.  orth.cu: no multiply-add contraction -- the tube tracer
# takes its walk steps, and with them the TOF weights of each scanned slice,
# from exact comparisons of crossing parameters, which tie on rays through
# voxel corners; without contraction they round exactly as the FP64
# restatement's do.
FILE_FLAGS = {"orth.cu": ["-fmad=false"]}


def _sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    return hs


def _mtime(p):
    return os.path.getmtime(p) if os.path.exists(p) else 0.0


def needs_build() -> bool:
    if not os.path.exists(LIB):
        return True
    t = _mtime(LIB)
    return any(_mtime(p) > t for p in _sources() + _headers() + [__file__])


def build(force: bool = False, verbose: bool = False, ptxas_info: bool = False) -> str:
    """Compile the library; returns its path.  Raises RuntimeError on failure."""
    if not force and not needs_build():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    newest_header = max((_mtime(h) for h in _headers()), default=0.0)

    def compile_one(src):
        obj = os.path.join(OBJ_DIR, os.path.basename(src) + ".o")
        if not force and _mtime(obj) > max(_mtime(src), newest_header, _mtime(__file__)):
            return obj, ""
        cmd = [NVCC, *ARCH, *FLAGS, *FILE_FLAGS.get(os.path.basename(src), []), "-c", src, "-o", obj]
        if ptxas_info:
            cmd += ["-Xptxas", "-v"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed on {os.path.basename(src)}:\n{r.stdout}\n{r.stderr}")
        return obj, r.stdout + r.stderr

    with ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(compile_one, _sources()))
    if verbose:
        for _, log in results:
            if log:
                print(log)
    objs = [o for o, _ in results]
    tmp = LIB + ".tmp"
    cmd = [NVCC, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    force = "--force" in sys.argv
    print(build(force=force, verbose=True, ptxas_info="--ptxas-info" in sys.argv))
