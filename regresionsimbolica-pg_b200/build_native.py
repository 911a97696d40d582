"""Build recipes for the native pieces: libwarpsym.so (product) and the CPU oracle (tests).

libwarpsym.so is compiled for sm_100a only, with the reference's floating-point flags
(-O3 --use_fast_math, src/warpsymbolic/gpu/cuda/setup.py:35) so that per-operation results are
bit-identical to the reference evaluator.  Objects are rebuilt when a source or header is newer.
"""
from __future__ import annotations

import concurrent.futures as cf
import glob
import os
import shutil
import subprocess

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
REPO_DIR = os.path.dirname(PKG_DIR)
CSRC = os.path.join(PKG_DIR, "csrc")
BUILD_DIR = os.path.join(PKG_DIR, "_build")
LIB_PATH = os.path.join(PKG_DIR, "libwarpsym.so")
# the bounds-checked build (-DWS_BOUNDS_CHECK): same sources, kernels record out-of-range
# indices instead of faulting (csrc/ws_bounds.cuh)
BC_BUILD_DIR = os.path.join(PKG_DIR, "_build_bc")
BC_LIB_PATH = os.path.join(PKG_DIR, "libwarpsym_bc.so")
ORACLE_DIR = os.path.join(REPO_DIR, "oracle")
ORACLE_LIB = os.path.join(ORACLE_DIR, "libws_oracle.so")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "--use_fast_math", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
              "-Xptxas", "-warn-spills", "-I", os.path.join(REPO_DIR, "include")]


def _newest(paths):
    return max((os.path.getmtime(p) for p in paths), default=0.0)


def _run(cmd):
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError("command failed: %s\n%s%s" % (" ".join(cmd), res.stdout, res.stderr))
    return res.stdout + res.stderr


def build_native(verbose: bool = False, jobs: int = 8, bounds_check: bool = False) -> str:
    """Compiles csrc/*.cu into libwarpsym.so (sm_100a), or with bounds_check into
    libwarpsym_bc.so.  Returns the library path."""
    build_dir = BC_BUILD_DIR if bounds_check else BUILD_DIR
    lib_path = BC_LIB_PATH if bounds_check else LIB_PATH
    flags = NVCC_FLAGS + (["-DWS_BOUNDS_CHECK"] if bounds_check else [])
    os.makedirs(build_dir, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        glob.glob(os.path.join(REPO_DIR, "include", "*.h")) + [os.path.abspath(__file__)]
    hdr_time = _newest(headers)
    objs, todo = [], []
    for src in sources:
        obj = os.path.join(build_dir, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        if not os.path.exists(obj) or os.path.getmtime(obj) < max(os.path.getmtime(src), hdr_time):
            todo.append((src, obj))

    def compile_one(pair):
        src, obj = pair
        return _run([NVCC, "-c", src, "-o", obj] + ARCH + flags)

    if todo:
        with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
            for out in ex.map(compile_one, todo):
                if verbose and out.strip():
                    print(out)
    if todo or not os.path.exists(lib_path) or os.path.getmtime(lib_path) < _newest(objs):
        _run([NVCC, "-shared", "-o", lib_path] + objs + ARCH + ["-lcudart"])
    return lib_path


def build_oracle() -> str:
    """Compiles the CPU oracle (test infrastructure) into oracle/libws_oracle.so."""
    srcs = sorted(glob.glob(os.path.join(ORACLE_DIR, "*.cpp")))
    deps = srcs + [os.path.join(REPO_DIR, "include", "warpsym.h")]
    if not os.path.exists(ORACLE_LIB) or os.path.getmtime(ORACLE_LIB) < _newest(deps):
        _run(["g++", "-O2", "-std=c++17", "-fopenmp", "-fPIC", "-shared", "-ffp-contract=off",
              "-fno-fast-math"] + srcs + ["-o", ORACLE_LIB])
    return ORACLE_LIB


def build_reference_checker(ref_root: str) -> None:
    """Builds the reference extension from its sources in the checkout `ref_root` into
    oracle/_ref (test infrastructure), and installs the reference's Python package into
    baseline/_ref when it is not there yet.  Nothing happens when the checkout is absent (GPU
    boxes use the copies built here)."""
    if not ref_root or not os.path.isdir(os.path.join(ref_root, "src")):
        return
    _run(["bash", os.path.join(ORACLE_DIR, "build_ref.sh"), ref_root])
    if not os.path.isdir(os.path.join(REPO_DIR, "baseline", "_ref", "warpsymbolic")):
        _run(["bash", os.path.join(REPO_DIR, "baseline", "install_ref.sh"), ref_root])


if __name__ == "__main__":
    print(build_native(verbose=True))
    print(build_oracle())
