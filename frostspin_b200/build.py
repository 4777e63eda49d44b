"""Build recipe for the frostspin_b200 CUDA library (sm_100a only).

Compiles every ``csrc/*.cu`` into ``_lib/libfrostspin_b200.so`` in-tree with
nvcc, one object per source, then links a shared library exposing the C ABI
declared in ``include/frostspin_b200.h``.  Run ``python -m frostspin_b200.build``
or call :func:`build`.  nvcc cross-compiles without a GPU.
"""

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
REPO_DIR = os.path.dirname(PKG_DIR)
CSRC_DIR = os.path.join(PKG_DIR, "csrc")
LIB_DIR = os.path.join(PKG_DIR, "_lib")
OBJ_DIR = os.path.join(LIB_DIR, "obj")
LIB_NAME = "libfrostspin_b200.so"
LIB_PATH = os.path.join(LIB_DIR, LIB_NAME)
INCLUDE_DIR = os.path.join(REPO_DIR, "include")

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-O3",
    "-lineinfo",
    "-std=c++17",
    "-Xcompiler",
    "-fPIC",
    "--expt-relaxed-constexpr",
    "-Xptxas",
    "-warn-spills",
]


def _nvcc():
    cuda_home = os.environ.get("CUDA_HOME", "/usr/local/cuda")
    cand = os.path.join(cuda_home, "bin", "nvcc")
    if os.path.exists(cand):
        return cand
    found = shutil.which("nvcc")
    if found is None:
        raise RuntimeError("nvcc not found: set CUDA_HOME")
    return found


def _sources():
    return sorted(
        os.path.join(CSRC_DIR, f) for f in os.listdir(CSRC_DIR) if f.endswith(".cu")
    )


def _headers():
    hs = [os.path.join(INCLUDE_DIR, f) for f in os.listdir(INCLUDE_DIR)]
    hs += [
        os.path.join(CSRC_DIR, f) for f in os.listdir(CSRC_DIR) if f.endswith(".cuh")
    ]
    return hs


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src, verbose):
    obj = os.path.join(OBJ_DIR, os.path.basename(src)[:-3] + ".o")
    if not _stale(obj, [src, *_headers()]):
        return obj
    cmd = [
        _nvcc(),
        *ARCH_FLAGS,
        *NVCC_FLAGS,
        "-I",
        INCLUDE_DIR,
        "-c",
        src,
        "-o",
        obj,
    ]
    if verbose:
        print(" ".join(cmd), flush=True)
    res = subprocess.run(cmd, capture_output=True, text=True, check=False)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src}:\n{res.stdout}\n{res.stderr}")
    if verbose and res.stderr.strip():
        print(res.stderr, file=sys.stderr)
    return obj


def build(*, verbose=False, force=False):
    """Compile the CUDA library if any source or header is newer than it."""
    os.makedirs(OBJ_DIR, exist_ok=True)
    srcs = _sources()
    if force:
        for f in os.listdir(OBJ_DIR):
            os.remove(os.path.join(OBJ_DIR, f))
    with ThreadPoolExecutor(max_workers=min(8, len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), srcs))
    if force or _stale(LIB_PATH, objs):
        cmd = [
            _nvcc(),
            *ARCH_FLAGS,
            "-shared",
            "-o",
            LIB_PATH,
            *objs,
            "-cudart",
            "static",
        ]
        if verbose:
            print(" ".join(cmd), flush=True)
        res = subprocess.run(cmd, capture_output=True, text=True, check=False)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stdout}\n{res.stderr}")
    return LIB_PATH


if __name__ == "__main__":
    print(build(verbose=True, force="--force" in sys.argv))
