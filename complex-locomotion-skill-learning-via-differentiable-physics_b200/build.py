"""Build the sm_100a shared library ``lib/libcls_b200.so`` in-tree with nvcc.

The library is a plain C ABI (``include/cls_b200.h``); it links the CUDA
runtime statically so it loads on a machine without a GPU (for symbol checks).
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIB_DIR = os.path.join(HERE, "lib")
LIB = os.path.join(LIB_DIR, "libcls_b200.so")
SOURCES = ["ms_runtime.cu", "ms_dense.cu", "ms_env.cu", "mpm_runtime.cu", "noalloc.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]
OBJ_DIR = os.path.join(HERE, "_build")


def _inputs():
    files = []
    for name in os.listdir(CSRC):
        if name.endswith((".cu", ".cuh", ".h")):
            files.append(os.path.join(CSRC, name))
    files.append(os.path.join(HERE, "..", "include", "cls_b200.h"))
    return files


def needs_build():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.exists(f) and os.path.getmtime(f) > t for f in _inputs())


def build(force=False, verbose=False):
    """Compile every CUDA source (in parallel, one nvcc per file) and link
    them into one shared library (sm_100a only)."""
    if not force and not needs_build():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    os.makedirs(LIB_DIR, exist_ok=True)
    os.makedirs(OBJ_DIR, exist_ok=True)
    srcs = [os.path.join(CSRC, s) for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]
    nvcc = os.environ.get("NVCC", "nvcc")
    objs = [os.path.join(OBJ_DIR, os.path.basename(s)[:-3] + ".o") for s in srcs]

    def compile_one(src_obj):
        src, obj = src_obj
        cmd = [nvcc, *ARCH, *FLAGS, "-c", "-o", obj, src]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.check_call(cmd)

    with ThreadPoolExecutor(max_workers=len(srcs)) as ex:
        list(ex.map(compile_one, zip(srcs, objs)))
    tmp = LIB + ".tmp"
    cmd = [nvcc, *ARCH, "-shared", "-o", tmp, *objs]
    if verbose:
        print(" ".join(cmd), file=sys.stderr)
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
