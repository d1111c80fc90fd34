"""Build the flexmm_b200 CUDA library in-tree for sm_100a.

    python -m flexmm_b200.build

compiles each ``flexmm_b200/csrc/*.cu`` with nvcc into an object under
``flexmm_b200/_lib/obj`` (in parallel, each only when it or a header is newer
than its object) and links them into ``flexmm_b200/_lib/libflexmm_b200.so``.
"""
import glob
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
OBJ_DIR = os.path.join(OUT_DIR, "obj")
LIB = os.path.join(OUT_DIR, "libflexmm_b200.so")
INCLUDE = os.path.join(os.path.dirname(HERE), "include")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "-Xcompiler", "-fPIC"]

LINK = []


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def headers():
    return sorted(glob.glob(os.path.join(CSRC, "*.cuh"))) + \
        sorted(glob.glob(os.path.join(INCLUDE, "*.h")))


def deps():
    return sources() + headers()


def _obj(src):
    return os.path.join(OBJ_DIR, os.path.basename(src)[:-3] + ".o")


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in deps())


def build(force=False, verbose=False):
    if not force and up_to_date():
        return LIB
    os.makedirs(OBJ_DIR, exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    th = max([os.path.getmtime(h) for h in headers()] + [0.0])

    def stale(src):
        o = _obj(src)
        return force or not os.path.exists(o) or \
            os.path.getmtime(o) < max(th, os.path.getmtime(src))

    def compile_one(src):
        o = _obj(src)
        cmd = [nvcc] + NVCC_FLAGS + ["-I", INCLUDE, "-c", src, "-o", o + ".tmp"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.check_call(cmd)
        os.replace(o + ".tmp", o)

    todo = [s for s in sources() if stale(s)]
    if todo:
        with ThreadPoolExecutor(max_workers=min(len(todo), os.cpu_count() or 4)) as ex:
            list(ex.map(compile_one, todo))
    tmp = LIB + ".tmp"
    # -z defs: an unresolved symbol fails the build instead of the first load
    cmd = [nvcc] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-Xlinker", "-z,defs"] + \
        [_obj(s) for s in sources()] + ["-o", tmp] + LINK
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.check_call(cmd)
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose=True))
