"""Builds libwar.so (the sm_100a engine) in place with nvcc.

    python build.py            compile if any source is newer than the library
    python build.py --force    always compile
    python build.py --verbose  also print ptxas register / spill / shared-memory use

Each .cu file under csrc/ is compiled for sm_100a (-gencode arch=compute_100a,code=sm_100a) and the
objects are linked into csrc/../libwar.so, next to this file.
"""
import glob
import os
import subprocess
import sys
import concurrent.futures as cf

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libwar.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
         "--expt-relaxed-constexpr", "-I" + os.path.join(HERE, "..", "include")]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def headers():
    return sorted(glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) +
                  glob.glob(os.path.join(HERE, "..", "include", "*.h")))


def stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(f) > t for f in sources() + headers() + [__file__])


def compile_one(src, verbose):
    obj = os.path.join(BUILD, os.path.basename(src)[:-3] + ".o")
    cmd = [NVCC] + ARCH + FLAGS + (["-Xptxas", "-v"] if verbose else []) + ["-c", src, "-o", obj]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError("nvcc failed for %s:\n%s%s" % (src, p.stdout, p.stderr))
    return obj, p.stderr


def build(force=False, verbose=False):
    if not force and not stale():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(lambda s: compile_one(s, verbose), sources()))
    if verbose:
        for obj, log in results:
            sys.stdout.write(log)
    objs = [o for o, _ in results]
    tmp = LIB + ".tmp"
    cmd = [NVCC] + ARCH + ["-shared", "-o", tmp] + objs + ["-lcudart"]
    p = subprocess.run(cmd, capture_output=True, text=True)
    if p.returncode != 0:
        raise RuntimeError("link failed:\n%s%s" % (p.stdout, p.stderr))
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv))
