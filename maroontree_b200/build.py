"""Build the sm_100a shared library in-tree.

``python -m maroontree_b200.build`` compiles ``csrc/*.cu`` with nvcc for
``sm_100a`` into ``maroontree_b200/_lib/libmaroontree_b200.so``.  Device code is
compiled with ``-fmad=false`` (the only fused multiply-adds are explicit
``__fmaf_rn`` calls) and host code with ``-ffp-contract=off`` so the float
order of the reference is kept on both sides.  Each translation unit is
compiled to an object of its own (in parallel, only the stale ones) and the
objects are linked into one library.
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT_DIR = os.path.join(HERE, "_lib")
OBJ_DIR = os.path.join(OUT_DIR, "obj")
LIB = os.path.join(OUT_DIR, "libmaroontree_b200.so")
HEADER = os.path.join(HERE, "..", "include", "maroontree_b200.h")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17",
    "-fmad=false", "--prec-div=true", "--prec-sqrt=true",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
    "-Xptxas", "-warn-spills",
]


def sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(".cu"))


def _headers_mtime():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".h"))]
    hs.append(HEADER)
    return max(os.path.getmtime(h) for h in hs)


def _obj(src):
    return os.path.join(OBJ_DIR, os.path.basename(src)[:-3] + ".o")


def _obj_stale(src, hdr_t):
    o = _obj(src)
    if not os.path.exists(o):
        return True
    t = os.path.getmtime(o)
    return os.path.getmtime(src) > t or hdr_t > t


def _stale():
    if not os.path.exists(LIB):
        return True
    hdr_t = _headers_mtime()
    return any(_obj_stale(s, hdr_t) for s in sources()) or any(
        os.path.getmtime(_obj(s)) > os.path.getmtime(LIB) for s in sources())


def build(force=False, verbose=False):
    if not force and not _stale():
        return LIB
    os.makedirs(OBJ_DIR, exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    hdr_t = _headers_mtime()
    todo = [s for s in sources() if force or _obj_stale(s, hdr_t)]

    def compile_one(src):
        o = _obj(src)
        cmd = [nvcc, *NVCC_FLAGS, "-c", "-o", o + ".tmp", src]
        if verbose:
            print(" ".join(cmd))
        subprocess.run(cmd, check=True)
        os.replace(o + ".tmp", o)

    jobs = max(1, min(len(todo), os.cpu_count() or 1))
    with cf.ThreadPoolExecutor(jobs) as ex:
        for f in [ex.submit(compile_one, s) for s in todo]:
            f.result()
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "--cudart=static",
           "-o", LIB + ".tmp", *[_obj(s) for s in sources()]]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True)
    print(LIB)
