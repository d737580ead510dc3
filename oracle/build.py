"""Build the oracle (CPU restatement used only as the checker) into
``oracle/_build/liboracle.so``.

Flags: ``-fwrapv`` (Rust release integer wrap), ``-ffp-contract=off`` (no
implicit FMA: the AVX2 FMA sites of the reference are explicit ``fmaf`` calls),
``-fno-fast-math``.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "liboracle.so")
FLAGS = ["-O2", "-std=c++17", "-fPIC", "-shared", "-fwrapv", "-ffp-contract=off", "-fno-fast-math", "-pthread"]


def sources():
    return sorted(os.path.join(HERE, f) for f in os.listdir(HERE) if f.endswith(".cpp"))


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(HERE, f) for f in os.listdir(HERE) if f.endswith((".cpp", ".h"))]
    deps.append(os.path.join(HERE, "..", "include", "maroontree_b200.h"))
    deps.append(os.path.join(HERE, "..", "maroontree_b200", "csrc", "av1_tables.h"))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False):
    if not force and not _stale():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = [os.environ.get("CXX", "g++"), *FLAGS, "-o", LIB + ".tmp", *sources()]
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
