"""Build recipe for the CPU oracle (test infrastructure).

Compiles oracle/oracle_capi.cpp into oracle/_build/liboracle.so with g++,
OpenMP and -ffp-contract=off (the oracle's neighbor test depends on the
written operation order).  The reference itself is not built: its headers
require Eigen, GLFW and glm, none of which exist in this image.

Usage: python oracle/build.py [--force]
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
OUT_DIR = os.path.join(HERE, "_build")
LIB = os.path.join(OUT_DIR, "liboracle.so")
SOURCES = [os.path.join(HERE, "oracle_capi.cpp")]
HEADERS = [os.path.join(HERE, "sph_oracle.hpp"),
           os.path.join(ROOT, "include", "alluvion_b200.h")]


def _stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(p) > t for p in SOURCES + HEADERS)


def build(force=False):
    """Compile the oracle library if it is missing or out of date; return its path."""
    if not force and not _stale():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    cmd = ["g++", "-std=c++17", "-O3", "-march=x86-64-v3", "-ffp-contract=off",
           "-fopenmp", "-fPIC", "-shared", "-I", os.path.join(ROOT, "include"),
           *SOURCES, "-o", LIB + ".tmp"]
    subprocess.run(cmd, check=True)
    os.replace(LIB + ".tmp", LIB)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
