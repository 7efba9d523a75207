"""In-tree build of the engine's native libraries (sm_100a only).

  alluvion_b200/liballuvion_b200.so   CUDA kernels + the C ABI of
                                      include/alluvion_b200.h (nvcc)
  alluvion_b200/_alluvion_b200*.so    pybind11 module: the reference's Python
                                      object model (Store, Pile, SolverDf, ...)
                                      over include/alluvion_b200_solver.hpp (g++)

Usage: python -m alluvion_b200.build [--force] [--verbose]
"""
import glob
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
INCLUDE = os.path.join(ROOT, "include")
ENGINE_DIR = os.path.join(PKG, "csrc", "engine")
ENGINE_LIB = os.path.join(PKG, "liballuvion_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")

NVCC_FLAGS = [
    "-std=c++17", "-O3", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
    "--expt-relaxed-constexpr",
]


def _newest(paths):
    return max((os.path.getmtime(p) for p in paths), default=0.0)


def engine_sources():
    return sorted(glob.glob(os.path.join(ENGINE_DIR, "*.cu")))


def engine_deps():
    return (engine_sources() + glob.glob(os.path.join(ENGINE_DIR, "*.cuh"))
            + glob.glob(os.path.join(ENGINE_DIR, "*.hpp"))
            + glob.glob(os.path.join(ENGINE_DIR, "*.h"))
            + [os.path.join(INCLUDE, "alluvion_b200.h")])


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def build_engine(force=False, verbose=False, ptxas_info=False):
    """Compiles every engine .cu into one shared library; returns its path."""
    if not force and os.path.exists(ENGINE_LIB) and \
            os.path.getmtime(ENGINE_LIB) >= _newest(engine_deps()):
        return ENGINE_LIB
    build_dir = os.path.join(PKG, "_build")
    os.makedirs(build_dir, exist_ok=True)
    objs = []
    jobs = []
    extra = ["-Xptxas", "-v"] if ptxas_info else []
    for src in engine_sources():
        obj = os.path.join(build_dir, os.path.basename(src) + ".o")
        if force or not os.path.exists(obj) or os.path.getmtime(obj) < _newest(
                [src] + engine_deps()[len(engine_sources()):]):
            jobs.append([NVCC, *NVCC_FLAGS, *extra, "-I", INCLUDE, "-I", ENGINE_DIR,
                         "-c", src, "-o", obj])
        objs.append(obj)
    # translation units are independent: compile them side by side
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as pool:
        for f in [pool.submit(_run, cmd, verbose) for cmd in jobs]:
            f.result()
    tmp = ENGINE_LIB + ".tmp"
    _run([NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", *objs,
          "-o", tmp, "-lcuda"], verbose)
    os.replace(tmp, ENGINE_LIB)
    return ENGINE_LIB


PY_SRC = os.path.join(PKG, "csrc", "py", "pyalluvion_b200.cpp")


def pymodule_path():
    import sysconfig
    return os.path.join(PKG, "_alluvion_b200" + sysconfig.get_config_var("EXT_SUFFIX"))


def build_pymodule(force=False, verbose=False):
    """Compiles the pybind11 module against liballuvion_b200.so (host code
    only: the C++ layer calls the C ABI); returns its path."""
    import sysconfig
    import pybind11
    out = pymodule_path()
    deps = [PY_SRC, ENGINE_LIB, os.path.join(INCLUDE, "alluvion_b200.h"),
            os.path.join(INCLUDE, "alluvion_b200.hpp"),
            os.path.join(INCLUDE, "alluvion_b200_solver.hpp")]
    if not force and os.path.exists(out) and os.path.getmtime(out) >= _newest(deps):
        return out
    tmp = out + ".tmp"
    _run([os.environ.get("CXX", "g++"), "-std=c++17", "-O2", "-shared", "-fPIC",
          "-fvisibility=hidden", "-I", INCLUDE, "-I", pybind11.get_include(),
          "-I", sysconfig.get_paths()["include"], PY_SRC, "-o", tmp,
          "-L", PKG, "-lalluvion_b200", "-Wl,-rpath,$ORIGIN"], verbose)
    os.replace(tmp, out)
    return out


def build_all(force=False, verbose=False):
    return [build_engine(force=force, verbose=verbose),
            build_pymodule(force=force, verbose=verbose)]


if __name__ == "__main__":
    for p in build_all(force="--force" in sys.argv, verbose="--verbose" in sys.argv):
        print(p)
