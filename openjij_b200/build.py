"""Build recipes for the native parts of openjij_b200.

* ``libojb200.so`` — every CUDA source under csrc/ compiled for sm_100a
  (``-gencode arch=compute_100a,code=sm_100a``), the C ABI of
  include/openjij_b200.h, CUDA runtime linked statically.
* ``_cxxjij*.so`` — the pybind11 host module (csrc/cxxjij_host.cpp) that keeps
  OpenJij's ``cxxjij`` Python surface and calls the C ABI.

Both are written next to this file (in-tree), so they travel with the source.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
ROOT = os.path.dirname(HERE)
INCLUDE = os.path.join(ROOT, "include")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libojb200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
              "-I" + INCLUDE, "-I" + CSRC]


def _run(cmd, verbose):
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)


def _stale(target, sources):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(s) > t for s in sources)


def build_cuda(verbose=False, force=False, extra=()):
    os.makedirs(BUILD, exist_ok=True)
    headers = glob.glob(os.path.join(CSRC, "*.cuh")) + glob.glob(os.path.join(CSRC, "*.h")) + \
        [os.path.join(INCLUDE, "openjij_b200.h")]
    objs, jobs = [], []
    for cu in sorted(glob.glob(os.path.join(CSRC, "*.cu"))):
        obj = os.path.join(BUILD, os.path.basename(cu) + ".o")
        if force or _stale(obj, [cu] + headers):
            jobs.append([NVCC] + ARCH + NVCC_FLAGS + list(extra) + ["-c", cu, "-o", obj])
        objs.append(obj)
    # one nvcc per source, as many at once as there are cores
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, os.cpu_count() or 1)) as pool:
        for f in [pool.submit(_run, cmd, verbose) for cmd in jobs]:
            f.result()
    if force or _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs +
             ["-Xlinker", "-rpath,$ORIGIN"], verbose)
    return LIB


def host_module_path():
    return os.path.join(HERE, "_cxxjij" + sysconfig.get_config_var("EXT_SUFFIX"))


def build_host(verbose=False, force=False):
    import pybind11
    src = os.path.join(CSRC, "cxxjij_host.cpp")
    out = host_module_path()
    deps = [src, os.path.join(INCLUDE, "openjij_b200.h"), LIB]
    if not (force or _stale(out, deps)):
        return out
    cxx = os.environ.get("CXX", "g++")
    cmd = [cxx, "-O3", "-std=c++17", "-shared", "-fPIC", "-fvisibility=hidden",
           "-I" + pybind11.get_include(), "-I" + sysconfig.get_paths()["include"], "-I" + INCLUDE,
           src, "-o", out, "-L" + HERE, "-lojb200", "-Wl,-rpath,$ORIGIN"]
    _run(cmd, verbose)
    return out


def build_all(verbose=False, force=False):
    build_cuda(verbose=verbose, force=force)
    if os.path.exists(os.path.join(CSRC, "cxxjij_host.cpp")):
        build_host(verbose=verbose, force=force)


if __name__ == "__main__":
    build_all(verbose=True, force="--force" in sys.argv)
