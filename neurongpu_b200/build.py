"""Builds libneurongpu.so (sm_100a CUDA kernels + C++ host driver + C ABI).

The library is built in-tree at neurongpu_b200/lib/libneurongpu.so so that
the copy of the repository that runs on a GPU machine carries it.

Usage:  python -m neurongpu_b200.build [--force] [--verbose]
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
LIBDIR = os.path.join(HERE, "lib")
OBJDIR = os.path.join(HERE, "lib", "obj")
LIB = os.path.join(LIBDIR, "libneurongpu.so")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CUDA_HOME = os.environ.get("CUDA_HOME", "/usr/local/cuda")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

CU_SOURCES = ["ngpu_kernels.cu", "ngpu_rk5_aeif_cond_beta.cu", "ngpu_rk5_aeif_cond_alpha.cu",
              "ngpu_rk5_aeif_psc.cu", "ngpu_rk5_izh_cond_beta.cu", "ngpu_rk5_batch.cu",
              "ngpu_step_proposer.cu", "ngpu_connect_device.cu", "ngpu_deliver_api.cu",
              "ngpu_deliver_static.cu", "ngpu_remote.cu"]
CPP_SOURCES = ["ngpu_core.cpp", "ngpu_connect.cpp", "neurongpu_C.cpp"]


def _headers_mtime():
    m = 0.0
    for d in (CSRC, os.path.join(HERE, "..", "include")):
        for f in os.listdir(d):
            if f.endswith((".h", ".cuh")):
                m = max(m, os.path.getmtime(os.path.join(d, f)))
    return m


def _compile(src, force, verbose):
    path = os.path.join(CSRC, src)
    obj = os.path.join(OBJDIR, src + ".o")
    if (not force and os.path.exists(obj)
            and os.path.getmtime(obj) >= max(os.path.getmtime(path), _headers_mtime())):
        return obj
    if src.endswith(".cu"):
        cmd = [NVCC] + ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                               "--expt-relaxed-constexpr", "-c", path, "-o", obj]
        if verbose:
            cmd += ["-Xptxas", "-v"]
    else:
        cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-fopenmp", "-ffp-contract=off",
               "-I" + os.path.join(CUDA_HOME, "include"), "-c", path, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compile failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))
    if verbose and r.stderr:
        sys.stderr.write(r.stderr)
    return obj


def build(force=False, verbose=False):
    """Compiles every source and links the shared library; returns its path."""
    os.makedirs(OBJDIR, exist_ok=True)
    srcs = CU_SOURCES + CPP_SOURCES
    with ThreadPoolExecutor(max_workers=min(max(os.cpu_count() or 1, 1), len(srcs))) as ex:
        objs = list(ex.map(lambda s: _compile(s, force, verbose), srcs))
    if (force or not os.path.exists(LIB)
            or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs)):
        cmd = ["g++", "-shared", "-fopenmp", "-o", LIB] + objs + [
            "-L" + os.path.join(CUDA_HOME, "lib64"), "-lcudart", "-Wl,-rpath," + os.path.join(CUDA_HOME, "lib64")]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed: %s\n%s" % (r.stdout, r.stderr))
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="--verbose" in sys.argv))
