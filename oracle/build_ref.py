"""Builds the reference library (golosio/NeuronGPU) for sm_100a into oracle/_ref/.

Test infrastructure only: the product never loads this library. It is the
GPU-side reference baseline that bench.py times beside the B200 core on the
same GPU (`reference_gpu` in the bench line).

Recipe (the reference's own autotools build needs MPI and a generated
config.h, neither of which exists here):
  * the sources are the ones `Makefile.am:93-138` lists (`ngpu_src_files`),
    compiled where they lie in the reference tree, never copied;
  * flags follow `Makefile.am:139-151`: `-O3 -Wall -fPIC -fopenmp`,
    `--maxrregcount=55`, relocatable device code, `-lcurand`;
  * `oracle/ref_stub/config.h` defines HAVE_MPI (the single-GPU entry points
    are declared only under it, `src/neurongpu.cu:284,426,1093`) and
    `oracle/ref_stub/mpi.h` is a single-rank MPI stand-in;
  * `oracle/ref_harness.cu` is linked in to set the RK5 tolerance constant
    (`src/rk5.cu:55`) through the device link.
Each source is compiled separately (in parallel) and the objects are
device-linked into one shared library.

Usage: python oracle/build_ref.py [--force]
The reference tree is taken from NGB200_REFERENCE_DIR (default
/root/reference); without it the build is skipped.
"""
import os
import re
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
OBJ = os.path.join(OUT, "obj")
LIB = os.path.join(OUT, "libneurongpu_ref.so")
STUB = os.path.join(HERE, "ref_stub")
HARNESS = os.path.join(HERE, "ref_harness.cu")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def reference_dir():
    return os.environ.get("NGB200_REFERENCE_DIR", "/root/reference")


def source_list(ref):
    """Sources of the library as Makefile.am's `ngpu_src_files` lists them."""
    text = open(os.path.join(ref, "Makefile.am")).read()
    m = re.search(r"ngpu_src_files\s*=(.*?)(?:\n\s*\n)", text, re.S)
    if not m:
        raise RuntimeError("ngpu_src_files not found in Makefile.am")
    names = re.findall(r"\$\(top_srcdir\)/(src/[\w.]+)", m.group(1))
    return [os.path.join(ref, n) for n in names]


def _compile(src, force):
    obj = os.path.join(OBJ, os.path.basename(src) + ".o")
    deps = [src, os.path.join(STUB, "mpi.h"), os.path.join(STUB, "config.h")]
    if not force and os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(d) for d in deps):
        return obj
    src_dir = os.path.dirname(src)
    cmd = [NVCC, "-ccbin=g++", "--compiler-options", "-O3 -Wall -fPIC -fopenmp",
           "-I", STUB, "-I", src_dir] + ARCH + [
           "--maxrregcount=55", "--relocatable-device-code", "true",
           "-x", "cu", "-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("compile failed: %s\n%s" % (" ".join(cmd), r.stderr[-4000:]))
    return obj


def build(force=False, jobs=None):
    ref = reference_dir()
    if not os.path.isdir(os.path.join(ref, "src")):
        raise RuntimeError("reference tree not found at %s" % ref)
    os.makedirs(OBJ, exist_ok=True)
    srcs = source_list(ref) + [HARNESS]
    jobs = jobs or max(1, min(16, os.cpu_count() or 1))
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), srcs))
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC, "-ccbin=g++", "--compiler-options", "-fPIC -fopenmp"] + ARCH + [
               "--relocatable-device-code", "true", "--shared", "-o", LIB] + objs + ["-lm", "-lcurand"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n" + r.stderr[-4000:])
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
