"""Builds the FP64 CPU oracle (test infrastructure) into oracle/lib/.

Usage: python oracle/build_oracle.py
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "ngpu_oracle.cpp")
LIB = os.path.join(HERE, "lib", "libngpu_oracle.so")


def build(force=False):
    os.makedirs(os.path.dirname(LIB), exist_ok=True)
    deps = [SRC, os.path.join(HERE, "..", "neurongpu_b200", "csrc", "ngpu_rng.h")]
    if (not force and os.path.exists(LIB)
            and os.path.getmtime(LIB) >= max(os.path.getmtime(d) for d in deps)):
        return LIB
    cmd = ["g++", "-O2", "-std=c++17", "-fPIC", "-shared", "-ffp-contract=off", "-fopenmp",
           SRC, "-o", LIB]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stderr)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
