"""Writes the golden fixtures taken from the reference into tests/golden/.

* The reference's NEST membrane-potential traces (python/test/test_*_nest.txt
  of golosio/NeuronGPU): two columns, time in ms and V_m in mV, recorded by
  NEST for the single-neuron test networks of python/test/test_aeif_*.py,
  test_iaf_psc_exp.py, test_iaf_psc_exp_g.py / test_iaf_psc_exp_hc.py
  (fast_iaf_psc_exp) and test_izh.py (izh); copied unchanged. They are the
  only external golden vectors for the hot path.
* The names of the reference's C ABI (the functions src/neurongpu_C.h
  declares) and of the public functions of pythonlib/neurongpu.py, one per
  line: the interface a drop-in replacement has to cover.

The tests read only these files, so they run where the reference is absent.

Usage: python tests/golden/make_golden.py REFERENCE_ROOT
       (or with the root in the environment variable NGB200_REFERENCE_DIR)
"""
import os
import re
import shutil
import sys

NAMES = ["aeif_cond_beta", "aeif_cond_alpha", "aeif_psc_alpha", "aeif_psc_exp",
         "aeif_psc_delta", "iaf_psc_exp", "fast_iaf_psc_exp", "izh"]


def main(ref):
    here = os.path.dirname(os.path.abspath(__file__))
    for n in NAMES:
        src = os.path.join(ref, "python", "test", "test_%s_nest.txt" % n)
        dst = os.path.join(here, "nest_%s.txt" % n)
        shutil.copyfile(src, dst)
        print(dst)
    hdr = open(os.path.join(ref, "src", "neurongpu_C.h")).read()
    abi = sorted(set(re.findall(r"\b(NeuronGPU_[A-Za-z0-9]+)\s*\(", hdr)))
    with open(os.path.join(here, "reference_c_abi.txt"), "w") as f:
        f.write("\n".join(abi) + "\n")
    py = open(os.path.join(ref, "pythonlib", "neurongpu.py")).read()
    api = sorted(set(re.findall(r"^def ([A-Za-z][A-Za-z0-9_]*)\(", py, re.M)))
    with open(os.path.join(here, "reference_pylib_api.txt"), "w") as f:
        f.write("\n".join(api) + "\n")
    print(len(abi), "C ABI names,", len(api), "Python functions")


if __name__ == "__main__":
    root = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("NGB200_REFERENCE_DIR")
    if not root:
        sys.exit("usage: make_golden.py REFERENCE_ROOT (or set NGB200_REFERENCE_DIR)")
    main(root)
