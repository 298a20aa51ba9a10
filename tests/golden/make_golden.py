"""Copies the reference's NEST membrane-potential traces into tests/golden/.

The traces ship with golosio/NeuronGPU (python/test/test_*_nest.txt): two
columns, time in ms and V_m in mV, recorded by NEST for the single-neuron
test networks of python/test/test_aeif_*.py, test_iaf_psc_exp.py,
test_iaf_psc_exp_g.py / test_iaf_psc_exp_hc.py (fast_iaf_psc_exp) and
test_izh.py (izh). They are
the only external golden vectors for the hot path. This script reads them
from a checkout of the reference (default /root/reference) and writes them
unchanged, so the tests can run where the reference is absent.

Usage: python tests/golden/make_golden.py [reference_root]
"""
import os
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


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
