"""The reference's own Python binding over this library (no GPU needed).

The reference's pythonlib/neurongpu.py is loaded unchanged except for the
library path it opens (line 17, `lib_path=...`, the one line a user
switching libraries edits), pointed at neurongpu_b200/lib/libneurongpu.so.
At import it looks up every C function it wraps through ctypes, so a
missing or renamed entry point fails the import; it also sets the
exception mode, which this library must accept. Then its kernel-parameter
functions run through our C ABI, and a compute call raises the
reference's ValueError with our message (no CPU fallback exists).

The reference checkout is read from NGB200_REFERENCE_DIR; without it (for
instance on a machine that has only this repository) the test is skipped.
"""
import os
import re
import types

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "neurongpu_b200", "lib", "libneurongpu.so")


def _reference_binding():
    ref = os.environ.get("NGB200_REFERENCE_DIR")
    if not ref:
        pytest.skip("NGB200_REFERENCE_DIR is not set")
    path = os.path.join(ref, "pythonlib", "neurongpu.py")
    if not os.path.exists(path):
        pytest.skip("no pythonlib/neurongpu.py under NGB200_REFERENCE_DIR")
    src = open(path).read()
    src, n = re.subn(r'^lib_path\s*=.*$', 'lib_path=%r' % LIB, src, count=1, flags=re.M)
    assert n == 1, "the reference binding's lib_path line was not found"
    mod = types.ModuleType("neurongpu_reference_binding")
    mod.__file__ = path
    exec(compile(src, path, "exec"), mod.__dict__)
    return mod


def test_reference_binding_loads_our_library():
    ng = _reference_binding()
    try:
        _check(ng)
    finally:
        # the library keeps one simulator per process (as the reference's
        # does): leave it fresh for the other tests
        ng._neurongpu.NGB200_Reset()


def _check(ng):
    assert os.path.samefile(ng._neurongpu._name, LIB)
    # kernel parameters through the reference's wrappers and our C ABI
    assert abs(ng.GetTimeResolution() - 0.1) < 1e-6
    ng.SetKernelStatus("rnd_seed", 1234)
    assert ng.GetKernelStatus("rnd_seed") == 1234
    st = ng.GetKernelStatus()
    assert "max_spike_buffer_size" in st and "verbosity_level" in st
    import torch
    if not torch.cuda.is_available():
        # the compute path fails loudly, in the reference's error convention
        with pytest.raises(ValueError):
            ng.Create("aeif_cond_beta", 10, 2)
        assert ng.GetErrorCode() == 2
