"""The drop-in boundary on a machine without a GPU: the C-ABI library loads,
exports every entry point declared in include/neurongpu_C.h, keeps the
reference's error convention, and the Python layer mirrors the reference's
public functions. No compute call is made."""
import ctypes
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "neurongpu_b200", "lib", "libneurongpu.so")
HDR = os.path.join(ROOT, "include", "neurongpu_C.h")

GOLDEN = os.path.join(ROOT, "tests", "golden")


def _golden_names(fname):
    """Names the reference exports (written by tests/golden/make_golden.py)."""
    with open(os.path.join(GOLDEN, fname)) as f:
        return [ln.strip() for ln in f if ln.strip()]


# public functions of the reference's pythonlib/neurongpu.py
REFERENCE_PY_API = _golden_names("reference_pylib_api.txt")


def declared_symbols():
    txt = open(HDR).read()
    return sorted(set(re.findall(r"\b((?:NeuronGPU|NGB200)_[A-Za-z0-9]+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    assert os.path.exists(LIB), "build the library first (python -m neurongpu_b200.build)"
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True,
                         text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    decl = declared_symbols()
    assert len(decl) > 130
    missing = [s for s in decl if s not in exported]
    assert not missing, missing
    lib = ctypes.CDLL(LIB)
    for s in decl:
        assert hasattr(lib, s)


def test_reference_c_abi_is_covered():
    """Every entry point of the reference's neurongpu_C.h is declared here."""
    names = set(_golden_names("reference_c_abi.txt"))
    assert len(names) == 126
    assert names <= set(declared_symbols())


def test_python_api_mirrors_reference():
    from neurongpu_b200 import neurongpu as api
    assert len(REFERENCE_PY_API) == 126
    for name in REFERENCE_PY_API:
        assert hasattr(api.Binding, name) or hasattr(api, name), name
    assert api.NodeSeq(5, 10)[2:4].ToList() == [7, 8]
    assert api.NodeSeq(5, 10)[-1] == 14
    with pytest.raises(ValueError):
        api.NodeSeq(0, 3)[3]


def test_kernel_params_and_error_convention_without_gpu():
    from neurongpu_b200 import neurongpu as api
    b = api.default_binding()
    st = api.GetKernelStatus()
    assert st["time_resolution"] == pytest.approx(0.1)
    assert st["max_spike_buffer_size"] == 20 and st["rnd_seed"] == 54321
    with pytest.raises(ValueError):
        api.SetKernelStatus("no_such_param", 1)
    # compute calls fail loudly without a device: no CPU fallback exists
    import torch
    if not torch.cuda.is_available():
        with pytest.raises(ValueError):
            api.Create("aeif_cond_beta", 10, 2)
        assert b.GetErrorCode() == 2
    # hosts of a partitioned network: without a launcher, host 0 of 1; an
    # invalid host index is an error with the reference's code
    assert api.MpiId() == 0 and api.MpiNp() == 1 and api.ProcMaster() == 1
    with pytest.raises(ValueError):
        b.SetHost(2, 2)
    assert b.GetErrorCode() == 2


def test_graft_build_entry_exists():
    import importlib.util
    spec = importlib.util.spec_from_file_location("ge", os.path.join(ROOT, "__graft_entry__.py"))
    m = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(m)
    assert callable(m.build) and callable(m.smoke)
