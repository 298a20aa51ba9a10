"""Python interface of the B200 simulation core (ctypes over the C ABI).

Mirrors the public functions of the reference's ``pythonlib/neurongpu.py``
(golosio/NeuronGPU) -- same names, argument meaning, return formats and error
behaviour (a failed call raises ``ValueError`` with the library's message) --
so that scripts written as ``import neurongpu as ngpu`` run unchanged with::

    from neurongpu_b200 import neurongpu as ngpu

The functions are methods of :class:`Binding`; the module-level names are
bound to a default instance over ``libneurongpu.so`` from this package (or
the library named by the NEURONGPU_LIB environment variable). Because the
C ABI is the reference's, ``Binding(path)`` can also drive any library that
exports it.
"""
import ctypes
import gc
import os
import sys

c_float_p = ctypes.POINTER(ctypes.c_float)
c_int_p = ctypes.POINTER(ctypes.c_int)
c_char_p = ctypes.POINTER(ctypes.c_char)
c_void_p = ctypes.c_void_p

conn_rule_name = ("one_to_one", "all_to_all", "fixed_total_number",
                  "fixed_indegree", "fixed_outdegree")

_HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_LIB = os.path.join(_HERE, "lib", "libneurongpu.so")


class NodeSeq(object):
    """Contiguous range of node indices (reference pythonlib/neurongpu.py:25-57)."""

    def __init__(self, i0, n=1):
        if i0 is None:
            i0, n = 0, -1
        self.i0 = i0
        self.n = n

    def Subseq(self, first, last):
        if last < 0 and last >= -self.n:
            last = last % self.n
        if first < 0 or last < first:
            raise ValueError("Sequence subset range error")
        if last >= self.n:
            raise ValueError("Sequence subset out of range")
        return NodeSeq(self.i0 + first, last - first + 1)

    def __getitem__(self, i):
        if isinstance(i, slice):
            if i.step is not None:
                raise ValueError("Subsequence cannot have a step")
            start = 0 if i.start is None else i.start
            stop = self.n if i.stop is None else i.stop
            return self.Subseq(start, stop - 1)
        if i < -self.n:
            raise ValueError("Sequence index error")
        if i >= self.n:
            raise ValueError("Sequence index out of range")
        if i < 0:
            i = i % self.n
        return self.i0 + i

    def ToList(self):
        return list(range(self.i0, self.i0 + self.n))

    def __len__(self):
        return self.n


class RemoteNodeSeq(object):
    def __init__(self, i_host=0, node_seq=None):
        self.i_host = i_host
        self.node_seq = node_seq if node_seq is not None else NodeSeq(None)


class ConnectionId(object):
    def __init__(self, i_source, i_group, i_conn):
        self.i_source = i_source
        self.i_group = i_group
        self.i_conn = i_conn


class SynGroup(object):
    def __init__(self, i_syn_group):
        self.i_syn_group = i_syn_group


def to_byte_str(s):
    if isinstance(s, str):
        return s.encode("ascii")
    if isinstance(s, bytes):
        return s
    raise ValueError("Variable cannot be converted to string")


def to_def_str(s):
    return s.decode("utf-8")


def _cstr(s):
    b = to_byte_str(s)
    return ctypes.create_string_buffer(b, len(b) + 1)


def waitenter(val):
    "Print val and wait for the Enter key (as the reference's module does)"
    return input(val)


def _is_seq(x):
    return isinstance(x, (list, tuple, NodeSeq))


# C signatures: name -> (restype, argtypes)
_I, _F, _U = ctypes.c_int, ctypes.c_float, ctypes.c_ubyte
_SIG = {
    "GetErrorMessage": (c_char_p, ()),
    "GetErrorCode": (ctypes.c_ubyte, ()),
    "SetOnException": (None, (_I,)),
    "SetRandomSeed": (_I, (ctypes.c_ulonglong,)),
    "SetTimeResolution": (_I, (_F,)),
    "GetTimeResolution": (_F, ()),
    "SetMaxSpikeBufferSize": (_I, (_I,)),
    "GetMaxSpikeBufferSize": (_I, ()),
    "SetSimTime": (_I, (_F,)),
    "SetVerbosityLevel": (_I, (_I,)),
    "Create": (_I, (c_char_p, _I, _I)),
    "CreatePoissonGenerator": (_I, (_I, _F)),
    "CreateRecord": (_I, (c_char_p, ctypes.POINTER(c_char_p), c_int_p, c_int_p, _I)),
    "GetRecordDataRows": (_I, (_I,)),
    "GetRecordDataColumns": (_I, (_I,)),
    "GetRecordData": (ctypes.POINTER(c_float_p), (_I,)),
    "SetNeuronScalParam": (_I, (_I, _I, c_char_p, _F)),
    "SetNeuronArrayParam": (_I, (_I, _I, c_char_p, c_void_p, _I)),
    "SetNeuronPtScalParam": (_I, (c_void_p, _I, c_char_p, _F)),
    "SetNeuronPtArrayParam": (_I, (c_void_p, _I, c_char_p, c_void_p, _I)),
    "IsNeuronScalParam": (_I, (_I, c_char_p)),
    "IsNeuronPortParam": (_I, (_I, c_char_p)),
    "IsNeuronArrayParam": (_I, (_I, c_char_p)),
    "IsNeuronGroupParam": (_I, (_I, c_char_p)),
    "SetNeuronIntVar": (_I, (_I, _I, c_char_p, _I)),
    "SetNeuronScalVar": (_I, (_I, _I, c_char_p, _F)),
    "SetNeuronArrayVar": (_I, (_I, _I, c_char_p, c_void_p, _I)),
    "SetNeuronPtIntVar": (_I, (c_void_p, _I, c_char_p, _I)),
    "SetNeuronPtScalVar": (_I, (c_void_p, _I, c_char_p, _F)),
    "SetNeuronPtArrayVar": (_I, (c_void_p, _I, c_char_p, c_void_p, _I)),
    "IsNeuronIntVar": (_I, (_I, c_char_p)),
    "IsNeuronScalVar": (_I, (_I, c_char_p)),
    "IsNeuronPortVar": (_I, (_I, c_char_p)),
    "IsNeuronArrayVar": (_I, (_I, c_char_p)),
    "GetNeuronParamSize": (_I, (_I, c_char_p)),
    "GetNeuronVarSize": (_I, (_I, c_char_p)),
    "GetNeuronParam": (c_float_p, (_I, _I, c_char_p)),
    "GetNeuronPtParam": (c_float_p, (c_void_p, _I, c_char_p)),
    "GetArrayParam": (c_float_p, (_I, c_char_p)),
    "GetNeuronGroupParam": (_F, (_I, c_char_p)),
    "GetNeuronIntVar": (c_int_p, (_I, _I, c_char_p)),
    "GetNeuronVar": (c_float_p, (_I, _I, c_char_p)),
    "GetNeuronPtIntVar": (c_int_p, (c_void_p, _I, c_char_p)),
    "GetNeuronPtVar": (c_float_p, (c_void_p, _I, c_char_p)),
    "GetArrayVar": (c_float_p, (_I, c_char_p)),
    "GetNIntVar": (_I, (_I,)), "GetNScalVar": (_I, (_I,)), "GetNPortVar": (_I, (_I,)),
    "GetNScalParam": (_I, (_I,)), "GetNPortParam": (_I, (_I,)),
    "GetNArrayParam": (_I, (_I,)), "GetNGroupParam": (_I, (_I,)),
    "GetNArrayVar": (_I, (_I,)),
    "GetIntVarNames": (ctypes.POINTER(c_char_p), (_I,)),
    "GetScalVarNames": (ctypes.POINTER(c_char_p), (_I,)),
    "GetPortVarNames": (ctypes.POINTER(c_char_p), (_I,)),
    "GetScalParamNames": (ctypes.POINTER(c_char_p), (_I,)),
    "GetPortParamNames": (ctypes.POINTER(c_char_p), (_I,)),
    "GetArrayParamNames": (ctypes.POINTER(c_char_p), (_I,)),
    "GetGroupParamNames": (ctypes.POINTER(c_char_p), (_I,)),
    "GetArrayVarNames": (ctypes.POINTER(c_char_p), (_I,)),
    "Calibrate": (_I, ()),
    "Simulate": (_I, ()),
    "StartSimulation": (_I, ()),
    "SimulationStep": (_I, ()),
    "EndSimulation": (_I, ()),
    "ConnectMpiInit": (_I, (_I, c_void_p)),
    "MpiId": (_I, ()), "MpiNp": (_I, ()), "ProcMaster": (_I, ()),
    "MpiFinalize": (_I, ()),
    "RandomInt": (ctypes.POINTER(ctypes.c_uint), (ctypes.c_size_t,)),
    "RandomUniform": (c_float_p, (ctypes.c_size_t,)),
    "RandomNormal": (c_float_p, (ctypes.c_size_t, _F, _F)),
    "RandomNormalClipped": (c_float_p, (ctypes.c_size_t, _F, _F, _F, _F, _F)),
    "Connect": (_I, (_I, _I, _U, _U, _F, _F)),
    "ConnSpecInit": (_I, ()),
    "SetConnSpecParam": (_I, (c_char_p, _I)),
    "ConnSpecIsParam": (_I, (c_char_p,)),
    "SynSpecInit": (_I, ()),
    "SetSynSpecIntParam": (_I, (c_char_p, _I)),
    "SetSynSpecFloatParam": (_I, (c_char_p, _F)),
    "SetSynSpecFloatPtParam": (_I, (c_char_p, c_void_p)),
    "SynSpecIsIntParam": (_I, (c_char_p,)),
    "SynSpecIsFloatParam": (_I, (c_char_p,)),
    "SynSpecIsFloatPtParam": (_I, (c_char_p,)),
    "ConnectSeqSeq": (_I, (_I, _I, _I, _I)),
    "ConnectSeqGroup": (_I, (_I, _I, c_void_p, _I)),
    "ConnectGroupSeq": (_I, (c_void_p, _I, _I, _I)),
    "ConnectGroupGroup": (_I, (c_void_p, _I, c_void_p, _I)),
    "RemoteConnectSeqSeq": (_I, (_I, _I, _I, _I, _I, _I)),
    "RemoteConnectSeqGroup": (_I, (_I, _I, _I, _I, c_void_p, _I)),
    "RemoteConnectGroupSeq": (_I, (_I, c_void_p, _I, _I, _I, _I)),
    "RemoteConnectGroupGroup": (_I, (_I, c_void_p, _I, _I, c_void_p, _I)),
    "GetSeqSeqConnections": (c_int_p, (_I, _I, _I, _I, _I, c_int_p)),
    "GetSeqGroupConnections": (c_int_p, (_I, _I, c_void_p, _I, _I, c_int_p)),
    "GetGroupSeqConnections": (c_int_p, (c_void_p, _I, _I, _I, _I, c_int_p)),
    "GetGroupGroupConnections": (c_int_p, (c_void_p, _I, c_void_p, _I, _I, c_int_p)),
    "GetConnectionStatus": (_I, (_I, _I, _I, c_int_p, c_char_p, c_char_p, c_float_p,
                                 c_float_p)),
    "CreateSynGroup": (_I, (c_char_p,)),
    "GetSynGroupNParam": (_I, (_I,)),
    "GetSynGroupParamNames": (ctypes.POINTER(c_char_p), (_I,)),
    "IsSynGroupParam": (_I, (_I, c_char_p)),
    "GetSynGroupParam": (_F, (_I, c_char_p)),
    "SetSynGroupParam": (_I, (_I, c_char_p, _F)),
    "ActivateSpikeCount": (_I, (_I, _I)),
    "ActivateRecSpikeTimes": (_I, (_I, _I, _I)),
    "GetNRecSpikeTimes": (_I, (_I,)),
    "GetRecSpikeTimes": (c_float_p, (_I,)),
    "SetNeuronGroupParam": (_I, (_I, _I, c_char_p, _F)),
    "GetNFloatParam": (_I, ()),
    "GetFloatParamNames": (ctypes.POINTER(c_char_p), ()),
    "IsFloatParam": (_I, (c_char_p,)),
    "GetFloatParam": (_F, (c_char_p,)),
    "SetFloatParam": (_I, (c_char_p, _F)),
    "GetNIntParam": (_I, ()),
    "GetIntParamNames": (ctypes.POINTER(c_char_p), ()),
    "IsIntParam": (_I, (c_char_p,)),
    "GetIntParam": (_I, (c_char_p,)),
    "SetIntParam": (_I, (c_char_p, _I)),
    "RemoteCreate": (_I, (_I, c_char_p, _I, _I)),
}

_EXT_SIG = {
    "NGB200_Reset": (_I, ()),
    "NGB200_StageEvaluations": (ctypes.c_ulonglong, ()),
    "NGB200_DeliveredEvents": (ctypes.c_ulonglong, ()),
    "NGB200_TotalSpikes": (ctypes.c_ulonglong, ()),
    "NGB200_LastSimulateSeconds": (ctypes.c_double, ()),
    "NGB200_SetGraphChunk": (_I, (_I,)),
    "NGB200_NNodes": (ctypes.c_longlong, ()),
    "NGB200_NConnections": (ctypes.c_longlong, ()),
    "NGB200_GetAllConnections": (ctypes.c_longlong, (c_int_p, c_int_p, c_int_p, c_int_p,
                                                     c_float_p, c_float_p)),
    "NGB200_FreeArray": (None, (c_void_p,)),
    "NGB200_KernelsPerStep": (ctypes.c_double, ()),
    "NGB200_SetRk5Batching": (_I, (_I,)),
    "NGB200_Rk5BatchOf": (_I, (_I,)),
    "NGB200_SetStepLog": (_I, (_I, _I)),
    "NGB200_GetStepLogCount": (ctypes.c_longlong, (_I,)),
    "NGB200_GetStepLog": (_I, (_I, c_float_p, _I)),
    "NGB200_TrainStepProposer": (_I, (_I, _I, _F, ctypes.c_ulonglong, c_float_p, c_float_p)),
    "NGB200_SetStepProposer": (_I, (_I, _I)),
    "NGB200_SetStepProposerParams": (_I, (c_float_p,)),
    "NGB200_GetStepProposerParams": (_I, (c_float_p,)),
    "NGB200_SetStepProposerMargin": (_I, (_F,)),
    "NGB200_MlpGradients": (_F, (c_float_p, _I, c_float_p, c_float_p)),
    "NGB200_MlpInfer": (_I, (c_float_p, _I, c_float_p, c_float_p)),
    "NGB200_LastSimulateDeviceMs": (ctypes.c_double, ()),
    "NGB200_SetRk5MaxSubsteps": (_I, (_I,)),
    "NGB200_SetWaitTest": (_I, (_I,)),
    "NGB200_ProposerPhaseAfter": (ctypes.c_uint, (ctypes.c_uint, _I, _I)),
    "NGB200_SetKernelTiming": (_I, (_I,)),
    "NGB200_GetKernelTiming": (_I, (_I, ctypes.POINTER(ctypes.c_double),
                                    ctypes.POINTER(ctypes.c_longlong))),
    "NGB200_GetRk5Tuning": (_I, (_I, ctypes.POINTER(ctypes.c_int),
                                 ctypes.POINTER(ctypes.c_float))),
    "NGB200_StreamingDeliveryRate": (_I, (ctypes.c_longlong, ctypes.c_longlong, _I,
                                          ctypes.POINTER(ctypes.c_double))),
    "NGB200_SetInstance": (_I, (_I,)),
    "NGB200_GetInstance": (_I, ()),
    "NGB200_SetHost": (_I, (_I, _I)),
    "NGB200_SimulateSteps": (_I, (ctypes.c_longlong,)),
    "NGB200_RemoteExchangeSteps": (_I, ()),
    "NGB200_PackRemoteSpikes": (ctypes.c_longlong, (_I, c_void_p, ctypes.c_longlong)),
    "NGB200_UnpackRemoteSpikes": (_I, (_I, _I, c_void_p, ctypes.c_longlong)),
}


class Binding(object):
    """The reference's Python API over one shared library."""

    def __init__(self, lib_path=None):
        path = lib_path or os.environ.get("NEURONGPU_LIB") or DEFAULT_LIB
        if not os.path.exists(path):
            raise RuntimeError(
                "libneurongpu.so not found at %s; build it with "
                "`python -m neurongpu_b200.build`" % path)
        self.lib_path = path
        self._keep = []
        self._lib = ctypes.CDLL(path)
        self._c = {}
        for name, (res, args) in _SIG.items():
            f = getattr(self._lib, "NeuronGPU_" + name)
            f.restype = res
            f.argtypes = args
            self._c[name] = f
        self.has_extensions = hasattr(self._lib, "NGB200_Reset")
        if self.has_extensions:
            for name, (res, args) in _EXT_SIG.items():
                f = getattr(self._lib, name)
                f.restype = res
                f.argtypes = args
                self._c[name] = f
        # errors are returned as codes and raised here as ValueError
        self._c["SetOnException"](1)
        # collective of a network partitioned over hosts (ConnectMpiInit)
        self._comm = None
        self._xbuf = None

    # -- errors ----------------------------------------------------------
    def GetErrorMessage(self):
        "Get error message from NeuronGPU exception"
        p = self._c["GetErrorMessage"]()
        return ctypes.cast(p, ctypes.c_char_p).value.decode("utf-8", "replace")

    def GetErrorCode(self):
        "Get error code from NeuronGPU exception"
        return self._c["GetErrorCode"]()

    def SetOnException(self, on_exception):
        "Define whether handle exceptions (1) or exit (0) in case of errors"
        return self._c["SetOnException"](ctypes.c_int(on_exception))

    def _call(self, name, *args):
        ret = self._c[name](*args)
        if self._c["GetErrorCode"]() != 0:
            raise ValueError(self.GetErrorMessage())
        return ret

    def _release(self, pt, value):
        """Frees a host array the library handed out (after its contents
        were copied into value) and returns value."""
        # a library without the extensions (the reference's own build) hands
        # out arrays that its callers never free (src/base_neuron.cu:459)
        if pt and self.has_extensions:
            self._c["NGB200_FreeArray"](ctypes.cast(pt, c_void_p))
        return value

    def _names(self, fn, count, *args):
        n = count
        pp = self._call(fn, *args)
        out = []
        for i in range(n):
            out.append(to_def_str(ctypes.cast(pp[i], ctypes.c_char_p).value))
        return out

    # -- kernel parameters -----------------------------------------------
    def SetRandomSeed(self, seed):
        "Set seed for random number generation"
        return self._call("SetRandomSeed", ctypes.c_ulonglong(seed))

    def SetTimeResolution(self, time_res):
        "Set time resolution in ms"
        return self._call("SetTimeResolution", ctypes.c_float(time_res))

    def GetTimeResolution(self):
        "Get time resolution in ms"
        return self._call("GetTimeResolution")

    def SetMaxSpikeBufferSize(self, max_size):
        "Set maximum size of spike buffer per node"
        return self._call("SetMaxSpikeBufferSize", ctypes.c_int(max_size))

    def GetMaxSpikeBufferSize(self):
        "Get maximum size of spike buffer per node"
        return self._call("GetMaxSpikeBufferSize")

    def SetSimTime(self, sim_time):
        "Set neural activity simulated time in ms"
        return self._call("SetSimTime", ctypes.c_float(sim_time))

    def SetVerbosityLevel(self, verbosity_level):
        "Set verbosity level"
        return self._call("SetVerbosityLevel", ctypes.c_int(verbosity_level))

    def GetNFloatParam(self):
        return self._call("GetNFloatParam")

    def GetFloatParamNames(self):
        "Get list of kernel float parameter names"
        return self._names("GetFloatParamNames", self.GetNFloatParam())

    def IsFloatParam(self, param_name):
        return self._call("IsFloatParam", _cstr(param_name)) != 0

    def GetFloatParam(self, param_name):
        return self._call("GetFloatParam", _cstr(param_name))

    def SetFloatParam(self, param_name, val):
        return self._call("SetFloatParam", _cstr(param_name), ctypes.c_float(val))

    def GetNIntParam(self):
        return self._call("GetNIntParam")

    def GetIntParamNames(self):
        "Get list of kernel int parameter names"
        return self._names("GetIntParamNames", self.GetNIntParam())

    def IsIntParam(self, param_name):
        return self._call("IsIntParam", _cstr(param_name)) != 0

    def GetIntParam(self, param_name):
        return self._call("GetIntParam", _cstr(param_name))

    def SetIntParam(self, param_name, val):
        return self._call("SetIntParam", _cstr(param_name), ctypes.c_int(val))

    def GetKernelStatus(self, var_key=None):
        "Get kernel status"
        if isinstance(var_key, (list, tuple)):
            return [self.GetKernelStatus(v) for v in var_key]
        if var_key is None:
            d = {}
            for n in self.GetFloatParamNames() + self.GetIntParamNames():
                d[n] = self.GetKernelStatus(n)
            return d
        if isinstance(var_key, (str, bytes)):
            if self.IsFloatParam(var_key):
                return self.GetFloatParam(var_key)
            if self.IsIntParam(var_key):
                return self.GetIntParam(var_key)
            raise ValueError("Unknown parameter in GetKernelStatus", var_key)
        raise ValueError("Unknown key type in GetKernelStatus", type(var_key))

    def SetKernelStatus(self, params, val=None):
        "Set kernel parameters using dictionaries"
        if isinstance(params, dict) and val is None:
            for k in params:
                self.SetKernelStatus(k, params[k])
        elif isinstance(params, str):
            if self.IsFloatParam(params):
                return self.SetFloatParam(params, val)
            if self.IsIntParam(params):
                return self.SetIntParam(params, val)
            raise ValueError("Unknown parameter in SetKernelStatus", params)
        else:
            raise ValueError("Wrong argument in SetKernelStatus")

    # -- nodes -------------------------------------------------------------
    def Create(self, model_name, n_node=1, n_ports=1, status_dict=None):
        "Create a neuron group"
        if isinstance(status_dict, dict):
            ng = self.Create(model_name, n_node, n_ports)
            self.SetStatus(ng, status_dict)
            return ng
        if status_dict is not None:
            raise ValueError("Wrong argument in Create")
        i_node = self._call("Create", _cstr(model_name), ctypes.c_int(n_node),
                            ctypes.c_int(n_ports))
        return NodeSeq(i_node, n_node)

    def CreatePoissonGenerator(self, n_node, rate):
        "Create a poisson-distributed spike generator"
        i_node = self._call("CreatePoissonGenerator", ctypes.c_int(n_node),
                            ctypes.c_float(rate))
        return NodeSeq(i_node, n_node)

    def RemoteCreate(self, i_host, model_name, n_node=1, n_ports=1, status_dict=None):
        "Create a remote neuron group"
        if isinstance(status_dict, dict):
            rg = self.RemoteCreate(i_host, model_name, n_node, n_ports)
            self.SetStatus(rg, status_dict)
            return rg
        i_node = self._call("RemoteCreate", ctypes.c_int(i_host), _cstr(model_name),
                            ctypes.c_int(n_node), ctypes.c_int(n_ports))
        # the group's first node is known on its own host only: the other
        # hosts receive it (the reference broadcasts it over MPI)
        if self._comm is not None and self._comm.size > 1:
            i_node = self._comm.broadcast_int(i_node, i_host)
        return RemoteNodeSeq(i_host, NodeSeq(i_node, n_node))

    def _nodes_arr(self, nodes):
        arr = (ctypes.c_int * len(nodes))(*nodes)
        return arr, ctypes.cast(arr, ctypes.c_void_p)

    def SetNeuronScalParam(self, i_node, n_node, param_name, val):
        return self._call("SetNeuronScalParam", ctypes.c_int(i_node), ctypes.c_int(n_node),
                          _cstr(param_name), ctypes.c_float(val))

    def SetNeuronArrayParam(self, i_node, n_node, param_name, param_list):
        arr = (ctypes.c_float * len(param_list))(*param_list)
        return self._call("SetNeuronArrayParam", ctypes.c_int(i_node), ctypes.c_int(n_node),
                          _cstr(param_name), ctypes.cast(arr, c_void_p),
                          ctypes.c_int(len(param_list)))

    def SetNeuronPtScalParam(self, nodes, param_name, val):
        a, p = self._nodes_arr(nodes)
        return self._call("SetNeuronPtScalParam", p, ctypes.c_int(len(nodes)),
                          _cstr(param_name), ctypes.c_float(val))

    def SetNeuronPtArrayParam(self, nodes, param_name, param_list):
        a, p = self._nodes_arr(nodes)
        arr = (ctypes.c_float * len(param_list))(*param_list)
        return self._call("SetNeuronPtArrayParam", p, ctypes.c_int(len(nodes)),
                          _cstr(param_name), ctypes.cast(arr, c_void_p),
                          ctypes.c_int(len(param_list)))

    def IsNeuronScalParam(self, i_node, param_name):
        return self._call("IsNeuronScalParam", ctypes.c_int(i_node), _cstr(param_name)) != 0

    def IsNeuronPortParam(self, i_node, param_name):
        return self._call("IsNeuronPortParam", ctypes.c_int(i_node), _cstr(param_name)) != 0

    def IsNeuronArrayParam(self, i_node, param_name):
        return self._call("IsNeuronArrayParam", ctypes.c_int(i_node), _cstr(param_name)) != 0

    def IsNeuronGroupParam(self, i_node, param_name):
        return self._call("IsNeuronGroupParam", ctypes.c_int(i_node), _cstr(param_name)) != 0

    def SetNeuronIntVar(self, i_node, n_node, var_name, val):
        return self._call("SetNeuronIntVar", ctypes.c_int(i_node), ctypes.c_int(n_node),
                          _cstr(var_name), ctypes.c_int(val))

    def SetNeuronScalVar(self, i_node, n_node, var_name, val):
        return self._call("SetNeuronScalVar", ctypes.c_int(i_node), ctypes.c_int(n_node),
                          _cstr(var_name), ctypes.c_float(val))

    def SetNeuronArrayVar(self, i_node, n_node, var_name, var_list):
        arr = (ctypes.c_float * len(var_list))(*var_list)
        return self._call("SetNeuronArrayVar", ctypes.c_int(i_node), ctypes.c_int(n_node),
                          _cstr(var_name), ctypes.cast(arr, c_void_p),
                          ctypes.c_int(len(var_list)))

    def SetNeuronPtIntVar(self, nodes, var_name, val):
        a, p = self._nodes_arr(nodes)
        return self._call("SetNeuronPtIntVar", p, ctypes.c_int(len(nodes)),
                          _cstr(var_name), ctypes.c_int(val))

    def SetNeuronPtScalVar(self, nodes, var_name, val):
        a, p = self._nodes_arr(nodes)
        return self._call("SetNeuronPtScalVar", p, ctypes.c_int(len(nodes)),
                          _cstr(var_name), ctypes.c_float(val))

    def SetNeuronPtArrayVar(self, nodes, var_name, var_list):
        a, p = self._nodes_arr(nodes)
        arr = (ctypes.c_float * len(var_list))(*var_list)
        return self._call("SetNeuronPtArrayVar", p, ctypes.c_int(len(nodes)),
                          _cstr(var_name), ctypes.cast(arr, c_void_p),
                          ctypes.c_int(len(var_list)))

    def IsNeuronIntVar(self, i_node, var_name):
        return self._call("IsNeuronIntVar", ctypes.c_int(i_node), _cstr(var_name)) != 0

    def IsNeuronScalVar(self, i_node, var_name):
        return self._call("IsNeuronScalVar", ctypes.c_int(i_node), _cstr(var_name)) != 0

    def IsNeuronPortVar(self, i_node, var_name):
        return self._call("IsNeuronPortVar", ctypes.c_int(i_node), _cstr(var_name)) != 0

    def IsNeuronArrayVar(self, i_node, var_name):
        return self._call("IsNeuronArrayVar", ctypes.c_int(i_node), _cstr(var_name)) != 0

    def GetNeuronParamSize(self, i_node, param_name):
        return self._call("GetNeuronParamSize", ctypes.c_int(i_node), _cstr(param_name))

    def GetNeuronVarSize(self, i_node, var_name):
        return self._call("GetNeuronVarSize", ctypes.c_int(i_node), _cstr(var_name))

    @staticmethod
    def _rows(data_pt, n_node, array_size):
        import numpy as np
        if n_node <= 0:
            return []
        a = np.ctypeslib.as_array(data_pt, shape=(n_node * max(array_size, 1),))
        if array_size > 1:
            return a.reshape(n_node, array_size).tolist()
        return a.tolist()

    def GetNeuronParam(self, i_node, n_node, param_name):
        "Get neuron parameter value"
        sz = self.GetNeuronParamSize(i_node, param_name)
        pt = self._call("GetNeuronParam", ctypes.c_int(i_node), ctypes.c_int(n_node),
                        _cstr(param_name))
        return self._release(pt, self._rows(pt, n_node, sz))

    def GetNeuronPtParam(self, nodes, param_name):
        a, p = self._nodes_arr(nodes)
        sz = self.GetNeuronParamSize(nodes[0], param_name)
        pt = self._call("GetNeuronPtParam", p, ctypes.c_int(len(nodes)), _cstr(param_name))
        return self._release(pt, self._rows(pt, len(nodes), sz))

    def GetArrayParam(self, i_node, n_node, param_name):
        "Get neuron array parameter"
        out = []
        for j in range(n_node):
            sz = self.GetNeuronParamSize(i_node + j, param_name)
            pt = self._call("GetArrayParam", ctypes.c_int(i_node + j), _cstr(param_name))
            out.append(self._release(pt, [pt[k] for k in range(sz)]))
        return out

    def GetNeuronListArrayParam(self, node_list, param_name):
        out = []
        for i in node_list:
            sz = self.GetNeuronParamSize(i, param_name)
            pt = self._call("GetArrayParam", ctypes.c_int(i), _cstr(param_name))
            out.append(self._release(pt, [pt[k] for k in range(sz)]))
        return out

    def GetNeuronGroupParam(self, i_node, param_name):
        return self._call("GetNeuronGroupParam", ctypes.c_int(i_node), _cstr(param_name))

    def GetNeuronIntVar(self, i_node, n_node, var_name):
        return self.GetNeuronIntVarArray(i_node, n_node, var_name).reshape(-1, 1).tolist()

    def GetNeuronIntVarArray(self, i_node, n_node, var_name):
        """GetNeuronIntVar as a numpy int32 array of n_node values (extension:
        one copy instead of a Python list of lists)."""
        import numpy as np
        pt = self._call("GetNeuronIntVar", ctypes.c_int(i_node), ctypes.c_int(n_node),
                        _cstr(var_name))
        if n_node <= 0:
            return self._release(pt, np.zeros(0, dtype=np.int32))
        return self._release(pt, np.ctypeslib.as_array(pt, shape=(n_node,)).copy())

    def GetNeuronVar(self, i_node, n_node, var_name):
        sz = self.GetNeuronVarSize(i_node, var_name)
        pt = self._call("GetNeuronVar", ctypes.c_int(i_node), ctypes.c_int(n_node),
                        _cstr(var_name))
        return self._release(pt, self._rows(pt, n_node, sz))

    def GetNeuronPtIntVar(self, nodes, var_name):
        a, p = self._nodes_arr(nodes)
        pt = self._call("GetNeuronPtIntVar", p, ctypes.c_int(len(nodes)), _cstr(var_name))
        return self._release(pt, [[pt[i]] for i in range(len(nodes))])

    def GetNeuronPtVar(self, nodes, var_name):
        a, p = self._nodes_arr(nodes)
        sz = self.GetNeuronVarSize(nodes[0], var_name)
        pt = self._call("GetNeuronPtVar", p, ctypes.c_int(len(nodes)), _cstr(var_name))
        return self._release(pt, self._rows(pt, len(nodes), sz))

    def GetArrayVar(self, i_node, n_node, var_name):
        out = []
        for j in range(n_node):
            sz = self.GetNeuronVarSize(i_node + j, var_name)
            pt = self._call("GetArrayVar", ctypes.c_int(i_node + j), _cstr(var_name))
            out.append(self._release(pt, [pt[k] for k in range(sz)]))
        return out

    def GetNeuronListArrayVar(self, node_list, var_name):
        out = []
        for i in node_list:
            sz = self.GetNeuronVarSize(i, var_name)
            pt = self._call("GetArrayVar", ctypes.c_int(i), _cstr(var_name))
            out.append(self._release(pt, [pt[k] for k in range(sz)]))
        return out

    def GetNeuronStatus(self, nodes, var_name):
        "Get neuron group scalar or array variable or parameter"
        if not _is_seq(nodes):
            raise ValueError("Unknown node type")
        if isinstance(nodes, NodeSeq):
            i0, n = nodes.i0, nodes.n
            if self.IsNeuronScalParam(i0, var_name) or self.IsNeuronPortParam(i0, var_name):
                return self.GetNeuronParam(i0, n, var_name)
            if self.IsNeuronArrayParam(i0, var_name):
                return self.GetArrayParam(i0, n, var_name)
            if self.IsNeuronIntVar(i0, var_name):
                return self.GetNeuronIntVar(i0, n, var_name)
            if self.IsNeuronScalVar(i0, var_name) or self.IsNeuronPortVar(i0, var_name):
                return self.GetNeuronVar(i0, n, var_name)
            if self.IsNeuronArrayVar(i0, var_name):
                return self.GetArrayVar(i0, n, var_name)
            if self.IsNeuronGroupParam(i0, var_name):
                return self.GetNeuronStatus(nodes.ToList(), var_name)
            raise ValueError("Unknown neuron variable or parameter")
        n0 = nodes[0]
        if self.IsNeuronScalParam(n0, var_name) or self.IsNeuronPortParam(n0, var_name):
            return self.GetNeuronPtParam(nodes, var_name)
        if self.IsNeuronArrayParam(n0, var_name):
            return self.GetNeuronListArrayParam(nodes, var_name)
        if self.IsNeuronIntVar(n0, var_name):
            return self.GetNeuronPtIntVar(nodes, var_name)
        if self.IsNeuronScalVar(n0, var_name) or self.IsNeuronPortVar(n0, var_name):
            return self.GetNeuronPtVar(nodes, var_name)
        if self.IsNeuronArrayVar(n0, var_name):
            return self.GetNeuronListArrayVar(nodes, var_name)
        if self.IsNeuronGroupParam(n0, var_name):
            return [self.GetNeuronGroupParam(i, var_name) for i in nodes]
        raise ValueError("Unknown neuron variable or parameter")

    def GetNIntVar(self, i_node):
        return self._call("GetNIntVar", ctypes.c_int(i_node))

    def GetNScalVar(self, i_node):
        return self._call("GetNScalVar", ctypes.c_int(i_node))

    def GetNPortVar(self, i_node):
        return self._call("GetNPortVar", ctypes.c_int(i_node))

    def GetNScalParam(self, i_node):
        return self._call("GetNScalParam", ctypes.c_int(i_node))

    def GetNPortParam(self, i_node):
        return self._call("GetNPortParam", ctypes.c_int(i_node))

    def GetNArrayParam(self, i_node):
        return self._call("GetNArrayParam", ctypes.c_int(i_node))

    def GetNGroupParam(self, i_node):
        return self._call("GetNGroupParam", ctypes.c_int(i_node))

    def GetNArrayVar(self, i_node):
        return self._call("GetNArrayVar", ctypes.c_int(i_node))

    def GetIntVarNames(self, i_node):
        return self._names("GetIntVarNames", self.GetNIntVar(i_node), ctypes.c_int(i_node))

    def GetScalVarNames(self, i_node):
        return self._names("GetScalVarNames", self.GetNScalVar(i_node), ctypes.c_int(i_node))

    def GetPortVarNames(self, i_node):
        return self._names("GetPortVarNames", self.GetNPortVar(i_node), ctypes.c_int(i_node))

    def GetScalParamNames(self, i_node):
        return self._names("GetScalParamNames", self.GetNScalParam(i_node), ctypes.c_int(i_node))

    def GetPortParamNames(self, i_node):
        return self._names("GetPortParamNames", self.GetNPortParam(i_node), ctypes.c_int(i_node))

    def GetArrayParamNames(self, i_node):
        return self._names("GetArrayParamNames", self.GetNArrayParam(i_node),
                           ctypes.c_int(i_node))

    def GetGroupParamNames(self, i_node):
        return self._names("GetGroupParamNames", self.GetNGroupParam(i_node),
                           ctypes.c_int(i_node))

    def GetArrayVarNames(self, i_node):
        return self._names("GetArrayVarNames", self.GetNArrayVar(i_node), ctypes.c_int(i_node))

    def SetNeuronGroupParam(self, nodes, param_name, val):
        if not isinstance(nodes, NodeSeq):
            raise ValueError("Wrong argument type in SetNeuronGroupParam")
        return self._call("SetNeuronGroupParam", ctypes.c_int(nodes.i0), ctypes.c_int(nodes.n),
                          _cstr(param_name), ctypes.c_float(val))

    def SetNeuronStatus(self, nodes, var_name, val):
        "Set neuron group scalar or array variable or parameter"
        if not _is_seq(nodes):
            raise ValueError("Unknown node type")
        if isinstance(val, dict):
            arr = self.DictToArray(val, len(nodes))
            for i in range(len(nodes)):
                self.SetNeuronStatus([nodes[i]], var_name, arr[i])
            return
        if isinstance(nodes, NodeSeq):
            i0, n = nodes.i0, nodes.n
            if self.IsNeuronGroupParam(i0, var_name):
                self.SetNeuronGroupParam(nodes, var_name, val)
            elif self.IsNeuronScalParam(i0, var_name):
                self.SetNeuronScalParam(i0, n, var_name, val)
            elif self.IsNeuronPortParam(i0, var_name) or self.IsNeuronArrayParam(i0, var_name):
                self.SetNeuronArrayParam(i0, n, var_name, val)
            elif self.IsNeuronIntVar(i0, var_name):
                self.SetNeuronIntVar(i0, n, var_name, val)
            elif self.IsNeuronScalVar(i0, var_name):
                self.SetNeuronScalVar(i0, n, var_name, val)
            elif self.IsNeuronPortVar(i0, var_name) or self.IsNeuronArrayVar(i0, var_name):
                self.SetNeuronArrayVar(i0, n, var_name, val)
            else:
                raise ValueError("Unknown neuron variable or parameter")
        else:
            n0 = nodes[0]
            if self.IsNeuronScalParam(n0, var_name):
                self.SetNeuronPtScalParam(nodes, var_name, val)
            elif self.IsNeuronPortParam(n0, var_name) or self.IsNeuronArrayParam(n0, var_name):
                self.SetNeuronPtArrayParam(nodes, var_name, val)
            elif self.IsNeuronIntVar(n0, var_name):
                self.SetNeuronPtIntVar(nodes, var_name, val)
            elif self.IsNeuronScalVar(n0, var_name):
                self.SetNeuronPtScalVar(nodes, var_name, val)
            elif self.IsNeuronPortVar(n0, var_name) or self.IsNeuronArrayVar(n0, var_name):
                self.SetNeuronPtArrayVar(nodes, var_name, val)
            else:
                raise ValueError("Unknown neuron variable or parameter")

    # -- recording ---------------------------------------------------------
    def CreateRecord(self, file_name, var_name_list, i_node_list, i_port_list):
        "Create a record of neuron variables"
        n = len(i_node_list)
        names = [_cstr(v) for v in var_name_list]
        name_arr = (c_char_p * n)(*[ctypes.cast(b, c_char_p) for b in names])
        return self._call("CreateRecord", _cstr(file_name), name_arr,
                          (ctypes.c_int * n)(*i_node_list), (ctypes.c_int * n)(*i_port_list),
                          ctypes.c_int(n))

    def GetRecordDataRows(self, i_record):
        return self._call("GetRecordDataRows", ctypes.c_int(i_record))

    def GetRecordDataColumns(self, i_record):
        return self._call("GetRecordDataColumns", ctypes.c_int(i_record))

    def GetRecordData(self, i_record):
        "Get record data"
        nr = self.GetRecordDataRows(i_record)
        nc = self.GetRecordDataColumns(i_record)
        pt = self._call("GetRecordData", ctypes.c_int(i_record))
        return self._release(pt, [[pt[r][c] for c in range(nc)] for r in range(nr)])

    def ActivateSpikeCount(self, nodes):
        "Activate spike count for node group"
        if not isinstance(nodes, NodeSeq):
            raise ValueError("Argument type of ActivateSpikeCount must be NodeSeq")
        return self._call("ActivateSpikeCount", ctypes.c_int(nodes.i0), ctypes.c_int(nodes.n))

    def ActivateRecSpikeTimes(self, nodes, max_n_rec_spike_times):
        "Activate spike time recording for node group"
        if not isinstance(nodes, NodeSeq):
            raise ValueError("Argument type of ActivateRecSpikeTimes must be NodeSeq")
        return self._call("ActivateRecSpikeTimes", ctypes.c_int(nodes.i0),
                          ctypes.c_int(nodes.n), ctypes.c_int(max_n_rec_spike_times))

    def GetNRecSpikeTimes(self, i_node):
        return self._call("GetNRecSpikeTimes", ctypes.c_int(i_node))

    def GetRecSpikeTimes(self, i_node):
        "Get recorded spike times for node"
        n = self.GetNRecSpikeTimes(i_node)
        pt = self._call("GetRecSpikeTimes", ctypes.c_int(i_node))
        return self._release(pt, [pt[k] for k in range(n)])

    # -- simulation ----------------------------------------------------------
    def Calibrate(self):
        "Calibrate simulation"
        return self._call("Calibrate")

    def Simulate(self, sim_time=1000.0):
        "Simulate neural activity"
        self.SetSimTime(sim_time)
        if self._comm is not None and self._comm.size > 1:
            return self._simulate_partitioned(sim_time)
        return self._call("Simulate")

    def _simulate_partitioned(self, sim_time):
        """Simulate on every host of a partitioned network: runs of E steps
        (the shortest delay of a remote connection, the same on every host),
        each followed by the spike exchange, so a remote spike reaches its
        image before any delivery of it is due (the reference exchanges
        every step, src/neurongpu.cu:490-521)."""
        self._call("StartSimulation")
        n_total = int(round(sim_time / self.GetTimeResolution()))
        e = self._call("NGB200_RemoteExchangeSteps")
        e = self._comm.min_int(e if e > 0 else 1 << 30)
        e = max(1, min(e, 1000))
        done = 0
        while done < n_total:
            k = min(e, n_total - done)
            self._call("NGB200_SimulateSteps", ctypes.c_longlong(k))
            self._exchange_spikes(k)
            done += k
        return self._call("EndSimulation")

    def _exchange_spikes(self, n_steps):
        """Packs this host's exported spikes of the last n_steps steps,
        all-gathers the lists over the hosts and pushes the other hosts'
        spikes into the images here."""
        comm = self._comm
        if self._xbuf is None:
            self._xbuf = comm.empty_u32(4 + 3 * 4096)
        cap = (self._xbuf.numel() - 4) // 3
        count = self.PackRemoteSpikes(n_steps, self._xbuf.data_ptr(), cap)
        if count > cap:
            self._xbuf = comm.empty_u32(4 + 3 * (2 * count))
            cap = (self._xbuf.numel() - 4) // 3
            count = self.PackRemoteSpikes(n_steps, self._xbuf.data_ptr(), cap)
        counts = comm.allgather_int(count)
        m = max(counts)
        if m == 0:
            return
        if self._xbuf.numel() < 4 + 3 * m:
            # every host sends the longest list's length: keep this host's
            # packed spikes in a buffer that long
            grown = comm.empty_u32(4 + 3 * (2 * m))
            grown[:self._xbuf.numel()] = self._xbuf
            self._xbuf = grown
        rows = comm.allgather_rows(self._xbuf, 4 + 3 * m)
        for h, c in enumerate(counts):
            if h != comm.rank and c > 0:
                self.UnpackRemoteSpikes(h, n_steps, comm.row_ptr(rows, h), c)
        # the unpacks read the gathered rows on the simulation stream: wait
        # for them before the rows' memory can be reused
        comm.sync()

    def StartSimulation(self):
        return self._call("StartSimulation")

    def SimulationStep(self):
        return self._call("SimulationStep")

    def EndSimulation(self):
        return self._call("EndSimulation")

    def ConnectMpiInit(self, comm=None):
        """Initialize the hosts of a network partitioned over GPUs, one
        process per GPU (the reference's MPI initialisation): the host index
        and count come from the job launcher (torchrun, mpirun); the spike
        exchange uses torch.distributed (NCCL over NVLink), or comm, an
        object with the methods of HostComm"""
        argv = (ctypes.c_char_p * 1)(b"python")
        ret = self._call("ConnectMpiInit", ctypes.c_int(1), ctypes.cast(argv, c_void_p))
        if comm is None and self.MpiNp() > 1:
            comm = HostComm()
        if comm is not None:
            self._call("NGB200_SetHost", ctypes.c_int(comm.rank), ctypes.c_int(comm.size))
        self._comm = comm
        return ret

    def MpiId(self):
        return self._call("MpiId")

    def Rank(self):
        return self.MpiId()

    def MpiNp(self):
        return self._call("MpiNp")

    def ProcMaster(self):
        return self._call("ProcMaster")

    def MpiFinalize(self):
        return self._call("MpiFinalize")

    # -- random arrays -----------------------------------------------------
    def RandomInt(self, n):
        "Generate n random integers"
        return self._call("RandomInt", ctypes.c_size_t(n))

    def RandomUniform(self, n):
        "Generate n random floats uniform in (0,1)"
        return self._call("RandomUniform", ctypes.c_size_t(n))

    def RandomNormal(self, n, mean, stddev):
        return self._call("RandomNormal", ctypes.c_size_t(n), ctypes.c_float(mean),
                          ctypes.c_float(stddev))

    def RandomNormalClipped(self, n, mean, stddev, vmin, vmax, vstep=0):
        return self._call("RandomNormalClipped", ctypes.c_size_t(n), ctypes.c_float(mean),
                          ctypes.c_float(stddev), ctypes.c_float(vmin), ctypes.c_float(vmax),
                          ctypes.c_float(vstep))

    # -- connections ---------------------------------------------------------
    def SingleConnect(self, i_source_node, i_target_node, i_port, weight, delay):
        "Connect two nodes"
        return self._call("Connect", ctypes.c_int(i_source_node), ctypes.c_int(i_target_node),
                          ctypes.c_ubyte(i_port), ctypes.c_ubyte(0), ctypes.c_float(weight),
                          ctypes.c_float(delay))

    def ConnSpecInit(self):
        return self._call("ConnSpecInit")

    def SetConnSpecParam(self, param_name, val):
        return self._call("SetConnSpecParam", _cstr(param_name), ctypes.c_int(val))

    def ConnSpecIsParam(self, param_name):
        return self._call("ConnSpecIsParam", _cstr(param_name)) != 0

    def SynSpecInit(self):
        return self._call("SynSpecInit")

    def SetSynSpecIntParam(self, param_name, val):
        return self._call("SetSynSpecIntParam", _cstr(param_name), ctypes.c_int(val))

    def SetSynSpecFloatParam(self, param_name, val):
        return self._call("SetSynSpecFloatParam", _cstr(param_name), ctypes.c_float(val))

    def SetSynSpecFloatPtParam(self, param_name, arr):
        if isinstance(arr, (list, tuple)):
            arr = (ctypes.c_float * len(arr))(*arr)
        self._keep.append(arr)
        return self._call("SetSynSpecFloatPtParam", _cstr(param_name),
                          ctypes.cast(arr, c_void_p))

    def SynSpecIsIntParam(self, param_name):
        return self._call("SynSpecIsIntParam", _cstr(param_name)) != 0

    def SynSpecIsFloatParam(self, param_name):
        return self._call("SynSpecIsFloatParam", _cstr(param_name)) != 0

    def SynSpecIsFloatPtParam(self, param_name):
        return self._call("SynSpecIsFloatPtParam", _cstr(param_name)) != 0

    def DictToArray(self, param_dict, array_size):
        "Array of values from an explicit array or a distribution dictionary"
        dist_name = None
        arr = None
        low, high = -1.0e35, 1.0e35
        mu = sigma = None
        vstep = 0
        for k, v in param_dict.items():
            if k == "array":
                dist_name, arr = "array", v
            elif k == "distribution":
                dist_name = v
            elif k == "low":
                low = v
            elif k == "high":
                high = v
            elif k == "mu":
                mu = v
            elif k == "sigma":
                sigma = v
            elif k == "step":
                vstep = v
            else:
                raise ValueError("Unknown parameter name in dictionary")
        if dist_name == "array":
            if isinstance(arr, (list, tuple)):
                if len(arr) != array_size:
                    raise ValueError("Wrong array size.")
                arr = (ctypes.c_float * len(arr))(*arr)
            return arr
        if dist_name == "normal":
            return self.RandomNormal(array_size, mu, sigma)
        if dist_name == "normal_clipped":
            return self.RandomNormalClipped(array_size, mu, sigma, low, high, vstep)
        if dist_name == "uniform":
            # extension: uniform in [low, high) from the library generator
            import numpy as np
            if low <= -1.0e35 or high >= 1.0e35:
                raise ValueError("uniform distribution needs low and high")
            pt = self.RandomUniform(array_size)
            a = np.ctypeslib.as_array(pt, shape=(array_size,))
            a *= np.float32(high - low)
            a += np.float32(low)
            return pt
        raise ValueError("Unknown distribution")

    @staticmethod
    def RuleArraySize(conn_dict, source, target):
        rule = conn_dict["rule"]
        if rule == "one_to_one":
            return len(source)
        if rule == "all_to_all":
            return len(source) * len(target)
        if rule == "fixed_total_number":
            return conn_dict["total_num"]
        if rule == "fixed_indegree":
            return len(target) * conn_dict["indegree"]
        if rule == "fixed_outdegree":
            return len(source) * conn_dict["outdegree"]
        raise ValueError("Unknown number of connections for this rule")

    def SetSynParamFromArray(self, param_name, par_dict, array_size):
        arr_name = param_name + "_array"
        if not self.SynSpecIsFloatPtParam(arr_name):
            raise ValueError("Synapse parameter cannot be set by arrays or distributions")
        arr = self.DictToArray(par_dict, array_size)
        self.SetSynSpecFloatPtParam(arr_name, arr)

    def Connect(self, source, target, conn_dict, syn_dict):
        "Connect two node groups"
        return self._connect("Connect", lambda sa, sn, ta, tn: (sa, sn, ta, tn),
                             source, target, conn_dict, syn_dict)

    def _connect(self, prefix, args, source, target, conn_dict, syn_dict):
        """Sets the connection and synapse specifications, then calls
        <prefix>SeqSeq / SeqGroup / GroupSeq / GroupGroup with the arguments
        args(source, n_source, target, n_target) forms."""
        if isinstance(source, RemoteNodeSeq):
            source = source.node_seq
        if isinstance(target, RemoteNodeSeq):
            target = target.node_seq
        if not _is_seq(source):
            raise ValueError("Unknown source type")
        if not _is_seq(target):
            raise ValueError("Unknown target type")
        gc.disable()
        self._keep = []
        try:
            self.ConnSpecInit()
            self.SynSpecInit()
            for k in conn_dict:
                if k == "rule":
                    if conn_dict[k] not in conn_rule_name:
                        raise ValueError("Unknown connection rule")
                    self.SetConnSpecParam(k, conn_rule_name.index(conn_dict[k]))
                elif self.ConnSpecIsParam(k):
                    self.SetConnSpecParam(k, conn_dict[k])
                else:
                    raise ValueError("Unknown connection parameter")
            array_size = self.RuleArraySize(conn_dict, source, target)
            for k in syn_dict:
                v = syn_dict[k]
                if self.SynSpecIsIntParam(k):
                    if k == "synapse_group" and isinstance(v, SynGroup):
                        v = v.i_syn_group
                    self.SetSynSpecIntParam(k, v)
                elif self.SynSpecIsFloatParam(k):
                    if isinstance(v, dict):
                        self.SetSynParamFromArray(k, v, array_size)
                    else:
                        self.SetSynSpecFloatParam(k, v)
                elif self.SynSpecIsFloatPtParam(k):
                    self.SetSynSpecFloatPtParam(k, v)
                else:
                    raise ValueError("Unknown synapse parameter")
            if isinstance(source, NodeSeq) and isinstance(target, NodeSeq):
                return self._call(prefix + "SeqSeq", *args(source.i0, source.n, target.i0, target.n))
            if not isinstance(source, NodeSeq):
                sa, sp = self._nodes_arr(source)
            if not isinstance(target, NodeSeq):
                ta, tp = self._nodes_arr(target)
            if isinstance(source, NodeSeq):
                return self._call(prefix + "SeqGroup", *args(source.i0, source.n, tp, len(target)))
            if isinstance(target, NodeSeq):
                return self._call(prefix + "GroupSeq", *args(sp, len(source), target.i0, target.n))
            return self._call(prefix + "GroupGroup", *args(sp, len(source), tp, len(target)))
        finally:
            self._keep = []
            gc.enable()

    def RemoteConnect(self, i_source_host, source, i_target_host, target, conn_dict,
                      syn_dict):
        """Connect two node groups of different hosts (every host runs the
        same call): the target host connects image nodes of the remote
        sources to its targets with the rule, the source host marks the
        sources as exported"""
        return self._connect("RemoteConnect",
                             lambda sa, sn, ta, tn: (i_source_host, sa, sn, i_target_host, ta, tn),
                             source, target, conn_dict, syn_dict)

    def GetConnections(self, source=None, target=None, syn_group=-1):
        "Get connections between two node groups"
        if source is None:
            source = NodeSeq(None)
        if target is None:
            target = NodeSeq(None)
        if isinstance(source, int):
            source = [source]
        if isinstance(target, int):
            target = [target]
        if not _is_seq(source):
            raise ValueError("Unknown source type")
        if not _is_seq(target):
            raise ValueError("Unknown target type")
        n_conn = ctypes.c_int(0)
        if isinstance(source, NodeSeq) and isinstance(target, NodeSeq):
            arr = self._call("GetSeqSeqConnections", source.i0, source.n, target.i0, target.n,
                             syn_group, ctypes.byref(n_conn))
        else:
            if not isinstance(source, NodeSeq):
                sa, sp = self._nodes_arr(source)
            if not isinstance(target, NodeSeq):
                ta, tp = self._nodes_arr(target)
            if isinstance(source, NodeSeq):
                arr = self._call("GetSeqGroupConnections", source.i0, source.n, tp, len(target),
                                 syn_group, ctypes.byref(n_conn))
            elif isinstance(target, NodeSeq):
                arr = self._call("GetGroupSeqConnections", sp, len(source), target.i0, target.n,
                                 syn_group, ctypes.byref(n_conn))
            else:
                arr = self._call("GetGroupGroupConnections", sp, len(source), tp, len(target),
                                 syn_group, ctypes.byref(n_conn))
        return self._release(arr, [ConnectionId(arr[3 * i], arr[3 * i + 1], arr[3 * i + 2])
                                   for i in range(n_conn.value)])

    def GetConnectionStatus(self, conn_id):
        i_target = ctypes.c_int(0)
        i_port = ctypes.c_char()
        i_syn = ctypes.c_char()
        delay = ctypes.c_float(0.0)
        weight = ctypes.c_float(0.0)
        self._call("GetConnectionStatus", conn_id.i_source, conn_id.i_group, conn_id.i_conn,
                   ctypes.byref(i_target), ctypes.byref(i_port), ctypes.byref(i_syn),
                   ctypes.byref(delay), ctypes.byref(weight))
        return {"source": conn_id.i_source, "target": i_target.value,
                "port": ord(i_port.value), "syn": ord(i_syn.value),
                "delay": delay.value, "weight": weight.value}

    # -- synapse groups ------------------------------------------------------
    def CreateSynGroup(self, model_name, status_dict=None):
        "Create a synapse group"
        if isinstance(status_dict, dict):
            sg = self.CreateSynGroup(model_name)
            self.SetStatus(sg, status_dict)
            return sg
        if status_dict is not None:
            raise ValueError("Wrong argument in CreateSynGroup")
        return SynGroup(self._call("CreateSynGroup", _cstr(model_name)))

    @staticmethod
    def _sg(syn_group, fn):
        if not isinstance(syn_group, SynGroup):
            raise ValueError("Wrong argument type in " + fn)
        return syn_group.i_syn_group

    def GetSynGroupNParam(self, syn_group):
        return self._call("GetSynGroupNParam", self._sg(syn_group, "GetSynGroupNParam"))

    def GetSynGroupParamNames(self, syn_group):
        i = self._sg(syn_group, "GetSynGroupParamNames")
        return self._names("GetSynGroupParamNames", self.GetSynGroupNParam(syn_group),
                           ctypes.c_int(i))

    def IsSynGroupParam(self, syn_group, param_name):
        i = self._sg(syn_group, "IsSynGroupParam")
        return self._call("IsSynGroupParam", i, _cstr(param_name)) != 0

    def GetSynGroupParam(self, syn_group, param_name):
        i = self._sg(syn_group, "GetSynGroupParam")
        return self._call("GetSynGroupParam", i, _cstr(param_name))

    def SetSynGroupParam(self, syn_group, param_name, val):
        i = self._sg(syn_group, "SetSynGroupParam")
        return self._call("SetSynGroupParam", i, _cstr(param_name), ctypes.c_float(val))

    def GetSynGroupStatus(self, syn_group, var_key=None):
        "Get synapse group status"
        self._sg(syn_group, "GetSynGroupStatus")
        if isinstance(var_key, (list, tuple)):
            return [self.GetSynGroupStatus(syn_group, v) for v in var_key]
        if var_key is None:
            return {n: self.GetSynGroupParam(syn_group, n)
                    for n in self.GetSynGroupParamNames(syn_group)}
        if isinstance(var_key, (str, bytes)):
            return self.GetSynGroupParam(syn_group, var_key)
        raise ValueError("Unknown key type in GetSynGroupStatus", type(var_key))

    def SetSynGroupStatus(self, syn_group, params, val=None):
        "Set synapse group parameters using dictionaries"
        self._sg(syn_group, "SetSynGroupStatus")
        if isinstance(params, dict) and val is None:
            for k in params:
                self.SetSynGroupStatus(syn_group, k, params[k])
        elif isinstance(params, str):
            return self.SetSynGroupParam(syn_group, params, val)
        else:
            raise ValueError("Wrong argument in SetSynGroupStatus")

    # -- generic status ------------------------------------------------------
    def SetStatus(self, gen_object, params, val=None):
        "Set neuron or synapse group parameters or variables using dictionaries"
        if isinstance(gen_object, RemoteNodeSeq):
            if gen_object.i_host == self.MpiId():
                self.SetStatus(gen_object.node_seq, params, val)
            return
        gc.disable()
        try:
            if isinstance(gen_object, SynGroup):
                return self.SetSynGroupStatus(gen_object, params, val)
            nodes = gen_object
            if val is not None:
                self.SetNeuronStatus(nodes, params, val)
            elif isinstance(params, dict):
                for k in params:
                    self.SetNeuronStatus(nodes, k, params[k])
            elif isinstance(params, (list, tuple)):
                if len(params) != len(nodes):
                    raise ValueError("List should have the same size as nodes")
                for d in params:
                    if not isinstance(d, dict):
                        raise ValueError("Type of list elements should be dict")
                    for k in d:
                        self.SetNeuronStatus(nodes, k, d[k])
            else:
                raise ValueError("Wrong argument in SetStatus")
        finally:
            gc.enable()

    def GetStatus(self, gen_object, var_key=None):
        "Get neuron group, connection or synapse group status"
        if isinstance(gen_object, SynGroup):
            return self.GetSynGroupStatus(gen_object, var_key)
        if isinstance(gen_object, NodeSeq):
            gen_object = gen_object.ToList()
        if isinstance(gen_object, (list, tuple)):
            return [self.GetStatus(g, var_key) for g in gen_object]
        if isinstance(var_key, (list, tuple)):
            return [self.GetStatus(gen_object, v) for v in var_key]
        if var_key is None:
            if isinstance(gen_object, ConnectionId):
                return self.GetConnectionStatus(gen_object)
            if isinstance(gen_object, int):
                i = gen_object
                names = (self.GetIntVarNames(i) + self.GetScalVarNames(i)
                         + self.GetScalParamNames(i) + self.GetPortVarNames(i)
                         + self.GetPortParamNames(i) + self.GetArrayVarNames(i)
                         + self.GetArrayParamNames(i) + self.GetGroupParamNames(i))
                return {n: self.GetStatus(i, n) for n in names}
            raise ValueError("Unknown object type in GetStatus")
        if isinstance(var_key, (str, bytes)):
            if isinstance(gen_object, ConnectionId):
                return self.GetConnectionStatus(gen_object)[var_key]
            if isinstance(gen_object, int):
                return self.GetNeuronStatus([gen_object], var_key)[0]
            raise ValueError("Unknown object type in GetStatus")
        raise ValueError("Unknown key type in GetStatus", type(var_key))

    # -- extensions of this build ------------------------------------------
    def Reset(self):
        "Destroy the simulation instance (new network in the same process)"
        return self._call("NGB200_Reset")

    def StageEvaluations(self):
        return self._call("NGB200_StageEvaluations")

    def DeliveredEvents(self):
        return self._call("NGB200_DeliveredEvents")

    def TotalSpikes(self):
        return self._call("NGB200_TotalSpikes")

    def LastSimulateSeconds(self):
        return self._call("NGB200_LastSimulateSeconds")

    def SetGraphChunk(self, n_steps):
        return self._call("NGB200_SetGraphChunk", ctypes.c_int(n_steps))

    def SetRk5MaxSubsteps(self, n_substeps):
        """RK5 sub-steps one neuron may take in one time step before
        Simulate fails with "RK5 integration exceeded the substep limit"
        (extension; default 200,000)."""
        return self._call("NGB200_SetRk5MaxSubsteps", ctypes.c_int(n_substeps))

    def SetWaitTest(self, mask):
        """Test hook (extension): bit 0 / bit 1 make the marked bounded
        device waits give up after one non-blocking test, so their time-out
        paths can be exercised; 0 restores normal waits."""
        return self._call("NGB200_SetWaitTest", ctypes.c_int(mask))

    def ProposerPhaseAfter(self, phase_in, ok1, ok2):
        """Host copy of the step proposer's barrier-parity bookkeeping
        (extension, for tests)."""
        return self._c["NGB200_ProposerPhaseAfter"](ctypes.c_uint(phase_in), ctypes.c_int(int(ok1)),
                                                    ctypes.c_int(int(ok2)))

    def LastSimulateDeviceMs(self):
        return self._call("NGB200_LastSimulateDeviceMs")

    def KernelsPerStep(self):
        "Kernel launches per time step in the last captured step graph"
        return self._call("NGB200_KernelsPerStep")

    def NNodes(self):
        return self._call("NGB200_NNodes")

    def NConnections(self):
        return self._call("NGB200_NConnections")

    def SetRk5Batching(self, on):
        """Extension: one RK5 launch per step for all groups of one model and
        port count (default on); call before the first simulation."""
        return self._call("NGB200_SetRk5Batching", ctypes.c_int(1 if on else 0))

    def Rk5BatchOf(self, i_node):
        return self._call("NGB200_Rk5BatchOf", ctypes.c_int(i_node))

    # -- learned RK5 step proposer (extension) ------------------------------
    MLP_NPARAM = 1313

    @staticmethod
    def _node_index(nodes):
        if nodes is None:
            return -1
        if isinstance(nodes, NodeSeq):
            return nodes.i0
        return int(nodes)

    def SetStepLog(self, nodes, capacity):
        """Log accepted RK5 sub-steps of the group of `nodes` (None: every
        supported group) for training the step proposer."""
        return self._call("NGB200_SetStepLog", ctypes.c_int(self._node_index(nodes)),
                          ctypes.c_int(capacity))

    def GetStepLogCount(self, nodes=None):
        return self._call("NGB200_GetStepLogCount", ctypes.c_int(self._node_index(nodes)))

    def GetStepLog(self, nodes=None, max_rows=1 << 20):
        import numpy as np
        out = np.zeros((max_rows, 8), dtype=np.float32)
        n = self._call("NGB200_GetStepLog", ctypes.c_int(self._node_index(nodes)),
                       out.ctypes.data_as(c_float_p), ctypes.c_int(max_rows))
        return out[:n]

    def TrainStepProposer(self, steps=4000, blocks=64, lr=3e-3, seed=1):
        """Trains the proposer on the logged sub-steps on the GPU; returns
        (rows, loss over the first 5% of steps, loss over the last 5%)."""
        l0, l1 = ctypes.c_float(0.0), ctypes.c_float(0.0)
        n = self._call("NGB200_TrainStepProposer", ctypes.c_int(steps), ctypes.c_int(blocks),
                       ctypes.c_float(lr), ctypes.c_ulonglong(seed), ctypes.byref(l0),
                       ctypes.byref(l1))
        return n, l0.value, l1.value

    def SetStepProposer(self, nodes, on=True):
        return self._call("NGB200_SetStepProposer", ctypes.c_int(self._node_index(nodes)),
                          ctypes.c_int(1 if on else 0))

    def SetStepProposerParams(self, params):
        import numpy as np
        p = np.ascontiguousarray(params, dtype=np.float32)
        if p.size != self.MLP_NPARAM:
            raise ValueError("the step proposer has %d parameters" % self.MLP_NPARAM)
        return self._call("NGB200_SetStepProposerParams", p.ctypes.data_as(c_float_p))

    def GetStepProposerParams(self):
        import numpy as np
        p = np.zeros(self.MLP_NPARAM, dtype=np.float32)
        self._call("NGB200_GetStepProposerParams", p.ctypes.data_as(c_float_p))
        return p

    def SetStepProposerMargin(self, margin):
        return self._call("NGB200_SetStepProposerMargin", ctypes.c_float(margin))

    def MlpGradients(self, data, params):
        """Mean gradient and loss of the GPU training kernels over the rows
        of `data` ([n, 8]: 6 features, target, unused)."""
        import numpy as np
        d = np.ascontiguousarray(data, dtype=np.float32)
        p = np.ascontiguousarray(params, dtype=np.float32)
        g = np.zeros(self.MLP_NPARAM, dtype=np.float32)
        loss = self._call("NGB200_MlpGradients", d.ctypes.data_as(c_float_p),
                          ctypes.c_int(d.shape[0]), p.ctypes.data_as(c_float_p),
                          g.ctypes.data_as(c_float_p))
        return g, loss

    def MlpInfer(self, x6, params):
        """Tensor-core inference of the proposer network on rows of 6 features."""
        import numpy as np
        x = np.ascontiguousarray(x6, dtype=np.float32)
        p = np.ascontiguousarray(params, dtype=np.float32)
        out = np.zeros(x.shape[0], dtype=np.float32)
        self._call("NGB200_MlpInfer", x.ctypes.data_as(c_float_p), ctypes.c_int(x.shape[0]),
                   p.ctypes.data_as(c_float_p), out.ctypes.data_as(c_float_p))
        return out

    def GetAllConnections(self):
        """Every connection as numpy arrays (source, target, port, syn_group,
        delay, weight) in delivery order, in one library call."""
        import numpy as np
        m = self.NConnections()
        cols = [np.zeros(m, dtype=np.int32) for _ in range(4)] + \
               [np.zeros(m, dtype=np.float32) for _ in range(2)]
        ptrs = [c.ctypes.data_as(c_int_p) for c in cols[:4]] + \
               [c.ctypes.data_as(c_float_p) for c in cols[4:]]
        self._call("NGB200_GetAllConnections", *ptrs)
        return dict(zip(("source", "target", "port", "syn", "delay", "weight"), cols))

    def SetKernelTiming(self, on):
        return self._call("NGB200_SetKernelTiming", ctypes.c_int(1 if on else 0))

    def GetKernelTiming(self, kind):
        "(total device ms, launches) of kernel class kind (0 update, 1 deliver, 2 stdp, 3 other)"
        t = ctypes.c_double(0.0)
        n = ctypes.c_longlong(0)
        self._call("NGB200_GetKernelTiming", ctypes.c_int(kind), ctypes.byref(t), ctypes.byref(n))
        return t.value, n.value

    def GetRk5Tuning(self, i_node):
        "(chosen RK5 kernel variant, [ms of variants 0..8]) for the group of i_node"
        v = ctypes.c_int(0)
        ms = (ctypes.c_float * 9)()
        self._call("NGB200_GetRk5Tuning", ctypes.c_int(i_node), ctypes.byref(v), ms)
        return v.value, list(ms)

    def StreamingDeliveryRate(self, n_slots, n_events, reps=10):
        """Events/s of the delivery's inner loop alone (n_events edges into
        n_slots accumulators): the bound of the delivery kernel"""
        r = ctypes.c_double(0.0)
        rc = self._c["NGB200_StreamingDeliveryRate"](ctypes.c_longlong(n_slots),
                                                     ctypes.c_longlong(n_events),
                                                     ctypes.c_int(reps), ctypes.byref(r))
        if rc != 0:
            raise ValueError("streaming delivery probe failed (%d)" % rc)
        return r.value

    # -- networks partitioned over hosts ---------------------------------
    def SetInstance(self, k):
        "Select simulation instance k (0..15) for every later call"
        if self._call("NGB200_SetInstance", ctypes.c_int(k)) != 0:
            raise ValueError("instance index out of range")
        return 0

    def GetInstance(self):
        return self._call("NGB200_GetInstance")

    def SetHost(self, i_host, n_hosts):
        "Host index and host count of this instance (partitioned networks)"
        return self._call("NGB200_SetHost", ctypes.c_int(i_host), ctypes.c_int(n_hosts))

    def SimulateSteps(self, n_steps):
        "Run n_steps steps of a started simulation"
        return self._call("NGB200_SimulateSteps", ctypes.c_longlong(n_steps))

    def RemoteExchangeSteps(self):
        "Shortest delay (steps) of a connection from an image node (0: none)"
        return self._call("NGB200_RemoteExchangeSteps")

    def PackRemoteSpikes(self, n_steps, buf_ptr, cap):
        """Spikes of this host's exported nodes in the last n_steps steps into
        the device buffer at buf_ptr (4 + 3 cap int32 words); returns the
        count, which may exceed cap (then pack again into a larger buffer)"""
        return self._call("NGB200_PackRemoteSpikes", ctypes.c_int(n_steps),
                          ctypes.c_void_p(buf_ptr), ctypes.c_longlong(cap))

    def UnpackRemoteSpikes(self, src_host, n_steps, buf_ptr, count):
        "Push host src_host's packed spikes (device buffer) into the images here"
        return self._call("NGB200_UnpackRemoteSpikes", ctypes.c_int(src_host),
                          ctypes.c_int(n_steps), ctypes.c_void_p(buf_ptr),
                          ctypes.c_longlong(count))


class HostComm(object):
    """Collectives of the hosts of a partitioned network over
    torch.distributed: NCCL (device tensors over NVLink) when the process
    group uses it, gloo otherwise. The default process group is created
    from the launcher's environment (RANK, WORLD_SIZE, MASTER_ADDR,
    MASTER_PORT) if none exists."""

    def __init__(self):
        import torch
        import torch.distributed as dist
        self._torch, self._dist = torch, dist
        if not dist.is_initialized():
            dist.init_process_group(backend="nccl" if torch.cuda.is_available() else "gloo")
        self.rank = dist.get_rank()
        self.size = dist.get_world_size()
        if dist.get_backend() == "nccl":
            self.device = torch.device("cuda", torch.cuda.current_device())
        else:
            self.device = torch.device("cpu")

    def _t(self, vals):
        return self._torch.tensor(vals, dtype=self._torch.int64, device=self.device)

    def broadcast_int(self, v, src):
        t = self._t([int(v)])
        self._dist.broadcast(t, src)
        return int(t.item())

    def min_int(self, v):
        t = self._t([int(v)])
        self._dist.all_reduce(t, op=self._dist.ReduceOp.MIN)
        return int(t.item())

    def allgather_int(self, v):
        parts = [self._t([0]) for _ in range(self.size)]
        self._dist.all_gather(parts, self._t([int(v)]))
        return [int(p.item()) for p in parts]

    def empty_u32(self, n):
        return self._torch.zeros(n, dtype=self._torch.int32, device=self.device)

    def allgather_rows(self, buf, n):
        parts = [self.empty_u32(n) for _ in range(self.size)]
        self._dist.all_gather(parts, buf[:n].contiguous())
        if self.device.type == "cuda":
            self._torch.cuda.current_stream().synchronize()
        return parts

    def row_ptr(self, rows, h):
        return rows[h].data_ptr()

    def sync(self):
        if self.device.type == "cuda":
            self._torch.cuda.synchronize()


_default = None
_PUBLIC = [n for n in dir(Binding) if not n.startswith("_")]


def _bind_module(binding):
    mod = sys.modules[__name__]
    for n in _PUBLIC:
        setattr(mod, n, getattr(binding, n))


def default_binding():
    """The binding behind the module-level functions (loads the library)."""
    global _default
    if _default is None:
        _default = Binding()
        _bind_module(_default)
    return _default


def __getattr__(name):
    # module-level API functions load the library on first use
    if name in _PUBLIC:
        return getattr(default_binding(), name)
    raise AttributeError(name)
