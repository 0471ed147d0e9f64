"""Python interface of the B200 spiking engine.

Same module name, functions, argument meaning and errors as NEST GPU's
pythonlib/nestgpu.py (NEST GPU 1.08), written against the same C ABI: it loads
libnestgpu_b200.so from this package's lib/ directory, or the library named by
the NESTGPU_LIB environment variable (so the reference library can be driven by
the same scripts).  Every failing call raises ValueError with the engine's
message (the reference turns C-ABI error codes into ValueError the same way).

Extensions with no counterpart in the reference: Reset, GetStats, ConnectArrays,
SetGraphSteps (they need libnestgpu_b200.so).
"""
import ctypes
import gc
import os

_here = os.path.dirname(os.path.abspath(__file__))
_default_lib = os.path.join(_here, "lib", "libnestgpu_b200.so")
lib_path = os.environ.get("NESTGPU_LIB", _default_lib)
if not os.path.exists(lib_path):
    raise ImportError("nestgpu: engine library not found at %s (build it with `make -C %s`)"
                      % (lib_path, _here))
_lib = ctypes.CDLL(lib_path)
is_b200_engine = hasattr(_lib, "NGPU_Reset")

c_float_p = ctypes.POINTER(ctypes.c_float)
c_int_p = ctypes.POINTER(ctypes.c_int)
c_char_p = ctypes.POINTER(ctypes.c_char)
c_void_p = ctypes.c_void_p
c_int_pp = ctypes.POINTER(ctypes.POINTER(ctypes.c_int))
c_float_pp = ctypes.POINTER(ctypes.POINTER(ctypes.c_float))
c_float_ppp = ctypes.POINTER(ctypes.POINTER(ctypes.POINTER(ctypes.c_float)))
c_char_pp = ctypes.POINTER(ctypes.c_char_p)

conn_rule_name = ("one_to_one", "all_to_all", "fixed_total_number", "fixed_indegree",
                  "fixed_outdegree")


def _bind(name, res, args):
    f = getattr(_lib, name)
    f.restype = res
    f.argtypes = args
    return f


_I, _F, _U8 = ctypes.c_int, ctypes.c_float, ctypes.c_ubyte
_sigs = {
    "NESTGPU_GetErrorMessage": (ctypes.c_char_p, []),
    "NESTGPU_GetErrorCode": (ctypes.c_ubyte, []),
    "NESTGPU_SetOnException": (None, [_I]),
    "NESTGPU_SetRandomSeed": (_I, [ctypes.c_ulonglong]),
    "NESTGPU_SetTimeResolution": (_I, [_F]),
    "NESTGPU_GetTimeResolution": (_F, []),
    "NESTGPU_SetMaxSpikeBufferSize": (_I, [_I]),
    "NESTGPU_GetMaxSpikeBufferSize": (_I, []),
    "NESTGPU_SetSimTime": (_I, [_F]),
    "NESTGPU_SetVerbosityLevel": (_I, [_I]),
    "NESTGPU_Create": (_I, [ctypes.c_char_p, _I, _I]),
    "NESTGPU_CreatePoissonGenerator": (_I, [_I, _F]),
    "NESTGPU_CreateRecord": (_I, [ctypes.c_char_p, c_char_pp, c_int_p, c_int_p, _I]),
    "NESTGPU_GetRecordDataRows": (_I, [_I]),
    "NESTGPU_GetRecordDataColumns": (_I, [_I]),
    "NESTGPU_GetRecordData": (c_float_pp, [_I]),
    "NESTGPU_SetNeuronScalParam": (_I, [_I, _I, ctypes.c_char_p, _F]),
    "NESTGPU_SetNeuronArrayParam": (_I, [_I, _I, ctypes.c_char_p, c_float_p, _I]),
    "NESTGPU_SetNeuronPtScalParam": (_I, [c_void_p, _I, ctypes.c_char_p, _F]),
    "NESTGPU_SetNeuronPtArrayParam": (_I, [c_void_p, _I, ctypes.c_char_p, c_float_p, _I]),
    "NESTGPU_IsNeuronScalParam": (_I, [_I, ctypes.c_char_p]),
    "NESTGPU_IsNeuronPortParam": (_I, [_I, ctypes.c_char_p]),
    "NESTGPU_IsNeuronArrayParam": (_I, [_I, ctypes.c_char_p]),
    "NESTGPU_SetNeuronIntVar": (_I, [_I, _I, ctypes.c_char_p, _I]),
    "NESTGPU_SetNeuronScalVar": (_I, [_I, _I, ctypes.c_char_p, _F]),
    "NESTGPU_SetNeuronArrayVar": (_I, [_I, _I, ctypes.c_char_p, c_float_p, _I]),
    "NESTGPU_SetNeuronPtIntVar": (_I, [c_void_p, _I, ctypes.c_char_p, _I]),
    "NESTGPU_SetNeuronPtScalVar": (_I, [c_void_p, _I, ctypes.c_char_p, _F]),
    "NESTGPU_SetNeuronPtArrayVar": (_I, [c_void_p, _I, ctypes.c_char_p, c_float_p, _I]),
    "NESTGPU_IsNeuronIntVar": (_I, [_I, ctypes.c_char_p]),
    "NESTGPU_IsNeuronScalVar": (_I, [_I, ctypes.c_char_p]),
    "NESTGPU_IsNeuronPortVar": (_I, [_I, ctypes.c_char_p]),
    "NESTGPU_IsNeuronArrayVar": (_I, [_I, ctypes.c_char_p]),
    "NESTGPU_GetNeuronParamSize": (_I, [_I, ctypes.c_char_p]),
    "NESTGPU_GetNeuronVarSize": (_I, [_I, ctypes.c_char_p]),
    "NESTGPU_GetNeuronParam": (c_float_p, [_I, _I, ctypes.c_char_p]),
    "NESTGPU_GetNeuronPtParam": (c_float_p, [c_void_p, _I, ctypes.c_char_p]),
    "NESTGPU_GetArrayParam": (c_float_p, [_I, ctypes.c_char_p]),
    "NESTGPU_GetNeuronIntVar": (c_int_p, [_I, _I, ctypes.c_char_p]),
    "NESTGPU_GetNeuronPtIntVar": (c_int_p, [c_void_p, _I, ctypes.c_char_p]),
    "NESTGPU_GetNeuronVar": (c_float_p, [_I, _I, ctypes.c_char_p]),
    "NESTGPU_GetNeuronPtVar": (c_float_p, [c_void_p, _I, ctypes.c_char_p]),
    "NESTGPU_GetArrayVar": (c_float_p, [_I, ctypes.c_char_p]),
    "NESTGPU_Calibrate": (_I, []),
    "NESTGPU_Simulate": (_I, []),
    "NESTGPU_StartSimulation": (_I, []),
    "NESTGPU_SimulationStep": (_I, []),
    "NESTGPU_EndSimulation": (_I, []),
    "NESTGPU_MpiId": (_I, []),
    "NESTGPU_MpiNp": (_I, []),
    "NESTGPU_ProcMaster": (_I, []),
    "NESTGPU_MpiFinalize": (_I, []),
    "NESTGPU_RandomInt": (ctypes.POINTER(ctypes.c_uint), [ctypes.c_size_t]),
    "NESTGPU_RandomUniform": (c_float_p, [ctypes.c_size_t]),
    "NESTGPU_RandomNormal": (c_float_p, [ctypes.c_size_t, _F, _F]),
    "NESTGPU_RandomNormalClipped": (c_float_p, [ctypes.c_size_t, _F, _F, _F, _F, _F]),
    "NESTGPU_Connect": (_I, [_I, _I, _U8, _U8, _F, _F]),
    "NESTGPU_ConnSpecInit": (_I, []),
    "NESTGPU_SetConnSpecParam": (_I, [ctypes.c_char_p, _I]),
    "NESTGPU_ConnSpecIsParam": (_I, [ctypes.c_char_p]),
    "NESTGPU_SynSpecInit": (_I, []),
    "NESTGPU_SetSynSpecIntParam": (_I, [ctypes.c_char_p, _I]),
    "NESTGPU_SetSynSpecFloatParam": (_I, [ctypes.c_char_p, _F]),
    "NESTGPU_SetSynSpecFloatPtParam": (_I, [ctypes.c_char_p, c_void_p]),
    "NESTGPU_SynSpecIsIntParam": (_I, [ctypes.c_char_p]),
    "NESTGPU_SynSpecIsFloatParam": (_I, [ctypes.c_char_p]),
    "NESTGPU_SynSpecIsFloatPtParam": (_I, [ctypes.c_char_p]),
    "NESTGPU_ConnectSeqSeq": (_I, [_I, _I, _I, _I]),
    "NESTGPU_ConnectSeqGroup": (_I, [_I, _I, c_void_p, _I]),
    "NESTGPU_ConnectGroupSeq": (_I, [c_void_p, _I, _I, _I]),
    "NESTGPU_ConnectGroupGroup": (_I, [c_void_p, _I, c_void_p, _I]),
    "NESTGPU_GetSeqSeqConnections": (c_int_p, [_I, _I, _I, _I, _I, c_int_p]),
    "NESTGPU_GetSeqGroupConnections": (c_int_p, [_I, _I, c_void_p, _I, _I, c_int_p]),
    "NESTGPU_GetGroupSeqConnections": (c_int_p, [c_void_p, _I, _I, _I, _I, c_int_p]),
    "NESTGPU_GetGroupGroupConnections": (c_int_p, [c_void_p, _I, c_void_p, _I, _I, c_int_p]),
    "NESTGPU_GetConnectionStatus": (_I, [_I, _I, _I, c_int_p, c_char_p, c_char_p, c_float_p, c_float_p]),
    "NESTGPU_ActivateSpikeCount": (_I, [_I, _I]),
    "NESTGPU_ActivateRecSpikeTimes": (_I, [_I, _I, _I]),
    "NESTGPU_SetRecSpikeTimesStep": (_I, [_I, _I, _I]),
    "NESTGPU_GetNRecSpikeTimes": (_I, [_I]),
    "NESTGPU_GetRecSpikeTimes": (_I, [_I, _I, c_int_pp, c_float_ppp]),
    "NESTGPU_SetNeuronGroupParam": (_I, [_I, _I, ctypes.c_char_p, _F]),
    "NESTGPU_IsNeuronGroupParam": (_I, [_I, ctypes.c_char_p]),
    "NESTGPU_GetNeuronGroupParam": (_F, [_I, ctypes.c_char_p]),
    "NESTGPU_GetNBoolParam": (_I, []),
    "NESTGPU_GetBoolParamNames": (c_char_pp, []),
    "NESTGPU_IsBoolParam": (_I, [ctypes.c_char_p]),
    "NESTGPU_GetBoolParam": (ctypes.c_bool, [ctypes.c_char_p]),
    "NESTGPU_SetBoolParam": (_I, [ctypes.c_char_p, ctypes.c_bool]),
    "NESTGPU_GetNFloatParam": (_I, []),
    "NESTGPU_GetFloatParamNames": (c_char_pp, []),
    "NESTGPU_IsFloatParam": (_I, [ctypes.c_char_p]),
    "NESTGPU_GetFloatParam": (_F, [ctypes.c_char_p]),
    "NESTGPU_SetFloatParam": (_I, [ctypes.c_char_p, _F]),
    "NESTGPU_GetNIntParam": (_I, []),
    "NESTGPU_GetIntParamNames": (c_char_pp, []),
    "NESTGPU_IsIntParam": (_I, [ctypes.c_char_p]),
    "NESTGPU_GetIntParam": (_I, [ctypes.c_char_p]),
    "NESTGPU_SetIntParam": (_I, [ctypes.c_char_p, _I]),
    "NESTGPU_CreateSynGroup": (_I, [ctypes.c_char_p]),
    "NESTGPU_GetSynGroupNParam": (_I, [_I]),
    "NESTGPU_GetSynGroupParamNames": (c_char_pp, [_I]),
    "NESTGPU_IsSynGroupParam": (_I, [_I, ctypes.c_char_p]),
    "NESTGPU_GetSynGroupParamIdx": (_I, [_I, ctypes.c_char_p]),
    "NESTGPU_GetSynGroupParam": (_F, [_I, ctypes.c_char_p]),
    "NESTGPU_SetSynGroupParam": (_I, [_I, ctypes.c_char_p, _F]),
}
for _n in ("IntVar", "ScalVar", "PortVar", "ScalParam", "PortParam", "GroupParam", "ArrayParam",
           "ArrayVar"):
    _sigs["NESTGPU_Get%sNames" % _n] = (c_char_pp, [_I])
    _sigs["NESTGPU_GetN%s" % _n] = (_I, [_I])
_c = {name: _bind(name, r, a) for name, (r, a) in _sigs.items()}
if is_b200_engine:
    _c["NGPU_FreeArray"] = _bind("NGPU_FreeArray", None, [c_void_p])
    _c["NGPU_Reset"] = _bind("NGPU_Reset", _I, [])
    _c["NGPU_GetStats"] = _bind("NGPU_GetStats", _I, [ctypes.POINTER(ctypes.c_ulonglong)] * 3 +
                                [ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_longlong),
                                 ctypes.POINTER(ctypes.c_uint)])
    _c["NGPU_ConnectArrays"] = _bind("NGPU_ConnectArrays", _I, [ctypes.c_size_t, c_void_p, c_void_p,
                                                                 c_void_p, c_void_p, c_void_p])
    _c["NGPU_SetGraphSteps"] = _bind("NGPU_SetGraphSteps", _I, [_I])
    _c["NGPU_SetHostRng"] = _bind("NGPU_SetHostRng", _I, [_I])
    _c["NGPU_SetRk5Budget"] = _bind("NGPU_SetRk5Budget", _I, [_I])
    _c["NGPU_SetDeliverBlocks"] = _bind("NGPU_SetDeliverBlocks", _I, [_I])
    _c["NGPU_SetBatchMax"] = _bind("NGPU_SetBatchMax", _I, [_I])
    _c["NGPU_SetUpdateThreads"] = _bind("NGPU_SetUpdateThreads", _I, [_I])
    _c["NGPU_SetDeliverGroup"] = _bind("NGPU_SetDeliverGroup", _I, [_I])
    _c["NGPU_SetProgrammaticLaunch"] = _bind("NGPU_SetProgrammaticLaunch", _I, [_I])
    _c["NGPU_SetUpdateOccupancy"] = _bind("NGPU_SetUpdateOccupancy", _I, [_I])
    _c["NGPU_SetUpdateTrialIter"] = _bind("NGPU_SetUpdateTrialIter", _I, [_I])
    _c["NGPU_SetDeliverAggregate"] = _bind("NGPU_SetDeliverAggregate", _I, [_I])
    _c["NGPU_SetDeliverPrefetch"] = _bind("NGPU_SetDeliverPrefetch", _I, [_I])
    _c["NGPU_SetDeliverPush"] = _bind("NGPU_SetDeliverPush", _I, [_I])
    _c["NGPU_DeliverPushActive"] = _bind("NGPU_DeliverPushActive", _I, [])
    _c["NGPU_SetPartition"] = _bind("NGPU_SetPartition", _I, [_I, _I])
    _c["NGPU_SetExchange"] = _bind("NGPU_SetExchange", _I, [c_void_p, c_void_p, ctypes.c_longlong, c_void_p,
                                                             c_void_p])
    _c["NGPU_GetBatchLength"] = _bind("NGPU_GetBatchLength", _I, [])
    _c["NGPU_SetPersistent"] = _bind("NGPU_SetPersistent", _I, [_I])
    _c["NGPU_TestBarrierTimeout"] = _bind("NGPU_TestBarrierTimeout", _I, [_I])
    _c["NGPU_TestTensorWaitTimeout"] = _bind("NGPU_TestTensorWaitTimeout", _I, [_I])
    _c["NGPU_Autotune"] = _bind("NGPU_Autotune", _I, [_I] + [ctypes.POINTER(_I)] * 4)
    _c["NGPU_GetLaunchMapping"] = _bind("NGPU_GetLaunchMapping", _I, [ctypes.POINTER(_I), _I])
    _c["NGPU_MeasureReductionRate"] = _bind("NGPU_MeasureReductionRate", ctypes.c_double,
                                            [ctypes.c_size_t, ctypes.c_longlong])
    _c["NGPU_GetSimDeviceMs"] = _bind("NGPU_GetSimDeviceMs", ctypes.c_double, [])
    _c["NGPU_GetLaunchCount"] = _bind("NGPU_GetLaunchCount", ctypes.c_longlong, [])
    _c["NGPU_ProfileSteps"] = _bind("NGPU_ProfileSteps", _I, [_I, ctypes.POINTER(ctypes.c_double)])
    _LL = ctypes.c_longlong
    _c["NGPU_StepModelNParams"] = _bind("NGPU_StepModelNParams", _I, [])
    _c["NGPU_Rk5LogStart"] = _bind("NGPU_Rk5LogStart", _I, [_LL])
    _c["NGPU_Rk5LogStop"] = _bind("NGPU_Rk5LogStop", _I, [])
    _c["NGPU_Rk5LogCount"] = _bind("NGPU_Rk5LogCount", _LL, [ctypes.POINTER(_LL)])
    _c["NGPU_Rk5LogGet"] = _bind("NGPU_Rk5LogGet", _I, [c_void_p, _LL, _LL])
    _c["NGPU_StepModelTrain"] = _bind("NGPU_StepModelTrain", _I, [_LL, _I, ctypes.c_float, ctypes.c_float,
                                                                  ctypes.c_float, ctypes.c_ulonglong, ctypes.POINTER(_LL),
                                                                  ctypes.POINTER(ctypes.c_float)])
    _c["NGPU_StepModelSet"] = _bind("NGPU_StepModelSet", _I, [c_void_p])
    _c["NGPU_StepModelGet"] = _bind("NGPU_StepModelGet", _I, [c_void_p])
    _c["NGPU_StepModelEnable"] = _bind("NGPU_StepModelEnable", _I, [_I])
    _c["NGPU_StepBoundMode"] = _bind("NGPU_StepBoundMode", _I, [_I])
    _c["NGPU_MlpForward"] = _bind("NGPU_MlpForward", _I, [c_void_p, c_void_p, _I, c_void_p])
    _c["NGPU_MlpGrad"] = _bind("NGPU_MlpGrad", _I, [c_void_p, c_void_p, c_void_p, _I, c_void_p, c_void_p])
    _c["NGPU_ConnectFixedIndegreeGPU"] = _bind("NGPU_ConnectFixedIndegreeGPU", _I,
                                               [_I, _I, _I, _I, _I, _I, _F, _F, _F, ctypes.c_ulonglong])
    _c["NGPU_SetPoissonStream"] = _bind("NGPU_SetPoissonStream", _I, [_I, _I, ctypes.c_uint])
    _c["NGPU_SetDeviceRuleMinEdges"] = _bind("NGPU_SetDeviceRuleMinEdges", _I, [ctypes.c_longlong])
    _c["NGPU_GetDeliveryShape"] = _bind("NGPU_GetDeliveryShape", _I, [ctypes.POINTER(_I)] * 3 +
                                        [ctypes.POINTER(ctypes.c_longlong)])
    _c["NGPU_GetDeliveryCsr"] = _bind("NGPU_GetDeliveryCsr", _I, [c_void_p] * 4)


def _b(s):
    return s.encode("utf-8") if isinstance(s, str) else s


def _check(ret=None):
    if _c["NESTGPU_GetErrorCode"]() != 0:
        raise ValueError(GetErrorMessage())
    return ret


def _free(p):
    if is_b200_engine and p:
        _c["NGPU_FreeArray"](ctypes.cast(p, c_void_p))


def _names(fn, *args):
    n = _c["NESTGPU_GetN" + fn](*args) if fn else None
    pp = _c["NESTGPU_Get%sNames" % fn](*args)
    _check()
    out = [pp[i].decode("utf-8") for i in range(n)]
    return out


class NodeSeq(object):
    """Contiguous range of node indices (i0, n); n = -1 with i0 = None means all nodes."""

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
    def __init__(self, i_host=0, node_seq=NodeSeq(None)):
        self.i_host = i_host
        self.node_seq = node_seq


class ConnectionId(object):
    def __init__(self, i_source, i_group, i_conn):
        self.i_source = i_source
        self.i_group = i_group
        self.i_conn = i_conn


class SynGroup(object):
    def __init__(self, i_syn_group):
        self.i_syn_group = i_syn_group


# ---------------------------------------------------------------- errors, kernel
def GetErrorMessage():
    return _c["NESTGPU_GetErrorMessage"]().decode("utf-8")


def GetErrorCode():
    return _c["NESTGPU_GetErrorCode"]()


def SetOnException(on_exception):
    _c["NESTGPU_SetOnException"](on_exception)


SetOnException(1)   # return errors to Python instead of exiting (reference nestgpu.py:115-119)


def SetRandomSeed(seed):
    return _check(_c["NESTGPU_SetRandomSeed"](seed))


def SetTimeResolution(time_res):
    return _check(_c["NESTGPU_SetTimeResolution"](time_res))


def GetTimeResolution():
    return _check(_c["NESTGPU_GetTimeResolution"]())


def SetMaxSpikeBufferSize(max_size):
    return _check(_c["NESTGPU_SetMaxSpikeBufferSize"](max_size))


def GetMaxSpikeBufferSize():
    return _check(_c["NESTGPU_GetMaxSpikeBufferSize"]())


def SetSimTime(sim_time):
    return _check(_c["NESTGPU_SetSimTime"](sim_time))


def SetVerbosityLevel(verbosity_level):
    return _check(_c["NESTGPU_SetVerbosityLevel"](verbosity_level))


# ---------------------------------------------------------------- nodes
def Create(model_name, n_node=1, n_ports=1, status_dict=None):
    "Create a neuron group"
    if isinstance(status_dict, dict):
        group = Create(model_name, n_node, n_ports)
        SetStatus(group, status_dict)
        return group
    elif status_dict is not None:
        raise ValueError("Wrong argument in Create")
    i_node = _c["NESTGPU_Create"](_b(model_name), n_node, n_ports)
    return _check(NodeSeq(i_node, n_node))


def CreatePoissonGenerator(n_node, rate):
    i_node = _c["NESTGPU_CreatePoissonGenerator"](n_node, rate)
    return _check(NodeSeq(i_node, n_node))


def CreateRecord(file_name, var_name_list, i_node_list, i_port_list):
    "Create a record of neuron variables"
    n = len(i_node_list)
    names = (ctypes.c_char_p * n)(*[_b(v) for v in var_name_list])
    ret = _c["NESTGPU_CreateRecord"](_b(file_name), names, (ctypes.c_int * n)(*i_node_list),
                                     (ctypes.c_int * n)(*i_port_list), n)
    return _check(ret)


def GetRecordDataRows(i_record):
    return _check(_c["NESTGPU_GetRecordDataRows"](i_record))


def GetRecordDataColumns(i_record):
    return _check(_c["NESTGPU_GetRecordDataColumns"](i_record))


def GetRecordData(i_record):
    "Get record data: one list per recorded step, time first"
    pt = _c["NESTGPU_GetRecordData"](i_record)
    _check()
    nr = GetRecordDataRows(i_record)
    nc = GetRecordDataColumns(i_record)
    return [[pt[ir][ic] for ic in range(nc)] for ir in range(nr)]


def _float_arr(vals):
    vals = list(vals)
    return (ctypes.c_float * len(vals))(*vals), len(vals)


def _int_arr(nodes):
    nodes = list(nodes)
    return ctypes.cast((ctypes.c_int * len(nodes))(*nodes), c_void_p), len(nodes)


def SetNeuronScalParam(i_node, n_node, param_name, val):
    return _check(_c["NESTGPU_SetNeuronScalParam"](i_node, n_node, _b(param_name), val))


def SetNeuronArrayParam(i_node, n_node, param_name, param_list):
    arr, n = _float_arr(param_list)
    return _check(_c["NESTGPU_SetNeuronArrayParam"](i_node, n_node, _b(param_name), arr, n))


def SetNeuronPtScalParam(nodes, param_name, val):
    pt, n = _int_arr(nodes)
    return _check(_c["NESTGPU_SetNeuronPtScalParam"](pt, n, _b(param_name), val))


def SetNeuronPtArrayParam(nodes, param_name, param_list):
    pt, n = _int_arr(nodes)
    arr, na = _float_arr(param_list)
    return _check(_c["NESTGPU_SetNeuronPtArrayParam"](pt, n, _b(param_name), arr, na))


def IsNeuronScalParam(i_node, param_name):
    return _check(_c["NESTGPU_IsNeuronScalParam"](i_node, _b(param_name)) != 0)


def IsNeuronPortParam(i_node, param_name):
    return _check(_c["NESTGPU_IsNeuronPortParam"](i_node, _b(param_name)) != 0)


def IsNeuronArrayParam(i_node, param_name):
    return _check(_c["NESTGPU_IsNeuronArrayParam"](i_node, _b(param_name)) != 0)


def IsNeuronGroupParam(i_node, param_name):
    return _check(_c["NESTGPU_IsNeuronGroupParam"](i_node, _b(param_name)) != 0)


def SetNeuronIntVar(i_node, n_node, var_name, val):
    return _check(_c["NESTGPU_SetNeuronIntVar"](i_node, n_node, _b(var_name), int(val)))


def SetNeuronScalVar(i_node, n_node, var_name, val):
    return _check(_c["NESTGPU_SetNeuronScalVar"](i_node, n_node, _b(var_name), val))


def SetNeuronArrayVar(i_node, n_node, var_name, var_list):
    arr, n = _float_arr(var_list)
    return _check(_c["NESTGPU_SetNeuronArrayVar"](i_node, n_node, _b(var_name), arr, n))


def SetNeuronPtIntVar(nodes, var_name, val):
    pt, n = _int_arr(nodes)
    return _check(_c["NESTGPU_SetNeuronPtIntVar"](pt, n, _b(var_name), int(val)))


def SetNeuronPtScalVar(nodes, var_name, val):
    pt, n = _int_arr(nodes)
    return _check(_c["NESTGPU_SetNeuronPtScalVar"](pt, n, _b(var_name), val))


def SetNeuronPtArrayVar(nodes, var_name, var_list):
    pt, n = _int_arr(nodes)
    arr, na = _float_arr(var_list)
    return _check(_c["NESTGPU_SetNeuronPtArrayVar"](pt, n, _b(var_name), arr, na))


def IsNeuronIntVar(i_node, var_name):
    return _check(_c["NESTGPU_IsNeuronIntVar"](i_node, _b(var_name)) != 0)


def IsNeuronScalVar(i_node, var_name):
    return _check(_c["NESTGPU_IsNeuronScalVar"](i_node, _b(var_name)) != 0)


def IsNeuronPortVar(i_node, var_name):
    return _check(_c["NESTGPU_IsNeuronPortVar"](i_node, _b(var_name)) != 0)


def IsNeuronArrayVar(i_node, var_name):
    return _check(_c["NESTGPU_IsNeuronArrayVar"](i_node, _b(var_name)) != 0)


def GetNeuronParamSize(i_node, param_name):
    return _check(_c["NESTGPU_GetNeuronParamSize"](i_node, _b(param_name)))


def GetNeuronVarSize(i_node, var_name):
    return _check(_c["NESTGPU_GetNeuronVarSize"](i_node, _b(var_name)))


def _rows(pt, n_node, size):
    """Python rows (lists for size > 1) from an engine-allocated float array, which is freed."""
    import numpy as np
    n = n_node * max(size, 1)
    a = np.ctypeslib.as_array(pt, shape=(n,)).astype(np.float64) if n > 0 else np.zeros(0)
    _free(pt)
    return a.reshape(n_node, size).tolist() if size > 1 else a.tolist()


def _ints(pt, n):
    """Python list from an engine-allocated int array, which is freed."""
    import numpy as np
    out = np.ctypeslib.as_array(pt, shape=(n,)).tolist() if n > 0 else []
    _free(pt)
    return out


def GetNeuronParam(i_node, n_node, param_name):
    pt = _c["NESTGPU_GetNeuronParam"](i_node, n_node, _b(param_name))
    _check()
    return _rows(pt, n_node, GetNeuronParamSize(i_node, param_name))


def GetNeuronPtParam(nodes, param_name):
    pt_n, n = _int_arr(nodes)
    pt = _c["NESTGPU_GetNeuronPtParam"](pt_n, n, _b(param_name))
    _check()
    return _rows(pt, n, GetNeuronParamSize(nodes[0], param_name))


def GetArrayParam(i_node, n_node, param_name):
    out = []
    for j in range(n_node):
        pt = _c["NESTGPU_GetArrayParam"](i_node + j, _b(param_name))
        _check()
        size = GetNeuronParamSize(i_node + j, param_name)
        out.append([pt[i] for i in range(size)])
        _free(pt)
    return out


def GetNeuronListArrayParam(node_list, param_name):
    out = []
    for nd in node_list:
        out += GetArrayParam(nd, 1, param_name)
    return out


def GetNeuronGroupParam(i_node, param_name):
    return _check(_c["NESTGPU_GetNeuronGroupParam"](i_node, _b(param_name)))


def GetNeuronIntVar(i_node, n_node, var_name):
    pt = _c["NESTGPU_GetNeuronIntVar"](i_node, n_node, _b(var_name))
    _check()
    return _ints(pt, n_node)


def GetNeuronVar(i_node, n_node, var_name):
    pt = _c["NESTGPU_GetNeuronVar"](i_node, n_node, _b(var_name))
    _check()
    return _rows(pt, n_node, GetNeuronVarSize(i_node, var_name))


def GetSpikeCountArray(nodes):
    """Spike counts of a node sequence as a NumPy int32 array (engine extension): the same
    device-to-host copy as GetStatus(nodes, "spike_count"), without building a Python list,
    for callers that read the counts of many neurons every call."""
    import numpy as np
    i0, n = _seq_args(nodes)
    pt = _c["NESTGPU_GetNeuronIntVar"](i0, n, _b("spike_count"))
    _check()
    out = np.ctypeslib.as_array(pt, shape=(n,)).copy() if n > 0 else np.zeros(0, dtype=np.int32)
    _free(pt)
    return out


def GetNeuronPtIntVar(nodes, var_name):
    pt_n, n = _int_arr(nodes)
    pt = _c["NESTGPU_GetNeuronPtIntVar"](pt_n, n, _b(var_name))
    _check()
    return _ints(pt, n)


def GetNeuronPtVar(nodes, var_name):
    pt_n, n = _int_arr(nodes)
    pt = _c["NESTGPU_GetNeuronPtVar"](pt_n, n, _b(var_name))
    _check()
    return _rows(pt, n, GetNeuronVarSize(nodes[0], var_name))


def GetArrayVar(i_node, n_node, var_name):
    out = []
    for j in range(n_node):
        pt = _c["NESTGPU_GetArrayVar"](i_node + j, _b(var_name))
        _check()
        size = GetNeuronVarSize(i_node + j, var_name)
        out.append([pt[i] for i in range(size)])
    return out


def GetNeuronListArrayVar(node_list, var_name):
    out = []
    for nd in node_list:
        out += GetArrayVar(nd, 1, var_name)
    return out


def _node_list(nodes):
    if isinstance(nodes, NodeSeq):
        return nodes.ToList()
    return list(nodes)


def GetNeuronStatus(nodes, var_name):
    "Get neuron group scalar or array variable or parameter"
    if not isinstance(nodes, (list, tuple, NodeSeq)):
        raise ValueError("Unknown node type")
    if isinstance(nodes, NodeSeq):
        i0, n = nodes.i0, nodes.n
        if IsNeuronScalParam(i0, var_name) or IsNeuronPortParam(i0, var_name):
            return GetNeuronParam(i0, n, var_name)
        if IsNeuronArrayParam(i0, var_name):
            return GetArrayParam(i0, n, var_name)
        if IsNeuronIntVar(i0, var_name):
            return GetNeuronIntVar(i0, n, var_name)
        if IsNeuronScalVar(i0, var_name) or IsNeuronPortVar(i0, var_name):
            return GetNeuronVar(i0, n, var_name)
        if IsNeuronArrayVar(i0, var_name):
            return GetArrayVar(i0, n, var_name)
        if IsNeuronGroupParam(i0, var_name):
            return GetNeuronStatus(nodes.ToList(), var_name)
        raise ValueError("Unknown neuron variable or parameter")
    nd0 = nodes[0]
    if IsNeuronScalParam(nd0, var_name) or IsNeuronPortParam(nd0, var_name):
        return GetNeuronPtParam(nodes, var_name)
    if IsNeuronArrayParam(nd0, var_name):
        return GetNeuronListArrayParam(nodes, var_name)
    if IsNeuronIntVar(nd0, var_name):
        return GetNeuronPtIntVar(nodes, var_name)
    if IsNeuronScalVar(nd0, var_name) or IsNeuronPortVar(nd0, var_name):
        return GetNeuronPtVar(nodes, var_name)
    if IsNeuronArrayVar(nd0, var_name):
        return GetNeuronListArrayVar(nodes, var_name)
    if IsNeuronGroupParam(nd0, var_name):
        return [GetNeuronGroupParam(nd, var_name) for nd in nodes]
    raise ValueError("Unknown neuron variable or parameter")


def GetNIntVar(i_node):
    return _check(_c["NESTGPU_GetNIntVar"](i_node))


def GetNScalVar(i_node):
    return _check(_c["NESTGPU_GetNScalVar"](i_node))


def GetIntVarNames(i_node):
    return _names("IntVar", i_node)


def GetScalVarNames(i_node):
    return _names("ScalVar", i_node)


def GetNPortVar(i_node):
    return _check(_c["NESTGPU_GetNPortVar"](i_node))


def GetPortVarNames(i_node):
    return _names("PortVar", i_node)


def GetNScalParam(i_node):
    return _check(_c["NESTGPU_GetNScalParam"](i_node))


def GetScalParamNames(i_node):
    return _names("ScalParam", i_node)


def GetNPortParam(i_node):
    return _check(_c["NESTGPU_GetNPortParam"](i_node))


def GetPortParamNames(i_node):
    return _names("PortParam", i_node)


def GetNArrayParam(i_node):
    return _check(_c["NESTGPU_GetNArrayParam"](i_node))


def GetArrayParamNames(i_node):
    return _names("ArrayParam", i_node)


def GetNGroupParam(i_node):
    return _check(_c["NESTGPU_GetNGroupParam"](i_node))


def GetGroupParamNames(i_node):
    return _names("GroupParam", i_node)


def GetNArrayVar(i_node):
    return _check(_c["NESTGPU_GetNArrayVar"](i_node))


def GetArrayVarNames(i_node):
    return _names("ArrayVar", i_node)


def SetNeuronGroupParam(nodes, param_name, val):
    nodes = nodes if isinstance(nodes, NodeSeq) else NodeSeq(nodes[0], len(nodes))
    return _check(_c["NESTGPU_SetNeuronGroupParam"](nodes.i0, nodes.n, _b(param_name), val))


def SetNeuronStatus(nodes, var_name, val):
    "Set neuron group scalar or array variable or parameter"
    if not isinstance(nodes, (list, tuple, NodeSeq)):
        raise ValueError("Unknown node type")
    if isinstance(val, dict):
        arr = DictToArray(val, len(nodes))
        nl = _node_list(nodes)
        for i in range(len(nl)):
            SetNeuronStatus([nl[i]], var_name, arr[i])
        return
    if isinstance(nodes, NodeSeq):
        i0, n = nodes.i0, nodes.n
        if IsNeuronGroupParam(i0, var_name):
            SetNeuronGroupParam(nodes, var_name, val)
        elif IsNeuronScalParam(i0, var_name):
            SetNeuronScalParam(i0, n, var_name, val)
        elif IsNeuronPortParam(i0, var_name) or IsNeuronArrayParam(i0, var_name):
            SetNeuronArrayParam(i0, n, var_name, val)
        elif IsNeuronIntVar(i0, var_name):
            SetNeuronIntVar(i0, n, var_name, val)
        elif IsNeuronScalVar(i0, var_name):
            SetNeuronScalVar(i0, n, var_name, val)
        elif IsNeuronPortVar(i0, var_name) or IsNeuronArrayVar(i0, var_name):
            SetNeuronArrayVar(i0, n, var_name, val)
        else:
            raise ValueError("Unknown neuron variable or parameter")
    else:
        nd0 = nodes[0]
        if IsNeuronScalParam(nd0, var_name):
            SetNeuronPtScalParam(nodes, var_name, val)
        elif IsNeuronPortParam(nd0, var_name) or IsNeuronArrayParam(nd0, var_name):
            SetNeuronPtArrayParam(nodes, var_name, val)
        elif IsNeuronIntVar(nd0, var_name):
            SetNeuronPtIntVar(nodes, var_name, val)
        elif IsNeuronScalVar(nd0, var_name):
            SetNeuronPtScalVar(nodes, var_name, val)
        elif IsNeuronPortVar(nd0, var_name) or IsNeuronArrayVar(nd0, var_name):
            SetNeuronPtArrayVar(nodes, var_name, val)
        elif IsNeuronGroupParam(nd0, var_name):
            SetNeuronGroupParam(nodes, var_name, val)
        else:
            raise ValueError("Unknown neuron variable or parameter")


# ---------------------------------------------------------------- simulation
def Calibrate():
    return _check(_c["NESTGPU_Calibrate"]())


def Simulate(sim_time=1000.0):
    "Simulate neural activity"
    SetSimTime(sim_time)
    return _check(_c["NESTGPU_Simulate"]())


def StartSimulation():
    return _check(_c["NESTGPU_StartSimulation"]())


def SimulationStep():
    return _check(_c["NESTGPU_SimulationStep"]())


def EndSimulation():
    return _check(_c["NESTGPU_EndSimulation"]())


def ConnectMpiInit():
    raise ValueError("MPI is not available (single-GPU engine)")


def MpiId():
    return _c["NESTGPU_MpiId"]()


def Rank():
    return MpiId()


def MpiNp():
    return _c["NESTGPU_MpiNp"]()


def ProcMaster():
    return _c["NESTGPU_ProcMaster"]()


def MpiFinalize():
    return _c["NESTGPU_MpiFinalize"]()


# ---------------------------------------------------------------- random numbers
def _copy_out(pt, ctype, n):
    """ctypes array holding a copy of an engine-allocated array of n elements (freed)."""
    out = (ctype * n)()
    if n > 0:
        ctypes.memmove(out, pt, n * ctypes.sizeof(ctype))
    _free(pt)
    return out


def RandomInt(n):
    pt = _c["NESTGPU_RandomInt"](n)
    _check()
    return list(_copy_out(pt, ctypes.c_uint, n))


def RandomUniform(n):
    pt = _c["NESTGPU_RandomUniform"](n)
    _check()
    return list(_copy_out(pt, ctypes.c_float, n))


def RandomNormal(n, mean, stddev):
    pt = _c["NESTGPU_RandomNormal"](n, mean, stddev)
    _check()
    return _copy_out(pt, ctypes.c_float, n)


def RandomNormalClipped(n, mean, stddev, vmin, vmax, vstep=0):
    pt = _c["NESTGPU_RandomNormalClipped"](n, mean, stddev, vmin, vmax, vstep)
    _check()
    return _copy_out(pt, ctypes.c_float, (n // 4 + 1) * 4)


# ---------------------------------------------------------------- connections
def SingleConnect(i_source_node, i_target_node, i_port, weight, delay):
    return _check(_c["NESTGPU_Connect"](i_source_node, i_target_node, i_port, 0, weight, delay))


def ConnSpecInit():
    return _check(_c["NESTGPU_ConnSpecInit"]())


def SetConnSpecParam(param_name, val):
    return _check(_c["NESTGPU_SetConnSpecParam"](_b(param_name), val))


def ConnSpecIsParam(param_name):
    return _check(_c["NESTGPU_ConnSpecIsParam"](_b(param_name)) != 0)


def SynSpecInit():
    return _check(_c["NESTGPU_SynSpecInit"]())


def SetSynSpecIntParam(param_name, val):
    return _check(_c["NESTGPU_SetSynSpecIntParam"](_b(param_name), val))


def SetSynSpecFloatParam(param_name, val):
    return _check(_c["NESTGPU_SetSynSpecFloatParam"](_b(param_name), val))


def SetSynSpecFloatPtParam(param_name, arr):
    if isinstance(arr, (list, tuple)):
        arr = (ctypes.c_float * len(arr))(*arr)
    return _check(_c["NESTGPU_SetSynSpecFloatPtParam"](_b(param_name), ctypes.cast(arr, c_void_p)))


def SynSpecIsIntParam(param_name):
    return _check(_c["NESTGPU_SynSpecIsIntParam"](_b(param_name)) != 0)


def SynSpecIsFloatParam(param_name):
    return _check(_c["NESTGPU_SynSpecIsFloatParam"](_b(param_name)) != 0)


def SynSpecIsFloatPtParam(param_name):
    return _check(_c["NESTGPU_SynSpecIsFloatPtParam"](_b(param_name)) != 0)


def DictToArray(param_dict, array_size):
    """Array of `array_size` values from {"array": [...]} or a distribution
    ("normal", "normal_clipped" with mu, sigma, low, high, step)."""
    dist_name, arr, low, high, mu, sigma, vstep = None, None, -1.0e35, 1.0e35, None, None, 0
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
    elif dist_name == "normal":
        return RandomNormal(array_size, mu, sigma)
    elif dist_name == "normal_clipped":
        return RandomNormalClipped(array_size, mu, sigma, low, high, vstep)
    raise ValueError("Unknown distribution")


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


def SetSynParamFromArray(param_name, par_dict, array_size):
    arr_param_name = param_name + "_array"
    if not SynSpecIsFloatPtParam(arr_param_name):
        raise ValueError("Synapse parameter cannot be set by arrays or distributions")
    arr = DictToArray(par_dict, array_size)
    SetSynSpecFloatPtParam(arr_param_name, arr)
    return arr


def Connect(source, target, conn_dict, syn_dict):
    "Connect two node groups"
    if not isinstance(source, (list, tuple, NodeSeq)):
        raise ValueError("Unknown source type")
    if not isinstance(target, (list, tuple, NodeSeq)):
        raise ValueError("Unknown target type")
    gc.disable()
    keep = []   # arrays handed to the engine by pointer stay alive during the call
    try:
        ConnSpecInit()
        SynSpecInit()
        for param_name in conn_dict:
            if param_name == "rule":
                if conn_dict[param_name] not in conn_rule_name:
                    raise ValueError("Unknown connection rule")
                SetConnSpecParam(param_name, conn_rule_name.index(conn_dict[param_name]))
            elif ConnSpecIsParam(param_name):
                SetConnSpecParam(param_name, conn_dict[param_name])
            else:
                raise ValueError("Unknown connection parameter")
        array_size = RuleArraySize(conn_dict, source, target)
        for param_name in syn_dict:
            if SynSpecIsIntParam(param_name):
                val = syn_dict[param_name]
                if param_name == "synapse_group" and isinstance(val, SynGroup):
                    val = val.i_syn_group
                SetSynSpecIntParam(param_name, val)
            elif SynSpecIsFloatParam(param_name):
                fpar = syn_dict[param_name]
                if isinstance(fpar, dict):
                    keep.append(SetSynParamFromArray(param_name, fpar, array_size))
                else:
                    SetSynSpecFloatParam(param_name, fpar)
            elif SynSpecIsFloatPtParam(param_name):
                arr = syn_dict[param_name]
                if isinstance(arr, (list, tuple)):
                    arr = (ctypes.c_float * len(arr))(*arr)
                keep.append(arr)
                SetSynSpecFloatPtParam(param_name, arr)
            else:
                raise ValueError("Unknown synapse parameter")
        if isinstance(source, NodeSeq) and isinstance(target, NodeSeq):
            ret = _c["NESTGPU_ConnectSeqSeq"](source.i0, source.n, target.i0, target.n)
        else:
            if not isinstance(source, NodeSeq):
                s_arr = (ctypes.c_int * len(source))(*source)
                keep.append(s_arr)
                s_pt = ctypes.cast(s_arr, c_void_p)
            if not isinstance(target, NodeSeq):
                t_arr = (ctypes.c_int * len(target))(*target)
                keep.append(t_arr)
                t_pt = ctypes.cast(t_arr, c_void_p)
            if isinstance(source, NodeSeq):
                ret = _c["NESTGPU_ConnectSeqGroup"](source.i0, source.n, t_pt, len(target))
            elif isinstance(target, NodeSeq):
                ret = _c["NESTGPU_ConnectGroupSeq"](s_pt, len(source), target.i0, target.n)
            else:
                ret = _c["NESTGPU_ConnectGroupGroup"](s_pt, len(source), t_pt, len(target))
        return _check(ret)
    finally:
        gc.enable()


def RemoteConnect(i_source_host, source, i_target_host, target, conn_dict, syn_dict):
    raise ValueError("MPI is not available (single-GPU engine)")


def GetConnections(source=None, target=None, syn_group=-1):
    "Get connections between two node groups"
    if source is None:
        source = NodeSeq(None)
    if target is None:
        target = NodeSeq(None)
    if isinstance(source, int):
        source = [source]
    if isinstance(target, int):
        target = [target]
    if not isinstance(source, (list, tuple, NodeSeq)):
        raise ValueError("Unknown source type")
    if not isinstance(target, (list, tuple, NodeSeq)):
        raise ValueError("Unknown target type")
    n_conn = ctypes.c_int(0)
    if isinstance(source, NodeSeq) and isinstance(target, NodeSeq):
        arr = _c["NESTGPU_GetSeqSeqConnections"](source.i0, source.n, target.i0, target.n, syn_group,
                                                  ctypes.byref(n_conn))
    else:
        if not isinstance(source, NodeSeq):
            s_arr = (ctypes.c_int * len(source))(*source)
            s_pt = ctypes.cast(s_arr, c_void_p)
        if not isinstance(target, NodeSeq):
            t_arr = (ctypes.c_int * len(target))(*target)
            t_pt = ctypes.cast(t_arr, c_void_p)
        if isinstance(source, NodeSeq):
            arr = _c["NESTGPU_GetSeqGroupConnections"](source.i0, source.n, t_pt, len(target),
                                                        syn_group, ctypes.byref(n_conn))
        elif isinstance(target, NodeSeq):
            arr = _c["NESTGPU_GetGroupSeqConnections"](s_pt, len(source), target.i0, target.n,
                                                        syn_group, ctypes.byref(n_conn))
        else:
            arr = _c["NESTGPU_GetGroupGroupConnections"](s_pt, len(source), t_pt, len(target),
                                                          syn_group, ctypes.byref(n_conn))
    _check()
    out = [ConnectionId(arr[3 * i], arr[3 * i + 1], arr[3 * i + 2]) for i in range(n_conn.value)]
    _free(arr)
    return out


def GetConnectionStatus(conn_id):
    i_target = ctypes.c_int(0)
    i_port = ctypes.c_char()
    i_syn = ctypes.c_char()
    delay = ctypes.c_float(0.0)
    weight = ctypes.c_float(0.0)
    _c["NESTGPU_GetConnectionStatus"](conn_id.i_source, conn_id.i_group, conn_id.i_conn,
                                      ctypes.byref(i_target), ctypes.byref(i_port), ctypes.byref(i_syn),
                                      ctypes.byref(delay), ctypes.byref(weight))
    _check()
    return {"source": conn_id.i_source, "target": i_target.value, "port": ord(i_port.value),
            "syn": ord(i_syn.value), "delay": delay.value, "weight": weight.value}


def SetStatus(gen_object, params, val=None):
    "Set neuron group parameters or variables using dictionaries"
    if isinstance(gen_object, RemoteNodeSeq):
        if gen_object.i_host == MpiId():
            SetStatus(gen_object.node_seq, params, val)
        return
    if isinstance(gen_object, SynGroup):
        if val is not None:
            return SetSynGroupParam(gen_object, params, val)
        if not isinstance(params, dict):
            raise ValueError("Wrong argument in SetStatus")
        for k, v in params.items():
            SetSynGroupParam(gen_object, k, v)
        return None
    gc.disable()
    try:
        nodes = gen_object
        if val is not None:
            SetNeuronStatus(nodes, params, val)
        elif isinstance(params, dict):
            for param_name in params:
                SetNeuronStatus(nodes, param_name, params[param_name])
        elif isinstance(params, (list, tuple)):
            if len(params) != len(nodes):
                raise ValueError("List should have the same size as nodes")
            for param_dict in params:
                if not isinstance(param_dict, dict):
                    raise ValueError("Type of list elements should be dict")
                for param_name in param_dict:
                    SetNeuronStatus(nodes, param_name, param_dict[param_name])
        else:
            raise ValueError("Wrong argument in SetStatus")
        _check()
    finally:
        gc.enable()


def GetStatus(gen_object, var_key=None):
    "Get neuron group or connection status"
    if isinstance(gen_object, SynGroup):
        if var_key is None:
            return {k: GetSynGroupParam(gen_object, k) for k in GetSynGroupParamNames(gen_object)}
        if isinstance(var_key, (list, tuple)):
            return [GetSynGroupParam(gen_object, k) for k in var_key]
        return GetSynGroupParam(gen_object, var_key)
    if isinstance(gen_object, NodeSeq):
        if isinstance(var_key, str):
            return GetNeuronStatus(gen_object, var_key)
        gen_object = gen_object.ToList()
    if isinstance(gen_object, (list, tuple)):
        if isinstance(var_key, str) and len(gen_object) and isinstance(gen_object[0], int):
            return GetNeuronStatus(list(gen_object), var_key)
        return [GetStatus(elem, var_key) for elem in gen_object]
    if isinstance(var_key, (list, tuple)):
        return [GetStatus(gen_object, v) for v in var_key]
    if var_key is None:
        if isinstance(gen_object, ConnectionId):
            return GetConnectionStatus(gen_object)
        if isinstance(gen_object, int):
            i_node = gen_object
            names = (GetIntVarNames(i_node) + GetScalVarNames(i_node) + GetScalParamNames(i_node) +
                     GetPortVarNames(i_node) + GetPortParamNames(i_node) + GetArrayVarNames(i_node) +
                     GetArrayParamNames(i_node) + GetGroupParamNames(i_node))
            return {name: GetStatus(i_node, name) for name in names}
        raise ValueError("Unknown object type in GetStatus")
    if isinstance(var_key, (str, bytes)):
        if isinstance(gen_object, ConnectionId):
            return GetConnectionStatus(gen_object)[var_key]
        if isinstance(gen_object, int):
            return GetNeuronStatus([gen_object], var_key)[0]
        raise ValueError("Unknown object type in GetStatus")
    raise ValueError("Unknown key type in GetStatus", type(var_key))


def CreateSynGroup(model_name, status_dict=None):
    "Create a synapse group (models: stdp, test_syn_model)"
    if status_dict is not None and not isinstance(status_dict, dict):
        raise ValueError("Wrong argument in CreateSynGroup")
    syn_group = SynGroup(_check(_c["NESTGPU_CreateSynGroup"](_b(model_name))))
    if status_dict:
        SetStatus(syn_group, status_dict)
    return syn_group


def _syn_index(syn_group):
    if not isinstance(syn_group, SynGroup):
        raise ValueError("Wrong argument type: a synapse group is expected")
    return syn_group.i_syn_group


def GetSynGroupNParam(syn_group):
    return _check(_c["NESTGPU_GetSynGroupNParam"](_syn_index(syn_group)))


def GetSynGroupParamNames(syn_group):
    n = GetSynGroupNParam(syn_group)
    pp = _c["NESTGPU_GetSynGroupParamNames"](_syn_index(syn_group))
    _check()
    return [pp[i].decode("utf-8") for i in range(n)]


def IsSynGroupParam(syn_group, param_name):
    return _check(_c["NESTGPU_IsSynGroupParam"](_syn_index(syn_group), _b(param_name))) != 0


def GetSynGroupParamIdx(syn_group, param_name):
    return _check(_c["NESTGPU_GetSynGroupParamIdx"](_syn_index(syn_group), _b(param_name)))


def GetSynGroupParam(syn_group, param_name):
    v = _c["NESTGPU_GetSynGroupParam"](_syn_index(syn_group), _b(param_name))
    _check()
    return v


def SetSynGroupParam(syn_group, param_name, val):
    return _check(_c["NESTGPU_SetSynGroupParam"](_syn_index(syn_group), _b(param_name), float(val)))


# ---------------------------------------------------------------- spike recording
def _seq_args(nodes):
    if isinstance(nodes, NodeSeq):
        return nodes.i0, nodes.n
    nodes = list(nodes)
    if nodes != list(range(nodes[0], nodes[0] + len(nodes))):
        raise ValueError("Only node sequences are allowed here")
    return nodes[0], len(nodes)


def ActivateSpikeCount(nodes):
    i0, n = _seq_args(nodes)
    return _check(_c["NESTGPU_ActivateSpikeCount"](i0, n))


def ActivateRecSpikeTimes(nodes, max_n_rec_spike_times):
    i0, n = _seq_args(nodes)
    return _check(_c["NESTGPU_ActivateRecSpikeTimes"](i0, n, max_n_rec_spike_times))


def SetRecSpikeTimesStep(nodes, rec_spike_times_step):
    i0, n = _seq_args(nodes)
    return _check(_c["NESTGPU_SetRecSpikeTimesStep"](i0, n, rec_spike_times_step))


def GetNRecSpikeTimes(i_node):
    return _check(_c["NESTGPU_GetNRecSpikeTimes"](i_node))


def GetRecSpikeTimes(nodes):
    i0, n = _seq_args(nodes)
    n_pt = ctypes.POINTER(ctypes.c_int)()
    t_pt = ctypes.POINTER(ctypes.POINTER(ctypes.c_float))()
    _c["NESTGPU_GetRecSpikeTimes"](i0, n, ctypes.byref(n_pt), ctypes.byref(t_pt))
    _check()
    return [[t_pt[i][j] for j in range(n_pt[i])] for i in range(n)]


# ---------------------------------------------------------------- kernel parameters
def GetNBoolParam():
    return _c["NESTGPU_GetNBoolParam"]()


def GetBoolParamNames():
    pp = _c["NESTGPU_GetBoolParamNames"]()
    return [pp[i].decode() for i in range(GetNBoolParam())]


def IsBoolParam(param_name):
    return _c["NESTGPU_IsBoolParam"](_b(param_name)) != 0


def GetBoolParam(param_name):
    return _check(_c["NESTGPU_GetBoolParam"](_b(param_name)))


def SetBoolParam(param_name, val):
    return _check(_c["NESTGPU_SetBoolParam"](_b(param_name), val))


def GetNFloatParam():
    return _c["NESTGPU_GetNFloatParam"]()


def GetFloatParamNames():
    pp = _c["NESTGPU_GetFloatParamNames"]()
    return [pp[i].decode() for i in range(GetNFloatParam())]


def IsFloatParam(param_name):
    return _c["NESTGPU_IsFloatParam"](_b(param_name)) != 0


def GetFloatParam(param_name):
    return _check(_c["NESTGPU_GetFloatParam"](_b(param_name)))


def SetFloatParam(param_name, val):
    return _check(_c["NESTGPU_SetFloatParam"](_b(param_name), val))


def GetNIntParam():
    return _c["NESTGPU_GetNIntParam"]()


def GetIntParamNames():
    pp = _c["NESTGPU_GetIntParamNames"]()
    return [pp[i].decode() for i in range(GetNIntParam())]


def IsIntParam(param_name):
    return _c["NESTGPU_IsIntParam"](_b(param_name)) != 0


def GetIntParam(param_name):
    return _check(_c["NESTGPU_GetIntParam"](_b(param_name)))


def SetIntParam(param_name, val):
    return _check(_c["NESTGPU_SetIntParam"](_b(param_name), val))


def GetKernelStatus(var_key=None):
    if isinstance(var_key, (list, tuple)):
        return [GetKernelStatus(v) for v in var_key]
    if var_key is None:
        d = {}
        for n in GetFloatParamNames():
            d[n] = GetFloatParam(n)
        for n in GetIntParamNames():
            d[n] = GetIntParam(n)
        for n in GetBoolParamNames():
            d[n] = GetBoolParam(n)
        return d
    if IsFloatParam(var_key):
        return GetFloatParam(var_key)
    if IsIntParam(var_key):
        return GetIntParam(var_key)
    if IsBoolParam(var_key):
        return GetBoolParam(var_key)
    raise ValueError("Unknown parameter in GetKernelStatus", var_key)


def SetKernelStatus(params, val=None):
    if isinstance(params, str) and val is not None:
        params = {params: val}
    if not isinstance(params, dict):
        raise ValueError("Wrong argument in SetKernelStatus")
    for k, v in params.items():
        if IsFloatParam(k):
            SetFloatParam(k, v)
        elif IsIntParam(k):
            SetIntParam(k, v)
        elif IsBoolParam(k):
            SetBoolParam(k, v)
        else:
            raise ValueError("Unknown parameter in SetKernelStatus", k)


def RemoteCreate(i_host, model_name, n_node=1, n_ports=1, status_dict=None):
    raise ValueError("MPI is not available (single-GPU engine)")


# ---------------------------------------------------------------- engine extensions
def Reset():
    """Discard the current network and start an empty one (engine extension)."""
    if not is_b200_engine:
        raise ValueError("Reset needs libnestgpu_b200.so")
    return _check(_c["NGPU_Reset"]())


def GetStats():
    """Engine counters: RK5 derivative evaluations, synaptic events, spikes, wall time of
    the last Simulate loop [s], steps, device status bits (engine extension)."""
    if not is_b200_engine:
        raise ValueError("GetStats needs libnestgpu_b200.so")
    a, b, c = ctypes.c_ulonglong(), ctypes.c_ulonglong(), ctypes.c_ulonglong()
    s, st, stat = ctypes.c_double(), ctypes.c_longlong(), ctypes.c_uint()
    _c["NGPU_GetStats"](ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), ctypes.byref(s),
                        ctypes.byref(st), ctypes.byref(stat))
    _check()
    return {"n_derivs": a.value, "n_events": b.value, "n_spikes": c.value, "sim_seconds": s.value,
            "steps": st.value, "status": stat.value}


def ConnectArrays(source, target, weight, delay, port=None):
    """Bulk connect edge lists (numpy arrays or sequences, one entry per edge)."""
    import numpy as np
    if not is_b200_engine:
        raise ValueError("ConnectArrays needs libnestgpu_b200.so")
    s = np.ascontiguousarray(source, dtype=np.int32)
    t = np.ascontiguousarray(target, dtype=np.int32)
    w = np.ascontiguousarray(weight, dtype=np.float32)
    d = np.ascontiguousarray(delay, dtype=np.float32)
    p = np.ascontiguousarray(port, dtype=np.uint8) if port is not None else None
    n = s.size
    if not (t.size == n and w.size == n and d.size == n and (p is None or p.size == n)):
        raise ValueError("edge arrays must have the same length")
    return _check(_c["NGPU_ConnectArrays"](n, s.ctypes.data, t.ctypes.data,
                                           p.ctypes.data if p is not None else None,
                                           w.ctypes.data, d.ctypes.data))


def GetSimDeviceMs():
    """Device time [ms] of the last Simulate call, from CUDA events on the engine stream."""
    return _check(_c["NGPU_GetSimDeviceMs"]())


def GetLaunchCount():
    """Engine kernels launched so far (graph replays count every kernel node)."""
    return _check(_c["NGPU_GetLaunchCount"]())


def ProfileSteps(n):
    """Run n simulation steps with per-kernel CUDA events; average ms per step of
    (neuron updates, record gather, spike delivery)."""
    out = (ctypes.c_double * 3)()
    _c["NGPU_ProfileSteps"](n, out)
    _check()
    return list(out)


def ConnectFixedIndegreeGPU(source, target, indegree, weight, delay_min, delay_max, receptor=0,
                            seed=1):
    """Per-target fixed in-degree block generated on the GPU (engine extension)."""
    return _check(_c["NGPU_ConnectFixedIndegreeGPU"](source.i0, source.n, target.i0, target.n, indegree,
                                                     receptor, weight, delay_min, delay_max, seed))


def SetPoissonStream(nodes, stream):
    """poisson_generator nodes draw from streams stream, stream+1, ... (engine extension,
    before calibration): a generator's draws then depend only on (kernel seed, stream,
    out-edge index, time step), not on where it sits in the network."""
    _need_b200("SetPoissonStream")
    if not isinstance(nodes, NodeSeq):
        nodes = NodeSeq(nodes[0], len(nodes)) if len(nodes) else NodeSeq(0, 0)
    return _check(_c["NGPU_SetPoissonStream"](nodes.i0, nodes.n, int(stream) & 0xffffffff))


def SetDeviceRuleMinEdges(n):
    """Connect calls with the fixed_total_number / fixed_indegree / fixed_outdegree rule and
    at least n edges are expanded on the device at calibration (engine extension)."""
    _need_b200("SetDeviceRuleMinEdges")
    return _check(_c["NGPU_SetDeviceRuleMinEdges"](int(n)))


def GetDeliveryCsr():
    """The recurrent delivery layout after calibration (engine extension): a dict with
    n_nodes, dmin, dspan, seg_off (int64, n_nodes*dspan+1: segment (source s, delay step
    dmin+d) is seg_off[s*dspan+d] .. seg_off[s*dspan+d+1]) and per edge target, port,
    weight (order inside a segment unspecified)."""
    import numpy as np
    _need_b200("GetDeliveryCsr")
    nn, dmin, dspan, ne = _I(), _I(), _I(), ctypes.c_longlong()
    _c["NGPU_GetDeliveryShape"](ctypes.byref(nn), ctypes.byref(dmin), ctypes.byref(dspan), ctypes.byref(ne))
    _check()
    off = np.zeros(nn.value * dspan.value + 1, dtype=np.int64)
    tgt = np.zeros(max(ne.value, 1), dtype=np.int32)
    port = np.zeros(max(ne.value, 1), dtype=np.uint8)
    w = np.zeros(max(ne.value, 1), dtype=np.float32)
    _c["NGPU_GetDeliveryCsr"](off.ctypes.data, tgt.ctypes.data, port.ctypes.data, w.ctypes.data)
    _check()
    return {"n_nodes": nn.value, "dmin": dmin.value, "dspan": dspan.value, "seg_off": off,
            "target": tgt[:ne.value], "port": port[:ne.value], "weight": w[:ne.value]}


def SetHostRng(on=True):
    """Use cuRAND's host generator for connection random numbers (engine extension)."""
    if not is_b200_engine:
        raise ValueError("SetHostRng needs libnestgpu_b200.so")
    return _check(_c["NGPU_SetHostRng"](1 if on else 0))


def SetDeliverBlocks(n):
    """Thread blocks of the delivery kernel (engine extension; 0 = automatic)."""
    return _check(_c["NGPU_SetDeliverBlocks"](n))


def SetBatchMax(n):
    """Upper bound of time steps integrated per batch (engine extension; before calibration)."""
    return _check(_c["NGPU_SetBatchMax"](n))


def SetRk5Budget(n):
    """RK5 steps per neuron in the main update kernel before the straggler kernel takes over
    (engine extension; 0 disables the hand-off)."""
    return _check(_c["NGPU_SetRk5Budget"](n))


def SetUpdateThreads(n):
    """Threads per block of the aeif update kernel: 64, 128 or 256 (engine extension)."""
    _need_b200("SetUpdateThreads")
    return _check(_c["NGPU_SetUpdateThreads"](n))


def SetPersistent(on=True):
    """iaf_psc_exp-only networks: run the steps in one cooperative launch per graph's worth
    of steps, or in per-batch launches captured in CUDA graphs (the default; engine
    extension)."""
    _need_b200("SetPersistent")
    return _check(_c["NGPU_SetPersistent"](1 if on else 0))


def GetBatchLength():
    """Steps per time batch (kernel launch) of the calibrated network (engine extension)."""
    _need_b200("GetBatchLength")
    n = _c["NGPU_GetBatchLength"]()
    _check()
    return n


def SetUpdateOccupancy(on=True):
    """Register-capped variant of the aeif update kernel (engine extension): 1 (or True) three
    256-thread blocks per SM, 2 five 128-thread blocks (trial-per-iteration update, uniform
    parameters), 0 none."""
    _need_b200("SetUpdateOccupancy")
    v = int(on) if not isinstance(on, bool) else (1 if on else 0)
    return _check(_c["NGPU_SetUpdateOccupancy"](v))


def SetUpdateTrialIter(on=True):
    """aeif update kernel advancing one RK5 trial per loop iteration (engine extension;
    results are identical either way)."""
    _need_b200("SetUpdateTrialIter")
    return _check(_c["NGPU_SetUpdateTrialIter"](1 if on else 0))


def SetDeliverPrefetch(on=True):
    """Delivery loads the next work item's spike and segment offsets ahead (engine extension;
    results are identical either way)."""
    _need_b200("SetDeliverPrefetch")
    return _check(_c["NGPU_SetDeliverPrefetch"](1 if on else 0))


def SetDeliverPush(on=True):
    """Delivery at emission for networks of iaf_psc_exp groups (engine extension, default off):
    each spike's out-edges are added by the update kernel in the step it is emitted, with no
    delivery kernel; takes effect at calibration (call before the first Simulate); results
    are identical either way."""
    _need_b200("SetDeliverPush")
    return _check(_c["NGPU_SetDeliverPush"](1 if on else 0))


def DeliverPushActive():
    """True if delivery at emission is active (engine extension; after calibration)."""
    _need_b200("DeliverPushActive")
    return bool(_check(_c["NGPU_DeliverPushActive"]()))


def SetDeliverAggregate(on=True):
    """Warp-aggregated reductions in the delivery kernel with 32-lane work items (engine
    extension; results are identical either way)."""
    _need_b200("SetDeliverAggregate")
    return _check(_c["NGPU_SetDeliverAggregate"](1 if on else 0))


def SetPartition(rank, world):
    """This process simulates share `rank` of `world` of every node group (engine extension,
    before calibration); see partition.py for the spike exchange."""
    _need_b200("SetPartition")
    return _check(_c["NGPU_SetPartition"](int(rank), int(world)))


EXCHANGE_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p)


def SetExchange(send_ptr, recv_ptr, cap, fn):
    """Exchange buffers (device pointers to (cap + 1) int4 records per process) and the
    all-gather function called after every time batch (an EXCHANGE_FN; keep a reference to
    it while the engine runs)."""
    _need_b200("SetExchange")
    return _check(_c["NGPU_SetExchange"](send_ptr, recv_ptr, int(cap), ctypes.cast(fn, c_void_p), None))


def SetDeliverGroup(g):
    """Lanes per spike-delivery work item: 8, 16 or 32 (engine extension)."""
    _need_b200("SetDeliverGroup")
    return _check(_c["NGPU_SetDeliverGroup"](g))


def SetProgrammaticLaunch(on=True):
    """Programmatic dependent launch of the kernels of a time batch (engine extension;
    results are the same either way): True, False, or None for the default (batches of one
    time step only)."""
    _need_b200("SetProgrammaticLaunch")
    return _check(_c["NGPU_SetProgrammaticLaunch"](-1 if on is None else (1 if on else 0)))


def Autotune(steps=200):
    """Pick the update block size, delivery lane group, delivery grid and RK5 step budget
    by timing `steps` simulation steps per candidate on the calibrated network (the network
    advances by those steps).  Returns the chosen settings and the number of trials."""
    _need_b200("Autotune")
    a, b, c, d = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    n = _c["NGPU_Autotune"](steps, ctypes.byref(a), ctypes.byref(b), ctypes.byref(c), ctypes.byref(d))
    _check()
    m = GetLaunchMapping()
    m["trials"] = n
    return m


def MeasureReductionRate(nbytes, n_ops):
    """1e9 FP64 reductions per second to random addresses of an `nbytes` device buffer (the
    delivery kernel's access pattern; engine extension)."""
    _need_b200("MeasureReductionRate")
    v = _c["NGPU_MeasureReductionRate"](nbytes, n_ops)
    _check()
    return v


def GetLaunchMapping():
    """The current launch mapping (engine extension): update block size and variant, delivery
    lane group and grid, RK5 step budget, persistent loop and programmatic launch."""
    _need_b200("GetLaunchMapping")
    v = (ctypes.c_int * 10)()
    _c["NGPU_GetLaunchMapping"](v, 10)
    _check()
    keys = ["update_threads", "update_occupancy", "deliver_group", "deliver_blocks", "rk5_budget",
            "persistent", "programmatic_launch", "update_trial_iter", "deliver_aggregate", "deliver_prefetch"]
    return dict(zip(keys, [int(x) for x in v]))


def SetGraphSteps(n):
    if not is_b200_engine:
        raise ValueError("SetGraphSteps needs libnestgpu_b200.so")
    return _check(_c["NGPU_SetGraphSteps"](n))


# ---- learned RK5 step-size proposal (engine extension, no reference counterpart)
def _need_b200(name):
    if not is_b200_engine:
        raise ValueError(name + " needs libnestgpu_b200.so")


def Rk5LogStart(capacity):
    """Log one tuple (10 step features, accepted h, error) per accepted RK5 step of every
    aeif neuron during the following Simulate calls, at most `capacity` tuples."""
    _need_b200("Rk5LogStart")
    return _check(_c["NGPU_Rk5LogStart"](int(capacity)))


def Rk5LogStop():
    _need_b200("Rk5LogStop")
    return _check(_c["NGPU_Rk5LogStop"]())


def Rk5LogCount():
    """(tuples stored, tuples offered) of the RK5 log."""
    _need_b200("Rk5LogCount")
    off = ctypes.c_longlong(0)
    n = _c["NGPU_Rk5LogCount"](ctypes.byref(off))
    _check()
    return n, off.value


def Rk5LogGet(first=0, n=None):
    """Logged tuples [n, 12] as a float32 array."""
    import numpy as np
    _need_b200("Rk5LogGet")
    if n is None:
        n = Rk5LogCount()[0] - first
    out = np.zeros((n, 12), dtype=np.float32)
    _c["NGPU_Rk5LogGet"](out.ctypes.data, first, n)
    _check()
    return out


def StepModelTrain(iters=3000, batch=4096, lr=2.0e-3, safety=0.9, floor=0.0, seed=1):
    """Train the step-size network on the logged tuples with the GPU kernels and make it
    the engine's model; returns (tuples used, final mean squared error).  In the RK5 loop
    the proposal is safety * (predicted step size), raised to at least floor * (the
    controller's h) when floor > 0."""
    _need_b200("StepModelTrain")
    nu, loss = ctypes.c_longlong(0), ctypes.c_float(0)
    _c["NGPU_StepModelTrain"](int(iters), int(batch), float(lr), float(safety), float(floor), int(seed),
                              ctypes.byref(nu), ctypes.byref(loss))
    _check()
    return nu.value, loss.value


def StepModelGet():
    import numpy as np
    _need_b200("StepModelGet")
    p = np.zeros(_c["NGPU_StepModelNParams"](), dtype=np.float32)
    _c["NGPU_StepModelGet"](p.ctypes.data)
    _check()
    return p


def StepModelSet(params):
    import numpy as np
    _need_b200("StepModelSet")
    p = np.ascontiguousarray(params, dtype=np.float32)
    if p.size != _c["NGPU_StepModelNParams"]():
        raise ValueError("step model parameter vector has the wrong size")
    return _check(_c["NGPU_StepModelSet"](p.ctypes.data))


def StepBoundMode(on=True):
    """Analysis mode: every RK5 step starts from the largest step that passes the error test,
    so the evaluation counter shows the floor for any step-size proposal (engine extension)."""
    _need_b200("StepBoundMode")
    return _check(_c["NGPU_StepBoundMode"](1 if on else 0))


def StepModelEnable(on=True):
    """Let the network propose the first trial h of RK5 steps (the error test, the
    rejection shrink and the plain controller stay as they are)."""
    _need_b200("StepModelEnable")
    return _check(_c["NGPU_StepModelEnable"](1 if on else 0))


def MlpForward(params, feat):
    """Network output for features [n, 10] computed by the GPU inference code."""
    import numpy as np
    _need_b200("MlpForward")
    p = np.ascontiguousarray(params, dtype=np.float32)
    f = np.ascontiguousarray(feat, dtype=np.float32).reshape(-1, 10)
    out = np.zeros(f.shape[0], dtype=np.float32)
    _c["NGPU_MlpForward"](p.ctypes.data, f.ctypes.data, f.shape[0], out.ctypes.data)
    _check()
    return out


def MlpGrad(params, feat, target):
    """(loss, gradient of the trainable block) computed by the GPU training kernels."""
    import numpy as np
    _need_b200("MlpGrad")
    p = np.ascontiguousarray(params, dtype=np.float32)
    f = np.ascontiguousarray(feat, dtype=np.float32).reshape(-1, 10)
    t = np.ascontiguousarray(target, dtype=np.float32)
    g = np.zeros(1441, dtype=np.float32)
    loss = ctypes.c_float(0)
    _c["NGPU_MlpGrad"](p.ctypes.data, f.ctypes.data, t.ctypes.data, f.shape[0], g.ctypes.data, ctypes.byref(loss))
    _check()
    return loss.value, g
