"""CPU oracle of the NEST GPU hot path, with a nestgpu-like Python surface.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the engine.  The C++ restatement lives in
oracle/ngpu_oracle.cpp (built into oracle/lib/liboracle.so by oracle/Makefile).

The class `Oracle` mirrors the calling conventions of the reference's
pythonlib/nestgpu.py (Create, SetStatus, GetStatus, Connect, CreateRecord,
GetRecordData, Simulate, ActivateSpikeCount, ActivateRecSpikeTimes,
GetRecSpikeTimes, GetConnections) so that a scenario can be played against the
oracle and against the CUDA engine with the same code.
"""
import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "lib", "liboracle.so")
_lib = None

CONN_RULES = ["one_to_one", "all_to_all", "fixed_total_number", "fixed_indegree",
              "fixed_outdegree"]


def build():
    """Compile the oracle library with its Makefile (gcc, no GPU needed)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = ctypes.CDLL(_LIB_PATH)
        c_int, c_float, c_void, c_ull = ctypes.c_int, ctypes.c_float, ctypes.c_void_p, ctypes.c_ulonglong
        fp = ctypes.POINTER(ctypes.c_float)
        ip = ctypes.POINTER(ctypes.c_int)
        sigs = {
            "orc_error": (ctypes.c_char_p, []),
            "orc_new": (c_void, [c_int]),
            "orc_delete": (None, [c_void]),
            "orc_set_time_resolution": (c_int, [c_void, c_float]),
            "orc_get_time_resolution": (c_float, [c_void]),
            "orc_set_seed": (c_int, [c_void, c_ull]),
            "orc_set_max_spike_buffer_size": (c_int, [c_void, c_int]),
            "orc_create": (c_int, [c_void, ctypes.c_char_p, c_int, c_int]),
            "orc_n_nodes": (c_int, [c_void]),
            "orc_node_model": (c_int, [c_void, c_int]),
            "orc_node_nport": (c_int, [c_void, c_int]),
            "orc_locate": (c_int, [c_void, c_int, ctypes.c_char_p]),
            "orc_set": (c_int, [c_void, c_int, c_int, ctypes.c_char_p, c_int, fp, c_int]),
            "orc_set_list": (c_int, [c_void, ip, c_int, ctypes.c_char_p, c_int, fp, c_int]),
            "orc_get": (c_int, [c_void, c_int, c_int, ctypes.c_char_p, c_int, fp]),
            "orc_set_spike_times": (c_int, [c_void, c_int, c_int, fp, fp]),
            "orc_random_int": (c_int, [c_void, ctypes.c_size_t, ctypes.POINTER(ctypes.c_uint)]),
            "orc_random_uniform": (c_int, [c_void, ctypes.c_size_t, fp]),
            "orc_random_normal": (c_int, [c_void, ctypes.c_size_t, c_float, c_float, fp]),
            "orc_random_normal_clipped": (c_int, [c_void, ctypes.c_size_t, c_float, c_float, c_float,
                                                  c_float, c_float, fp]),
            "orc_connect": (c_int, [c_void, c_int, ip, c_int, c_int, ip, c_int, c_int, c_int, c_int,
                                    c_int, c_float, c_float, fp, fp]),
            "orc_create_syn_group": (c_int, [c_void, ctypes.c_char_p]),
            "orc_set_syn_param": (c_int, [c_void, c_int, ctypes.c_char_p, c_float]),
            "orc_get_syn_param": (c_int, [c_void, c_int, ctypes.c_char_p, fp]),
            "orc_connect1": (c_int, [c_void, c_int, c_int, c_int, c_float, c_float]),
            "orc_n_conn": (ctypes.c_longlong, [c_void]),
            "orc_connect_arrays": (c_int, [c_void, ctypes.c_size_t, ip, ip, ip, fp, fp]),
            "orc_connect_generated": (c_int, [c_void, c_int, c_int, c_int, c_int, c_int, c_int, c_float,
                                              c_float, c_float, c_ull]),
            "orc_set_poisson_stream": (c_int, [c_void, c_int, c_int, ctypes.c_uint]),
            "orc_set_partition": (c_int, [c_void, c_int, c_int]),
            "orc_set_exchange": (c_int, [c_void, c_void, c_void]),
            "orc_step_spikes": (c_int, [c_void, ip, fp]),
            "orc_inject_spikes": (c_int, [c_void, ip, fp, c_int]),
            "orc_threads": (c_int, []),
            "orc_get_conns": (c_int, [c_void, ip, ip, ip, ip, ip, ip, fp, fp]),
            "orc_record": (c_int, [c_void, c_int, ctypes.c_char_p, c_int]),
            "orc_record_rows": (c_int, [c_void]),
            "orc_record_data": (c_int, [c_void, fp]),
            "orc_activate_spike_count": (c_int, [c_void, c_int, c_int]),
            "orc_activate_rec_spike_times": (c_int, [c_void, c_int, c_int, c_int]),
            "orc_get_spike_count": (c_int, [c_void, c_int, c_int, ip]),
            "orc_n_rec_spike_times": (c_int, [c_void, c_int]),
            "orc_rec_spike_times": (c_int, [c_void, c_int, fp]),
            "orc_calibrate": (c_int, [c_void]),
            "orc_simulate": (c_int, [c_void, c_float]),
            "orc_n_derivs": (ctypes.c_longlong, [c_void]),
            "orc_n_rk5_steps": (ctypes.c_longlong, [c_void]),
            "orc_n_rk5_trials": (ctypes.c_longlong, [c_void]),
            "orc_n_spikes": (ctypes.c_longlong, [c_void]),
            "orc_n_events": (ctypes.c_longlong, [c_void]),
            "orc_neural_time": (ctypes.c_double, [c_void]),
            "orc_exp_m": (c_float, [c_float]),
            "orc_log_m": (c_float, [c_float]),
            "orc_poisson_draw": (c_int, [c_float, c_ull, c_ull, ctypes.c_longlong]),
            "orc_philox": (None, [ctypes.c_uint] * 6 + [ctypes.POINTER(ctypes.c_uint)]),
            "orc_step_model_nparams": (c_int, []),
            "orc_log_start": (c_int, [c_void, ctypes.c_longlong]),
            "orc_log_stop": (c_int, [c_void]),
            "orc_set_bound_mode": (c_int, [c_void, c_int]),
            "orc_log_count": (ctypes.c_longlong, [c_void, ctypes.POINTER(ctypes.c_longlong)]),
            "orc_log_get": (c_int, [c_void, fp]),
            "orc_step_model_set": (c_int, [c_void, fp, c_int]),
            "orc_mlp_out": (None, [fp, fp, c_int, fp]),
            "orc_mlp_propose": (None, [fp, fp, c_int, fp]),
            "orc_mlp_grad": (ctypes.c_double, [fp, fp, fp, c_int, ctypes.POINTER(ctypes.c_double)]),
            "orc_mlp_grad_bf16": (ctypes.c_double, [fp, fp, fp, c_int, ctypes.POINTER(ctypes.c_double)]),
        }
        for name, (res, args) in sigs.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def _fptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))


def _iptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int))


class NodeSeq(object):
    """Contiguous node range (i0, n), indexable like the reference's NodeSeq."""

    def __init__(self, i0, n=1):
        self.i0 = i0
        self.n = n

    def __len__(self):
        return self.n

    def __getitem__(self, i):
        if isinstance(i, slice):
            start, stop, step = i.indices(self.n)
            if step != 1:
                raise ValueError("NodeSeq slices must be contiguous")
            return NodeSeq(self.i0 + start, max(stop - start, 0))
        if i < 0:
            i += self.n
        if i < 0 or i >= self.n:
            raise IndexError("node index out of range")
        return self.i0 + i

    def ToList(self):
        return list(range(self.i0, self.i0 + self.n))


def _nodes(x):
    if isinstance(x, int):
        return [x]
    if hasattr(x, "i0") and hasattr(x, "n"):
        return list(range(x.i0, x.i0 + x.n))
    return list(x)


class Oracle(object):
    """One simulated network.  fp64=False mirrors the FP32 CUDA arithmetic bit for
    bit; fp64=True integrates in double with the reference's formulas."""

    def __init__(self, fp64=False):
        self.L = lib()
        self.h = self.L.orc_new(1 if fp64 else 0)
        if not self.h:
            raise RuntimeError(self.L.orc_error().decode())
        self.n_rec = 0

    def __del__(self):
        try:
            if self.h:
                self.L.orc_delete(self.h)
        except Exception:
            pass

    def _chk(self, r):
        if r < 0:
            raise ValueError(self.L.orc_error().decode())
        return r

    # -- kernel settings
    def SetRandomSeed(self, seed):
        self._chk(self.L.orc_set_seed(self.h, seed))

    def SetTimeResolution(self, dt):
        self.L.orc_set_time_resolution(self.h, dt)

    def GetTimeResolution(self):
        return self.L.orc_get_time_resolution(self.h)

    def SetMaxSpikeBufferSize(self, n):
        self.L.orc_set_max_spike_buffer_size(self.h, n)

    def SetKernelStatus(self, params, val=None):
        if val is not None:
            params = {params: val}
        for k, v in params.items():
            if k == "rnd_seed":
                self.SetRandomSeed(v)
            elif k == "time_resolution":
                self.SetTimeResolution(v)
            elif k == "max_spike_buffer_size":
                self.SetMaxSpikeBufferSize(v)
            else:
                raise ValueError("Unknown kernel parameter " + k)

    # -- random numbers (same generator as the connection rules)
    def RandomInt(self, n):
        out = np.zeros(n, dtype=np.uint32)
        self._chk(self.L.orc_random_int(self.h, n, out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint))))
        return out

    def RandomUniform(self, n):
        out = np.zeros(n, dtype=np.float32)
        self._chk(self.L.orc_random_uniform(self.h, n, _fptr(out)))
        return out

    def RandomNormal(self, n, mean, sd):
        out = np.zeros(n, dtype=np.float32)
        self._chk(self.L.orc_random_normal(self.h, n, mean, sd, _fptr(out)))
        return out

    def RandomNormalClipped(self, n, mean, sd, vmin, vmax, vstep=0.0):
        out = np.zeros((n // 4 + 1) * 4, dtype=np.float32)
        self._chk(self.L.orc_random_normal_clipped(self.h, n, mean, sd, vmin, vmax, vstep, _fptr(out)))
        return out

    def _dict_to_array(self, d, size):
        dist, arr, low, high, mu, sigma, step = None, None, -1.0e35, 1.0e35, None, None, 0.0
        for k, v in d.items():
            if k == "array":
                dist, arr = "array", v
            elif k == "distribution":
                dist = v
            elif k == "low":
                low = v
            elif k == "high":
                high = v
            elif k == "mu":
                mu = v
            elif k == "sigma":
                sigma = v
            elif k == "step":
                step = v
            else:
                raise ValueError("Unknown parameter name in dictionary")
        if dist == "array":
            a = np.ascontiguousarray(arr, dtype=np.float32)
            if a.size != size:
                raise ValueError("Wrong array size.")
            return a
        if dist == "normal":
            return self.RandomNormal(size, mu, sigma)
        if dist == "normal_clipped":
            return self.RandomNormalClipped(size, mu, sigma, low, high, step)
        raise ValueError("Unknown distribution")

    # -- nodes
    def Create(self, model, n_node=1, n_ports=1, status_dict=None):
        i0 = self._chk(self.L.orc_create(self.h, model.encode(), n_node, n_ports))
        ns = NodeSeq(i0, n_node)
        if status_dict is not None:
            self.SetStatus(ns, status_dict)
        return ns

    def _set1(self, nodes, name, val):
        nodes = _nodes(nodes)
        kind = self._chk(self.L.orc_locate(self.h, nodes[0], name.encode()))
        if isinstance(val, dict):
            arr = self._dict_to_array(val, len(nodes))
            for i, nd in enumerate(nodes):
                self._set1([nd], name, float(arr[i]))
            return
        if kind == 5:
            t = np.ascontiguousarray(val, dtype=np.float32)
            for nd in nodes:
                if name == "spike_times":
                    self._chk(self.L.orc_set_spike_times(self.h, nd, t.size, _fptr(t), None))
                else:
                    raise ValueError("spike_heights must be set together with spike_times")
            return
        ni = np.asarray(nodes, dtype=np.int32)
        if kind in (1, 3):     # port quantity: one value per port
            vals = np.atleast_1d(np.asarray(val, dtype=np.float32))
            for p in range(vals.size):
                v = np.array([vals[p]], dtype=np.float32)
                self._chk(self.L.orc_set_list(self.h, _iptr(ni), ni.size, name.encode(), p, _fptr(v), 0))
        else:
            v = np.array([val], dtype=np.float32)
            self._chk(self.L.orc_set_list(self.h, _iptr(ni), ni.size, name.encode(), 0, _fptr(v), 0))

    def SetStatus(self, nodes, params, val=None):
        if isinstance(nodes, SynGroup):
            items = {params: val} if val is not None else params
            for k, v in items.items():
                self._chk(self.L.orc_set_syn_param(self.h, nodes.i_syn_group, k.encode(), float(v)))
            return
        if val is not None:
            self._set1(nodes, params, val)
        elif isinstance(params, dict):
            if "spike_times" in params:
                t = np.ascontiguousarray(params["spike_times"], dtype=np.float32)
                h = params.get("spike_heights")
                hp = None
                if h is not None:
                    h = np.ascontiguousarray(h, dtype=np.float32)
                    hp = _fptr(h)
                for nd in _nodes(nodes):
                    self._chk(self.L.orc_set_spike_times(self.h, nd, t.size, _fptr(t), hp))
                params = {k: v for k, v in params.items() if k not in ("spike_times", "spike_heights")}
            for k, v in params.items():
                self._set1(nodes, k, v)
        else:
            raise ValueError("Wrong argument in SetStatus")

    def GetStatus(self, nodes, var):
        if isinstance(nodes, SynGroup):
            out = np.zeros(1, dtype=np.float32)
            self._chk(self.L.orc_get_syn_param(self.h, nodes.i_syn_group, var.encode(), _fptr(out)))
            return float(out[0])
        nodes = _nodes(nodes)
        out = np.zeros(1, dtype=np.float32)
        res = []
        if var == "spike_count":
            c = np.zeros(1, dtype=np.int32)
            for nd in nodes:
                self._chk(self.L.orc_get_spike_count(self.h, nd, 1, _iptr(c)))
                res.append(int(c[0]))
            return res
        kind = self._chk(self.L.orc_locate(self.h, nodes[0], var.encode()))
        for nd in nodes:
            if kind in (1, 3):
                npt = self.L.orc_node_nport(self.h, nd)
                row = []
                for p in range(npt):
                    self._chk(self.L.orc_get(self.h, nd, 1, var.encode(), p, _fptr(out)))
                    row.append(float(out[0]))
                res.append(row)
            else:
                self._chk(self.L.orc_get(self.h, nd, 1, var.encode(), 0, _fptr(out)))
                res.append(float(out[0]))
        return res

    # -- synapse groups (src/syn_model.cu:136-238)
    def CreateSynGroup(self, model_name, status_dict=None):
        g = SynGroup(self._chk(self.L.orc_create_syn_group(self.h, model_name.encode())))
        if status_dict:
            self.SetStatus(g, status_dict)
        return g

    # -- connections
    def Connect(self, source, target, conn_dict, syn_dict):
        rule = conn_dict["rule"]
        if rule not in CONN_RULES:
            raise ValueError("Unknown connection rule")
        ir = CONN_RULES.index(rule)
        degree = 0
        for k, v in conn_dict.items():
            if k in ("indegree", "outdegree", "total_num"):
                degree = v
            elif k != "rule":
                raise ValueError("Unknown connection parameter")
        src_list = isinstance(source, (list, tuple, np.ndarray))
        tgt_list = isinstance(target, (list, tuple, np.ndarray))
        ns = len(source)
        nt = len(target)
        size = {"one_to_one": ns, "all_to_all": ns * nt, "fixed_total_number": degree,
                "fixed_indegree": nt * degree, "fixed_outdegree": ns * degree}[rule]
        port, syn, w, d, warr, darr = 0, 0, 0.0, 0.0, None, None
        for k, v in syn_dict.items():
            if k == "receptor":
                port = v
            elif k == "synapse_group":
                syn = v.i_syn_group if isinstance(v, SynGroup) else int(v)
            elif k == "weight":
                if isinstance(v, dict):
                    warr = self._dict_to_array(v, size)
                else:
                    w = v
            elif k == "delay":
                if isinstance(v, dict):
                    darr = self._dict_to_array(v, size)
                else:
                    d = v
            elif k == "weight_array":
                warr = np.ascontiguousarray(v, dtype=np.float32)
            elif k == "delay_array":
                darr = np.ascontiguousarray(v, dtype=np.float32)
            else:
                raise ValueError("Unknown synapse parameter")
        sarr = np.ascontiguousarray(source, dtype=np.int32) if src_list else None
        tarr = np.ascontiguousarray(target, dtype=np.int32) if tgt_list else None
        self._chk(self.L.orc_connect(
            self.h, ir, _iptr(sarr) if src_list else None, 0 if src_list else source.i0, ns,
            _iptr(tarr) if tgt_list else None, 0 if tgt_list else target.i0, nt, degree, port, syn, w, d,
            _fptr(warr) if warr is not None else None, _fptr(darr) if darr is not None else None))

    def ConnectArrays(self, source, target, port, weight, delay):
        """Bulk single connections (inserted in array order)."""
        s = np.ascontiguousarray(source, dtype=np.int32)
        t = np.ascontiguousarray(target, dtype=np.int32)
        p = np.ascontiguousarray(port, dtype=np.int32)
        w = np.ascontiguousarray(weight, dtype=np.float32)
        d = np.ascontiguousarray(delay, dtype=np.float32)
        self._chk(self.L.orc_connect_arrays(self.h, s.size, _iptr(s), _iptr(t), _iptr(p), _fptr(w), _fptr(d)))

    def ConnectFixedIndegreeGPU(self, source, target, indegree, weight, delay_min, delay_max, receptor=0,
                                seed=1):
        """The engine's per-target generated fixed in-degree block, restated on the host."""
        self._chk(self.L.orc_connect_generated(self.h, source.i0, source.n, target.i0, target.n, indegree,
                                               receptor, weight, delay_min, delay_max, seed))

    def SetPoissonStream(self, nodes, stream):
        """poisson_generator nodes draw from streams stream, stream+1, ..."""
        if not hasattr(nodes, "i0"):
            nodes = NodeSeq(nodes[0], len(nodes))
        self._chk(self.L.orc_set_poisson_stream(self.h, nodes.i0, nodes.n, int(stream) & 0xffffffff))

    # -- partitioned network: this process simulates its share of every group; exchange(self)
    #    is called after the update phase of every step and must pass the step's spikes
    #    (StepSpikes) to the other processes and inject theirs (InjectSpikes)
    def SetPartition(self, rank, world, exchange):
        self._chk(self.L.orc_set_partition(self.h, rank, world))
        fn = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p)

        def cb(user):
            try:
                exchange(self)
                return 0
            except Exception:
                return 1
        self._xch = fn(cb)
        self.L.orc_set_exchange(self.h, ctypes.cast(self._xch, ctypes.c_void_p), None)

    def StepSpikes(self):
        n = self.L.orc_step_spikes(self.h, None, None)
        nodes = np.zeros(max(n, 1), dtype=np.int32)
        heights = np.zeros(max(n, 1), dtype=np.float32)
        self.L.orc_step_spikes(self.h, _iptr(nodes), _fptr(heights))
        return nodes[:n], heights[:n]

    def InjectSpikes(self, nodes, heights):
        nodes = np.ascontiguousarray(nodes, dtype=np.int32)
        heights = np.ascontiguousarray(heights, dtype=np.float32)
        self._chk(self.L.orc_inject_spikes(self.h, _iptr(nodes), _fptr(heights), nodes.size))

    def Threads(self):
        return self.L.orc_threads()

    def ConnectionArrays(self):
        """All connections in reference order as a dict of numpy arrays."""
        n = self.L.orc_n_conn(self.h)
        a = {k: np.zeros(n, dtype=np.int32) for k in ("source", "group", "index", "target", "port", "syn")}
        a["delay"] = np.zeros(n, dtype=np.float32)
        a["weight"] = np.zeros(n, dtype=np.float32)
        self.L.orc_get_conns(self.h, _iptr(a["source"]), _iptr(a["group"]), _iptr(a["index"]),
                             _iptr(a["target"]), _iptr(a["port"]), _iptr(a["syn"]), _fptr(a["delay"]),
                             _fptr(a["weight"]))
        return a

    # -- recording
    def CreateRecord(self, file_name, var_name_list, i_node_list, i_port_list):
        for v, nd, p in zip(var_name_list, i_node_list, i_port_list):
            self.L.orc_record(self.h, nd, v.encode(), p)
        self.n_rec = len(var_name_list)
        return 0

    def GetRecordData(self, i_record=0):
        rows = self.L.orc_record_rows(self.h)
        out = np.zeros(rows * (self.n_rec + 1), dtype=np.float32)
        self.L.orc_record_data(self.h, _fptr(out))
        return out.reshape(rows, self.n_rec + 1)

    def ActivateSpikeCount(self, nodes):
        nodes = _nodes(nodes)
        self._chk(self.L.orc_activate_spike_count(self.h, nodes[0], len(nodes)))

    def ActivateRecSpikeTimes(self, nodes, max_n):
        nodes = _nodes(nodes)
        self._chk(self.L.orc_activate_rec_spike_times(self.h, nodes[0], len(nodes), max_n))

    def GetRecSpikeTimes(self, nodes):
        res = []
        for nd in _nodes(nodes):
            n = self._chk(self.L.orc_n_rec_spike_times(self.h, nd))
            out = np.zeros(max(n, 1), dtype=np.float32)
            self._chk(self.L.orc_rec_spike_times(self.h, nd, _fptr(out)))
            res.append(list(out[:n]))
        return res

    # -- simulation
    def Calibrate(self):
        self._chk(self.L.orc_calibrate(self.h))

    def Simulate(self, sim_time=1000.0):
        self._chk(self.L.orc_simulate(self.h, sim_time))

    def NDerivs(self):
        return self.L.orc_n_derivs(self.h)

    def NRk5Steps(self):
        return self.L.orc_n_rk5_steps(self.h)

    def NRk5Trials(self):
        return self.L.orc_n_rk5_trials(self.h)

    def NSpikes(self):
        return self.L.orc_n_spikes(self.h)

    def NEvents(self):
        return self.L.orc_n_events(self.h)

    # ---- learned RK5 step size (FP32 mode)
    def Rk5LogStart(self, capacity):
        self._chk(self.L.orc_log_start(self.h, int(capacity)))

    def Rk5LogStop(self):
        self._chk(self.L.orc_log_stop(self.h))

    def Rk5LogCount(self):
        off = ctypes.c_longlong(0)
        n = self.L.orc_log_count(self.h, ctypes.byref(off))
        return n, off.value

    def Rk5LogGet(self):
        """Logged tuples [n, 12]: 10 step features, accepted h, error of the accepted trial."""
        n, _ = self.Rk5LogCount()
        out = np.zeros((n, LOG_W), dtype=np.float32)
        if n:
            self.L.orc_log_get(self.h, _fptr(out))
        return out

    def StepBoundMode(self, on=True):
        """Analysis mode: every RK5 step starts from the largest step that passes the error
        test (bisection).  Its evaluation count is the floor any step proposal can reach."""
        self._chk(self.L.orc_set_bound_mode(self.h, 1 if on else 0))

    def StepModelSet(self, params, enable=True):
        p = np.ascontiguousarray(params, dtype=np.float32)
        assert p.size == STEP_MODEL_NPAR
        self._chk(self.L.orc_step_model_set(self.h, _fptr(p), 1 if enable else 0))


# learned step-size network: sizes of the flat parameter vector and of a log tuple
STEP_MODEL_NPAR = 1465
STEP_MODEL_NTRAIN = 1441
STEP_MODEL_TRAIN0 = 20
LOG_W = 12


def mlp_out(params, feat):
    """Network output for features [n, 10] (FP32, the engine kernel's arithmetic)."""
    p = np.ascontiguousarray(params, dtype=np.float32)
    f = np.ascontiguousarray(feat, dtype=np.float32).reshape(-1, 10)
    out = np.zeros(f.shape[0], dtype=np.float32)
    lib().orc_mlp_out(_fptr(p), _fptr(f), f.shape[0], _fptr(out))
    return out


def mlp_propose(params, feat):
    p = np.ascontiguousarray(params, dtype=np.float32)
    f = np.ascontiguousarray(feat, dtype=np.float32).reshape(-1, 10)
    out = np.zeros(f.shape[0], dtype=np.float32)
    lib().orc_mlp_propose(_fptr(p), _fptr(f), f.shape[0], _fptr(out))
    return out


def mlp_grad(params, feat, target):
    """FP64 mean squared error and its gradient w.r.t. the trainable block W1..b3."""
    p = np.ascontiguousarray(params, dtype=np.float32)
    f = np.ascontiguousarray(feat, dtype=np.float32).reshape(-1, 10)
    t = np.ascontiguousarray(target, dtype=np.float32)
    g = np.zeros(STEP_MODEL_NTRAIN, dtype=np.float64)
    loss = lib().orc_mlp_grad(_fptr(p), _fptr(f), _fptr(t), f.shape[0],
                              g.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return loss, g


def mlp_grad_bf16(params, feat, target):
    """mlp_grad with the operands of the GPU training kernel's tensor-core products
    rounded to BF16 where they enter a product (FP64 sums)."""
    p = np.ascontiguousarray(params, dtype=np.float32)
    f = np.ascontiguousarray(feat, dtype=np.float32).reshape(-1, 10)
    t = np.ascontiguousarray(target, dtype=np.float32)
    g = np.zeros(STEP_MODEL_NTRAIN, dtype=np.float64)
    loss = lib().orc_mlp_grad_bf16(_fptr(p), _fptr(f), _fptr(t), f.shape[0],
                                   g.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return loss, g


def exp_m(x):
    return lib().orc_exp_m(x)


def log_m(x):
    return lib().orc_log_m(x)


def poisson_draw(lam, seed, edge, tidx):
    return lib().orc_poisson_draw(lam, seed, edge, tidx)


def philox(c, k):
    out = (ctypes.c_uint * 4)()
    lib().orc_philox(c[0], c[1], c[2], c[3], k[0], k[1], out)
    return list(out)


class SynGroup(object):
    def __init__(self, i_syn_group):
        self.i_syn_group = i_syn_group


class ConnectionId(object):
    def __init__(self, i_source, i_group, i_conn):
        self.i_source = i_source
        self.i_group = i_group
        self.i_conn = i_conn


def _conn_filter(oracle, source, target):
    a = oracle.ConnectionArrays()
    keep = np.ones(a["source"].size, dtype=bool)
    if source is not None:
        keep &= np.isin(a["source"], np.asarray(_nodes(source)))
    if target is not None:
        keep &= np.isin(a["target"], np.asarray(_nodes(target)))
    return a, np.nonzero(keep)[0]


def _get_connections(self, source=None, target=None):
    a, idx = _conn_filter(self, source, target)
    return [ConnectionId(int(a["source"][i]), int(a["group"][i]), int(a["index"][i])) for i in idx]


def _conn_status(self, conn_ids, var_key=None):
    a = self.ConnectionArrays()
    key = {}
    for i in range(a["source"].size):
        key[(int(a["source"][i]), int(a["group"][i]), int(a["index"][i]))] = i
    res = []
    for c in conn_ids:
        i = key[(c.i_source, c.i_group, c.i_conn)]
        d = {"source": int(a["source"][i]), "target": int(a["target"][i]), "port": int(a["port"][i]),
             "syn": int(a["syn"][i]), "delay": float(a["delay"][i]), "weight": float(a["weight"][i])}
        if var_key is None:
            res.append(d)
        elif isinstance(var_key, (list, tuple)):
            res.append([d[k] for k in var_key])
        else:
            res.append(d[var_key])
    return res


Oracle.GetConnections = _get_connections
Oracle.GetConnStatusList = _conn_status
