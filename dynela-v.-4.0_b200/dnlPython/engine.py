"""Python handle over the C ABI of ``libdnlgpu.so`` (include/dnlgpu.h).

`Engine` owns one engine handle: one model, or a batch of independent models
advanced together.  There is no CPU path: construction raises
:class:`~dnlPython._abi.EngineUnavailable` when the library or a CUDA device is
missing.
"""
import ctypes
import os

import numpy as np

from . import _abi


def _pd(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Engine:
    def __init__(self, descs):
        lib = _abi.load_library()
        if lib.dnl_device_count() <= 0:
            raise _abi.EngineUnavailable("no CUDA device is visible to the engine")
        if isinstance(descs, _abi.ModelDesc):
            descs = [descs]
        self.descs = list(descs)
        self._cs = [d.cstruct() for d in self.descs]
        arr = (ctypes.POINTER(_abi.ModelDescC) * len(self._cs))(*[ctypes.pointer(c) for c in self._cs])
        h = ctypes.c_void_p()
        rc = lib.dnl_engine_batch_create(arr, len(self._cs), ctypes.byref(h))
        if rc != 0:
            raise _abi.EngineError(rc, lib.dnl_engine_last_error(None).decode())
        self._lib = lib
        self.h = h
        ni, nn, ne, nip = (ctypes.c_int32() for _ in range(4))
        lib.dnl_engine_sizes(h, ctypes.byref(ni), ctypes.byref(nn), ctypes.byref(ne), ctypes.byref(nip))
        self.n_instances, self.n_nodes, self.n_elems, self.n_ips = ni.value, nn.value, ne.value, nip.value

    def _check(self, rc):
        if rc != 0:
            raise _abi.EngineError(rc, self._lib.dnl_engine_last_error(self.h).decode())

    def init(self):
        self._check(self._lib.dnl_engine_init(self.h))
        return self

    def run(self, t_pause=np.inf, max_incs=0, check=True):
        """Advance to t_pause / max_incs.  check=False leaves a failed
        instance's error in control(i)['status'] instead of raising (batches)."""
        done = ctypes.c_int64()
        rc = self._lib.dnl_engine_run(self.h, float(t_pause), int(max_incs), ctypes.byref(done))
        if check or rc not in (_abi.DNL_ERR_NEG_JACOBIAN, _abi.DNL_ERR_NEWTON):
            self._check(rc)
        return done.value

    def element_pass(self, dt):
        self._check(self._lib.dnl_engine_element_pass(self.h, float(dt)))

    def control(self, instance=0):
        c = _abi.Control()
        self._check(self._lib.dnl_engine_control(self.h, int(instance), ctypes.byref(c)))
        return dict(time=c.time, time_step=c.time_step, t_end=c.t_end, increment=c.increment,
                    status=c.status, bad_index=c.bad_index, done=bool(c.done), fp64_resolves=c.fp64_resolves,
                    last_time_step=c.last_time_step)

    def offsets(self, instance):
        n0, e0, q0 = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
        self._check(self._lib.dnl_engine_instance_offsets(self.h, int(instance), ctypes.byref(n0),
                                                          ctypes.byref(e0), ctypes.byref(q0)))
        return n0.value, e0.value, q0.value

    def node_order(self, instance=0):
        """The engine's numbering of an instance's nodes: _abi.ORDER_GIVEN or
        _abi.ORDER_RCM (every node array of this handle stays in the
        description's numbering either way)."""
        o = ctypes.c_int32()
        self._check(self._lib.dnl_engine_node_order(self.h, int(instance), ctypes.byref(o)))
        return o.value

    @staticmethod
    def _out(out, shape):
        """A caller's output array (C-contiguous float64 of `shape`, for
        example a view of page-locked memory, which copies several times faster
        than pageable memory), or a new one."""
        if out is None:
            return np.zeros(shape)
        if out.shape != shape or out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError(f"output array must be C-contiguous float64 of shape {shape}")
        return out

    def nodes(self, field, out=None):
        out = self._out(out, (self.n_nodes, 3))
        self._check(self._lib.dnl_engine_get_nodes(self.h, int(field), _pd(out)))
        return out

    def set_nodes(self, field, values):
        a = np.ascontiguousarray(values, dtype=np.float64).reshape(self.n_nodes, 3)
        self._check(self._lib.dnl_engine_set_nodes(self.h, int(field), _pd(a)))

    def ips(self, out=None):
        out = self._out(out, (_abi.IP_NCOMP, self.n_ips))
        self._check(self._lib.dnl_engine_get_ips(self.h, _pd(out)))
        return out

    def ips_native(self, out=None):
        """The point state in the engine's own precision (float32 on the
        mixed path, float64 on the FP64 path), [IP_NCOMP, n_ips]."""
        dt = np.float32 if self.descs[0].precision == _abi.PREC_MIXED else np.float64
        shape = (_abi.IP_NCOMP, self.n_ips)
        if out is None:
            out = np.empty(shape, dtype=dt)
        elif out.shape != shape or out.dtype != dt or not out.flags.c_contiguous:
            raise ValueError(f"output array must be C-contiguous {np.dtype(dt).name} of shape {shape}")
        self._check(self._lib.dnl_engine_get_ips_native(self.h, out.ctypes.data_as(ctypes.c_void_p),
                                                         out.dtype.itemsize))
        return out

    def set_ips(self, values):
        a = np.ascontiguousarray(values, dtype=np.float64).reshape(_abi.IP_NCOMP, self.n_ips)
        self._check(self._lib.dnl_engine_set_ips(self.h, _pd(a)))

    def set_items(self, items):
        """Select the history items gathered by gather_items(): a list of
        (kind, field, index) with kind ITEM_NODE / ITEM_POINT / ITEM_KINETIC."""
        arr = (_abi.Item * max(1, len(items)))(*[_abi.Item(int(k), int(f), int(i), 0) for k, f, i in items])
        n = ctypes.c_int64()
        self._check(self._lib.dnl_engine_set_items(self.h, arr, len(items), ctypes.byref(n)))
        self._n_values = n.value
        return n.value

    def gather_items(self):
        """The selected items' values, item after item (3 doubles for a node,
        IP_NCOMP for a point, 1 for a kinetic energy)."""
        out = np.zeros(max(1, getattr(self, "_n_values", 0)))
        self._check(self._lib.dnl_engine_gather_items(self.h, _pd(out)))
        return out[:getattr(self, "_n_values", 0)]

    def node_averages(self, comps):
        """Nodal values of point-state components (IP_* or NODE_AVG_VON_MISES)
        as the reference extracts them for its node fields: [len(comps), n_nodes]."""
        c = (ctypes.c_int32 * len(comps))(*[int(x) for x in comps])
        out = np.zeros((len(comps), self.n_nodes))
        self._check(self._lib.dnl_engine_node_averages(self.h, c, len(comps), _pd(out)))
        return out

    def write_vtk(self, path, fields, prev=False, instance=0, title="DynELA FEM Code v.4.0"):
        """Result file of one instance in the reference's VTK format; `fields`
        are labels of _abi.VTK_FIELDS; prev: the nodal increments, speeds and
        accelerations of before the last increment (the reference's files
        written inside an increment)."""
        codes = [_abi.VTK_FIELDS[f] for f in fields]
        c = (ctypes.c_int32 * max(1, len(codes)))(*codes)
        self._check(self._lib.dnl_engine_write_vtk(self.h, int(instance), os.fsencode(path), title.encode(), c,
                                                   len(codes), int(bool(prev))))

    def set_history(self, schedules, capacity=0):
        """History records on the device: schedules [(start, next, save)],
        the save rule of HistoryFile::save evaluated after every increment;
        a record holds the items of set_items()."""
        arr = (_abi.HistorySchedule * max(1, len(schedules)))(*[_abi.HistorySchedule(*map(float, s))
                                                                for s in schedules])
        self._check(self._lib.dnl_engine_set_history(self.h, arr, len(schedules), int(capacity)))

    def history_records(self):
        """The records waiting, oldest first: a list of (time, increment,
        time step, due mask, values)."""
        n = ctypes.c_int64()
        self._check(self._lib.dnl_engine_history_records(self.h, None, 0, ctypes.byref(n)))
        width = _abi.HIST_HEAD + getattr(self, "_n_values", 0)
        buf = np.zeros((max(1, n.value), width))
        self._check(self._lib.dnl_engine_history_records(self.h, _pd(buf), n.value, ctypes.byref(n)))
        return [(r[0], int(r[1]), r[2], int(r[3]) | (int(r[4]) << 32), r[_abi.HIST_HEAD:])
                for r in buf[:n.value]]

    def energies(self, instance=0):
        out = np.zeros(3)
        self._check(self._lib.dnl_engine_energies(self.h, int(instance), _pd(out)))
        return out

    def set_timing(self, on=True):
        self._check(self._lib.dnl_engine_set_timing(self.h, int(bool(on))))

    def timings(self):
        out = np.zeros(4)
        self._check(self._lib.dnl_engine_timings(self.h, _pd(out)))
        return dict(element_ms=out[0], nodal_ms=out[1], timestep_ms=out[2], run_ms=out[3])

    def autotune(self, steps=8):
        """Pick the fastest element-pass variant; the simulation state is unchanged."""
        self._check(self._lib.dnl_engine_autotune(self.h, int(steps)))
        return self.variant()

    def variant(self):
        v = ctypes.c_int32()
        ms = np.zeros(_abi.NUM_VARIANTS)
        self._check(self._lib.dnl_engine_variant(self.h, ctypes.byref(v), _pd(ms)))
        return v.value, ms

    def set_variant(self, v):
        self._check(self._lib.dnl_engine_set_variant(self.h, int(v)))

    def set_graph_increments(self, n):
        """Increments captured in one graph replay (dnl_engine_set_graph_increments)."""
        self._check(self._lib.dnl_engine_set_graph_increments(self.h, int(n)))

    def launch_count(self):
        return int(self._lib.dnl_engine_launch_count(self.h))

    # ---- learned initial guess of the radial return
    def set_mode(self, mode):
        self._check(self._lib.dnl_engine_set_mode(self.h, int(mode)))

    def set_guess_network(self, net):
        self._check(self._lib.dnl_engine_set_guess_network(self.h, ctypes.byref(net)))

    def set_harvest(self, d_pairs_ptr, capacity, stride):
        """d_pairs_ptr: device pointer of capacity*8 float32 (e.g. a torch tensor's data_ptr())."""
        self._check(self._lib.dnl_engine_set_harvest(self.h, ctypes.c_void_p(d_pairs_ptr), int(capacity),
                                                     int(stride)))

    def harvest_count(self):
        n = ctypes.c_int64()
        self._check(self._lib.dnl_engine_harvest_count(self.h, ctypes.byref(n)))
        return n.value

    def set_guess_scope(self, scope):
        self._check(self._lib.dnl_engine_set_guess_scope(self.h, int(scope)))

    def newton_stats(self, reset=False):
        """(yield-function evaluations, yielding points, yielding points of the
        guess scope, their evaluations)."""
        out = (ctypes.c_int64 * 4)()
        self._check(self._lib.dnl_engine_newton_stats(self.h, out, int(bool(reset))))
        return tuple(int(v) for v in out)

    def close(self):
        if getattr(self, "h", None):
            self._lib.dnl_engine_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
