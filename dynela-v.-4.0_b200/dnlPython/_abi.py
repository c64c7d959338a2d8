"""ctypes mirror of ``include/dnlgpu.h`` and the loader of ``libdnlgpu.so``.

The engine library is built in-tree (``dynela-v.-4.0_b200/lib/libdnlgpu.so``).
There is no CPU fallback: if the library or a CUDA device is missing, the
functions here raise :class:`EngineUnavailable`.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG_ROOT = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG_ROOT, "lib", "libdnlgpu.so")

# element families
ELQUA4NAX = 1
ELHEX8N3D = 2
ELQUA4N2D = 3
NODES_PER_ELEMENT = {ELQUA4NAX: 4, ELHEX8N3D: 8, ELQUA4N2D: 4}
DIMS = {ELQUA4NAX: 2, ELHEX8N3D: 3, ELQUA4N2D: 2}

STRESS_NEWTON, STRESS_DIRECT = 0, 1
ORDER_GIVEN, ORDER_RCM, ORDER_AUTO = 0, 1, 2
NUM_VARIANTS = 12  # element-pass variants of the autotuner (DNL_NUM_VARIANTS)
TS_COURANT = 0
TS_POWER_ITERATION = 1
PREC_FP64 = 0
PREC_MIXED = 1
BC_FREE, BC_RESTRAIN, BC_SPEED = 0, 1, 2

DNL_OK = 0
DNL_ERR_NEG_JACOBIAN, DNL_ERR_NEWTON = -3, -4
ERRORS = {
    -1: "invalid argument",
    -2: "CUDA error",
    -3: "negative Jacobian",
    -4: "radial return did not converge",
    -5: "power iteration did not converge",
    -6: "unsupported option",
    -7: "no CUDA device",
}

# integration point state components (component-major arrays)
IP_STRESS, IP_STRAIN, IP_PLASTIC_STRAIN = 0, 6, 12
IP_EPSP, IP_DEPSP, IP_GAMMA, IP_GAMMA_CUM, IP_YIELD, IP_T = 18, 19, 20, 21, 22, 23
IP_PRESSURE, IP_EINT, IP_EINEL, IP_DENSITY, IP_DETJ0 = 24, 25, 26, 27, 28
IP_NCOMP = 29

NODE_COORDS, NODE_DISP, NODE_U, NODE_SPEED, NODE_ACCEL, NODE_MASS, NODE_FORCE, NODE_SPEED_PREV = range(8)
NODE_U_PREV, NODE_ACCEL_PREV = 8, 9
# nodal fields as the reference's writers read them inside an increment
# (before its field swap): the buffer of before the last increment
NODE_PREV = {NODE_U: NODE_U_PREV, NODE_SPEED: NODE_SPEED_PREV, NODE_ACCEL: NODE_ACCEL_PREV}

# device history records (dnl_engine_set_history): header words of a record
HIST_HEAD = 5


class HistorySchedule(ctypes.Structure):
    _fields_ = [("start", ctypes.c_double), ("next", ctypes.c_double), ("save", ctypes.c_double)]


# node averages of the point state (dnl_engine_node_averages)
NODE_AVG_VON_MISES = 64

# result-file fields (DNL_VTK_*), by the reference's VTK label (Field.C:17-48)
VTK_FIELDS = {"coords": 0, "disp": 1, "dispInc": 2, "speed": 3, "speedInc": 4, "density": 5, "gamma": 6,
              "gammaCumulate": 7, "internalEnergy": 8, "plasticStrain": 9, "plasticStrainRate": 10,
              "pressure": 11, "T": 12, "vonMises": 13, "yield": 14, "mass": 15, "PlasticStrain": 16,
              "Strain": 17, "Stress": 18}


class EngineUnavailable(RuntimeError):
    """The CUDA engine library or a CUDA device is missing."""


class EngineError(RuntimeError):
    def __init__(self, code, message=""):
        self.code = code
        super().__init__(f"{ERRORS.get(code, 'error')} ({code}){': ' + message if message else ''}")


class Material(ctypes.Structure):
    _fields_ = [(n, ctypes.c_double) for n in (
        "young", "poisson", "density", "heat_capacity", "taylor_quinney", "T0",
        "A", "B", "C", "n", "m", "depsp0", "Tm", "Tref")]


class Function(ctypes.Structure):
    _fields_ = [("n_points", ctypes.c_int32),
                ("x", ctypes.POINTER(ctypes.c_double)),
                ("y", ctypes.POINTER(ctypes.c_double))]


class ModelDescC(ctypes.Structure):
    _fields_ = [
        ("elem_type", ctypes.c_int32),
        ("n_nodes", ctypes.c_int32),
        ("n_elems", ctypes.c_int32),
        ("coords", ctypes.POINTER(ctypes.c_double)),
        ("conn", ctypes.POINTER(ctypes.c_int32)),
        ("elem_mat", ctypes.POINTER(ctypes.c_int32)),
        ("n_materials", ctypes.c_int32),
        ("materials", ctypes.POINTER(Material)),
        ("v_init", ctypes.POINTER(ctypes.c_double)),
        ("bc_code", ctypes.POINTER(ctypes.c_int8)),
        ("bc_value", ctypes.POINTER(ctypes.c_double)),
        ("bc_func", ctypes.POINTER(ctypes.c_int32)),
        ("n_functions", ctypes.c_int32),
        ("functions", ctypes.POINTER(Function)),
        ("t_start", ctypes.c_double),
        ("t_end", ctypes.c_double),
        ("ts_method", ctypes.c_int32),
        ("ts_freq", ctypes.c_int32),
        ("ts_safety", ctypes.c_double),
        ("rho_b", ctypes.c_double),
        ("precision", ctypes.c_int32),
        ("stress_method", ctypes.c_int32),
        ("node_order", ctypes.c_int32),
    ]


ITEM_NODE, ITEM_POINT, ITEM_KINETIC = range(3)
ITEM_WIDTH = {ITEM_NODE: 3, ITEM_POINT: IP_NCOMP, ITEM_KINETIC: 1}


class Item(ctypes.Structure):
    """dnl_item: one history item (kind DNL_ITEM_*, field, index)."""
    _fields_ = [("kind", ctypes.c_int32), ("field", ctypes.c_int32), ("index", ctypes.c_int32),
                ("reserved", ctypes.c_int32)]


class Control(ctypes.Structure):
    _fields_ = [("time", ctypes.c_double), ("time_step", ctypes.c_double), ("t_end", ctypes.c_double),
                ("increment", ctypes.c_int64), ("status", ctypes.c_int32), ("bad_index", ctypes.c_int32),
                ("done", ctypes.c_int32), ("fp64_resolves", ctypes.c_int32), ("last_time_step", ctypes.c_double)]


def _ptr(a, ctype):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctype))


class ModelDesc:
    """Plain-array description of one model; ``cstruct()`` returns the C view.

    Arrays are kept alive by this object for as long as the C view is used.
    """

    def __init__(self, elem_type, coords, conn, materials, elem_mat=None, v_init=None,
                 bc_code=None, bc_value=None, bc_func=None, functions=(), t_start=0.0, t_end=1.0,
                 ts_method=TS_COURANT, ts_freq=10, ts_safety=0.9, rho_b=0.8182, precision=PREC_FP64,
                 stress_method=STRESS_NEWTON, node_order=None):
        self.elem_type = int(elem_type)
        npe = NODES_PER_ELEMENT[self.elem_type]
        self.coords = np.ascontiguousarray(coords, dtype=np.float64).reshape(-1, 3)
        self.conn = np.ascontiguousarray(conn, dtype=np.int32).reshape(-1, npe)
        self.materials = [dict(m) for m in materials]
        nN = self.coords.shape[0]
        self.elem_mat = None if elem_mat is None else np.ascontiguousarray(elem_mat, dtype=np.int32)
        self.v_init = None if v_init is None else np.ascontiguousarray(v_init, dtype=np.float64).reshape(nN, 3)
        self.bc_code = None if bc_code is None else np.ascontiguousarray(bc_code, dtype=np.int8).reshape(nN, 3)
        self.bc_value = None if bc_value is None else np.ascontiguousarray(bc_value, dtype=np.float64).reshape(nN, 3)
        self.bc_func = None if bc_func is None else np.ascontiguousarray(bc_func, dtype=np.int32).reshape(nN, 3)
        self.functions = [(np.ascontiguousarray(x, dtype=np.float64), np.ascontiguousarray(y, dtype=np.float64))
                          for x, y in functions]
        self.t_start, self.t_end = float(t_start), float(t_end)
        self.ts_method, self.ts_freq = int(ts_method), int(ts_freq)
        self.ts_safety, self.rho_b = float(ts_safety), float(rho_b)
        self.precision = int(precision)
        self.stress_method = int(stress_method)
        self.node_order = ORDER_GIVEN if node_order is None else int(node_order)
        self._c = None

    @property
    def n_nodes(self):
        return self.coords.shape[0]

    @property
    def n_elems(self):
        return self.conn.shape[0]

    @property
    def nodes_per_element(self):
        return NODES_PER_ELEMENT[self.elem_type]

    @property
    def n_ips(self):
        return self.n_elems * self.nodes_per_element

    def copy(self, **changes):
        kw = dict(elem_type=self.elem_type, coords=self.coords.copy(), conn=self.conn.copy(),
                  materials=[dict(m) for m in self.materials], elem_mat=self.elem_mat, v_init=self.v_init,
                  bc_code=self.bc_code, bc_value=self.bc_value, bc_func=self.bc_func,
                  functions=self.functions, t_start=self.t_start, t_end=self.t_end,
                  ts_method=self.ts_method, ts_freq=self.ts_freq, ts_safety=self.ts_safety,
                  rho_b=self.rho_b, precision=self.precision, stress_method=self.stress_method,
                  node_order=self.node_order)
        kw.update(changes)
        return ModelDesc(**kw)

    def cstruct(self):
        keys = [f[0] for f in Material._fields_]
        self._mats = (Material * len(self.materials))(*[Material(*[float(m[k]) for k in keys])
                                                         for m in self.materials])
        self._funcs = (Function * max(1, len(self.functions)))()
        for i, (x, y) in enumerate(self.functions):
            self._funcs[i] = Function(len(x), _ptr(x, ctypes.c_double), _ptr(y, ctypes.c_double))
        c = ModelDescC()
        c.elem_type = self.elem_type
        c.n_nodes = self.n_nodes
        c.n_elems = self.n_elems
        c.coords = _ptr(self.coords, ctypes.c_double)
        c.conn = _ptr(self.conn, ctypes.c_int32)
        c.elem_mat = _ptr(self.elem_mat, ctypes.c_int32)
        c.n_materials = len(self.materials)
        c.materials = self._mats
        c.v_init = _ptr(self.v_init, ctypes.c_double)
        c.bc_code = _ptr(self.bc_code, ctypes.c_int8)
        c.bc_value = _ptr(self.bc_value, ctypes.c_double)
        c.bc_func = _ptr(self.bc_func, ctypes.c_int32)
        c.n_functions = len(self.functions)
        c.functions = self._funcs
        c.t_start, c.t_end = self.t_start, self.t_end
        c.ts_method, c.ts_freq = self.ts_method, self.ts_freq
        c.ts_safety, c.rho_b = self.ts_safety, self.rho_b
        c.precision = self.precision
        c.stress_method = self.stress_method
        c.node_order = self.node_order
        self._c = c
        return c


MLP_IN, MLP_HIDDEN, MLP_PAIR_WORDS = 5, 64, 8
MODE_PLAIN, MODE_STATS, MODE_HARVEST, MODE_GUESS = 0, 1, 2, 3
GUESS_ALL, GUESS_FIRST_YIELD = 0, 1


class Mlp(ctypes.Structure):
    """dnl_mlp: the learned initial guess of the radial return (FP32 weights)."""
    _fields_ = [("w1", (ctypes.c_float * 16) * MLP_HIDDEN), ("b1", ctypes.c_float * MLP_HIDDEN),
                ("w2", (ctypes.c_float * MLP_HIDDEN) * MLP_HIDDEN), ("b2", ctypes.c_float * MLP_HIDDEN),
                ("w3", (ctypes.c_float * MLP_HIDDEN) * MLP_HIDDEN), ("b3", ctypes.c_float * MLP_HIDDEN),
                ("w4", ctypes.c_float * MLP_HIDDEN), ("b4", ctypes.c_float),
                ("in_mean", ctypes.c_float * MLP_IN), ("in_scale", ctypes.c_float * MLP_IN),
                ("out_exp", ctypes.c_float), ("in_clip", ctypes.c_float)]

    NPARAM = 64 * 16 + 64 + 64 * 64 + 64 + 64 * 64 + 64 + 64 + 1
    _LAYOUT = (("w1", (64, 16)), ("b1", (64,)), ("w2", (64, 64)), ("b2", (64,)), ("w3", (64, 64)),
               ("b3", (64,)), ("w4", (64,)), ("b4", ()), ("in_mean", (5,)), ("in_scale", (5,)), ("out_exp", ()),
               ("in_clip", ()))

    def to_dict(self):
        import numpy as np
        a = np.frombuffer(bytes(self), dtype=np.float32)
        out, off = {}, 0
        for name, shape in self._LAYOUT:
            n = int(np.prod(shape)) if shape else 1
            out[name] = a[off:off + n].reshape(shape).copy() if shape else np.float32(a[off])
            off += n
        return out

    @classmethod
    def from_dict(cls, d):
        import numpy as np
        buf = np.concatenate([np.asarray(d.get(k, 0.0), dtype=np.float32).ravel() for k, _ in cls._LAYOUT])
        m = cls()
        ctypes.memmove(ctypes.addressof(m), buf.ctypes.data, buf.nbytes)
        return m


def material(young, poisson, density, heat_capacity, taylor_quinney, T0, A, B, C, n, m, depsp0, Tm, Tref):
    return dict(young=young, poisson=poisson, density=density, heat_capacity=heat_capacity,
                taylor_quinney=taylor_quinney, T0=T0, A=A, B=B, C=C, n=n, m=m, depsp0=depsp0, Tm=Tm, Tref=Tref)


_lib = None


def load_library():
    """Load libdnlgpu.so (built in-tree); raise if it is absent."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise EngineUnavailable(f"{LIB_PATH} is missing: build it with `python __graft_entry__.py build` "
                                "(no CPU fallback exists for the engine)")
    lib = ctypes.CDLL(LIB_PATH)
    vp = ctypes.c_void_p
    i32, i64, dbl = ctypes.c_int32, ctypes.c_int64, ctypes.c_double
    pd = ctypes.POINTER(ctypes.c_double)
    sig = {
        "dnl_device_count": (ctypes.c_int, []),
        "dnl_engine_create": (ctypes.c_int, [ctypes.POINTER(ModelDescC), ctypes.POINTER(vp)]),
        "dnl_engine_batch_create": (ctypes.c_int, [ctypes.POINTER(ctypes.POINTER(ModelDescC)), i32,
                                                   ctypes.POINTER(vp)]),
        "dnl_engine_destroy": (ctypes.c_int, [vp]),
        "dnl_engine_last_error": (ctypes.c_char_p, [vp]),
        "dnl_engine_init": (ctypes.c_int, [vp]),
        "dnl_engine_run": (ctypes.c_int, [vp, dbl, i64, ctypes.POINTER(i64)]),
        "dnl_engine_element_pass": (ctypes.c_int, [vp, dbl]),
        "dnl_engine_sizes": (ctypes.c_int, [vp] + [ctypes.POINTER(i32)] * 4),
        "dnl_engine_instance_offsets": (ctypes.c_int, [vp, i32] + [ctypes.POINTER(i32)] * 3),
        "dnl_engine_control": (ctypes.c_int, [vp, i32, ctypes.POINTER(Control)]),
        "dnl_engine_node_order": (ctypes.c_int, [vp, i32, ctypes.POINTER(i32)]),
        "dnl_engine_get_nodes": (ctypes.c_int, [vp, i32, pd]),
        "dnl_engine_set_nodes": (ctypes.c_int, [vp, i32, pd]),
        "dnl_engine_get_ips": (ctypes.c_int, [vp, pd]),
        "dnl_engine_get_ips_native": (ctypes.c_int, [vp, vp, i32]),
        "dnl_engine_set_ips": (ctypes.c_int, [vp, pd]),
        "dnl_engine_energies": (ctypes.c_int, [vp, i32, pd]),
        "dnl_engine_set_items": (ctypes.c_int, [vp, ctypes.POINTER(Item), i32, ctypes.POINTER(i64)]),
        "dnl_engine_gather_items": (ctypes.c_int, [vp, pd]),
        "dnl_engine_node_averages": (ctypes.c_int, [vp, ctypes.POINTER(i32), i32, pd]),
        "dnl_engine_set_history": (ctypes.c_int, [vp, ctypes.POINTER(HistorySchedule), i32, i32]),
        "dnl_engine_history_records": (ctypes.c_int, [vp, pd, i64, ctypes.POINTER(i64)]),
        "dnl_engine_write_vtk": (ctypes.c_int, [vp, i32, ctypes.c_char_p, ctypes.c_char_p, ctypes.POINTER(i32),
                                                i32, i32]),
        "dnl_engine_set_timing": (ctypes.c_int, [vp, i32]),
        "dnl_engine_timings": (ctypes.c_int, [vp, pd]),
        "dnl_engine_launch_count": (ctypes.c_int64, [vp]),
        "dnl_engine_set_graph_increments": (ctypes.c_int, [vp, i32]),
        "dnl_engine_autotune": (ctypes.c_int, [vp, i32]),
        "dnl_engine_variant": (ctypes.c_int, [vp, ctypes.POINTER(i32), pd]),
        "dnl_engine_set_variant": (ctypes.c_int, [vp, i32]),
        "dnl_variant_name": (ctypes.c_char_p, [i32, i32]),
        "dnl_element_pass_static": (ctypes.c_int, [i32, i32, i32, vp, vp, vp, ctypes.POINTER(Material),
                                                   dbl, vp, vp, vp]),
        "dnl_engine_set_mode": (ctypes.c_int, [vp, i32]),
        "dnl_engine_set_guess_network": (ctypes.c_int, [vp, ctypes.POINTER(Mlp)]),
        "dnl_engine_set_harvest": (ctypes.c_int, [vp, vp, i64, i32]),
        "dnl_engine_harvest_count": (ctypes.c_int, [vp, ctypes.POINTER(i64)]),
        "dnl_engine_newton_stats": (ctypes.c_int, [vp, ctypes.POINTER(i64), i32]),
        "dnl_engine_set_guess_scope": (ctypes.c_int, [vp, i32]),
        "dnl_mesh_order_rcm": (ctypes.c_int, [i32, i32, i32, ctypes.POINTER(i32), ctypes.POINTER(i32)]),
        "dnl_mesh_span": (ctypes.c_int, [i32, i32, i32, ctypes.POINTER(i32), ctypes.POINTER(i32), pd]),
        "dnl_mlp_forward": (ctypes.c_int, [ctypes.POINTER(Mlp), vp, i64, vp, vp]),
        "dnl_mlp_gradients": (ctypes.c_int, [ctypes.POINTER(Mlp), vp, vp, i64, ctypes.POINTER(Mlp),
                                             ctypes.POINTER(ctypes.c_float), vp]),
        "dnl_mlp_train": (ctypes.c_int, [ctypes.POINTER(Mlp), vp, vp, i64, i32, i32, ctypes.c_float,
                                         ctypes.c_uint64, ctypes.POINTER(ctypes.c_float), vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def exported_symbols():
    """Names the header declares (used by the ABI test)."""
    hdr = os.path.join(os.path.dirname(PKG_ROOT), "include", "dnlgpu.h")
    import re
    with open(hdr) as f:
        text = f.read()
    return sorted(set(re.findall(r"^\s*(?:int|int64_t|const char \*)\s*\*?(dnl_\w+)\s*\(", text, re.M)))


def mesh_order_rcm(conn, n_nodes):
    """Reverse Cuthill-McKee numbering of a mesh's nodes (dnl_mesh_order_rcm,
    host code): order[k] is the node numbered k."""
    lib = load_library()
    conn = np.ascontiguousarray(conn, dtype=np.int32)
    order = np.empty(int(n_nodes), dtype=np.int32)
    rc = lib.dnl_mesh_order_rcm(int(n_nodes), conn.shape[0], conn.shape[1], _ptr(conn, ctypes.c_int32),
                                _ptr(order, ctypes.c_int32))
    if rc != 0:
        raise EngineError(rc, "dnl_mesh_order_rcm: invalid mesh")
    return order


def mesh_span(conn, n_nodes, order=None):
    """Mean over the elements of (largest - smallest node number) under the
    numbering `order` (dnl_mesh_span; None: the given numbering)."""
    lib = load_library()
    conn = np.ascontiguousarray(conn, dtype=np.int32)
    if order is not None:
        order = np.ascontiguousarray(order, dtype=np.int32)
    out = ctypes.c_double()
    rc = lib.dnl_mesh_span(int(n_nodes), conn.shape[0], conn.shape[1], _ptr(conn, ctypes.c_int32),
                           _ptr(order, ctypes.c_int32), ctypes.byref(out))
    if rc != 0:
        raise EngineError(rc, "dnl_mesh_span: invalid mesh or numbering")
    return out.value
