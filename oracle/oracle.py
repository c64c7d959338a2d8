"""ctypes binding of oracle/liboracle.so, the C restatement of the DynELA hot
path (dnl_oracle.c).

Test infrastructure only: the checker the GPU engine is compared with.  The
engine never imports this module.
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "dynela-v.-4.0_b200"))
from dnlPython import _abi  # noqa: E402

_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            raise FileNotFoundError(f"{LIB} is not built (make -C oracle liboracle.so)")
        L = ctypes.CDLL(LIB)
        vp, pd = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)
        L.orc_create.restype = vp
        L.orc_create.argtypes = [ctypes.POINTER(_abi.ModelDescC)]
        L.orc_destroy.argtypes = [vp]
        L.orc_last_error.restype = ctypes.c_char_p
        L.orc_init.argtypes = [vp]
        L.orc_run.restype = ctypes.c_long
        L.orc_run.argtypes = [vp, ctypes.c_double, ctypes.c_long]
        L.orc_element_pass.argtypes = [vp, ctypes.c_double]
        for f in ("orc_get_nodes", "orc_set_nodes"):
            getattr(L, f).argtypes = [vp, ctypes.c_int, pd]
        L.orc_get_ips.argtypes = [vp, pd]
        L.orc_set_ips.argtypes = [vp, pd]
        L.orc_control.argtypes = [vp, pd]
        L.orc_courant.restype = ctypes.c_double
        L.orc_courant.argtypes = [vp]
        L.orc_element_lengths.argtypes = [vp, pd, pd]
        L.orc_energies.argtypes = [vp, pd]
        L.orc_sym_eigen3.argtypes = [pd, pd, pd]
        L.orc_polar_lnU.argtypes = [pd, pd, pd]
        L.orc_polar_lnU_h.argtypes = [pd, pd, pd]
        L.orc_set_polar_route.argtypes = [vp, ctypes.c_int]
        L.orc_radial_return.argtypes = [ctypes.POINTER(_abi.Material), pd, ctypes.c_double, pd]
        L.orc_jc_yield.restype = ctypes.c_double
        L.orc_jc_yield.argtypes = [ctypes.POINTER(_abi.Material)] + [ctypes.c_double] * 3
        L.orc_jc_hardening.restype = ctypes.c_double
        L.orc_jc_hardening.argtypes = [ctypes.POINTER(_abi.Material)] + [ctypes.c_double] * 4
        L.orc_abi_sizeof.restype = ctypes.c_long
        L.orc_abi_sizeof.argtypes = [ctypes.c_int]
        _lib = L
    return _lib


def _pd(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class OracleModel:
    """The C restatement on one model description."""

    def __init__(self, desc):
        self.desc = desc
        self._c = desc.cstruct()
        self.h = lib().orc_create(ctypes.byref(self._c))
        if not self.h:
            raise RuntimeError("orc_create failed: " + lib().orc_last_error().decode())

    def set_polar_route(self, route):
        """0: the reference's polar decomposition of C = F^T F; 1: the same
        from H = F - I (A = C - I), free of the cancellation in C's entries
        (orc_polar_lnU_h)."""
        lib().orc_set_polar_route(self.h, int(route))

    def init(self):
        rc = lib().orc_init(self.h)
        if rc:
            raise RuntimeError(f"orc_init failed ({rc}) {lib().orc_last_error().decode()}")

    def run(self, t_stop=np.inf, max_incs=0):
        return lib().orc_run(self.h, float(t_stop), int(max_incs))

    def element_pass(self, dt):
        rc = lib().orc_element_pass(self.h, float(dt))
        if rc:
            raise RuntimeError(f"orc_element_pass failed ({rc})")

    def control(self):
        out = np.zeros(4)
        lib().orc_control(self.h, _pd(out))
        return dict(time=out[0], time_step=out[1], increment=int(out[2]), status=int(out[3]))

    def nodes(self, field):
        out = np.zeros((self.desc.n_nodes, 3))
        assert lib().orc_get_nodes(self.h, field, _pd(out)) == 0
        return out

    def set_nodes(self, field, values):
        a = np.ascontiguousarray(values, dtype=np.float64).reshape(self.desc.n_nodes, 3)
        assert lib().orc_set_nodes(self.h, field, _pd(a)) == 0

    def ips(self):
        out = np.zeros((_abi.IP_NCOMP, self.desc.n_ips))
        lib().orc_get_ips(self.h, _pd(out))
        return out

    def set_ips(self, values):
        a = np.ascontiguousarray(values, dtype=np.float64).reshape(_abi.IP_NCOMP, self.desc.n_ips)
        lib().orc_set_ips(self.h, _pd(a))

    def courant(self):
        return lib().orc_courant(self.h)

    def element_lengths(self):
        ln = np.zeros(self.desc.n_elems)
        wv = np.zeros(self.desc.n_elems)
        lib().orc_element_lengths(self.h, _pd(ln), _pd(wv))
        return ln, wv

    def energies(self):
        out = np.zeros(3)
        lib().orc_energies(self.h, _pd(out))
        return out

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
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


def abi_sizeof(which):
    """sizeof(dnl_model_desc / dnl_material / dnl_function / dnl_control) as compiled from the header."""
    return lib().orc_abi_sizeof(which)


def radial_return(mat, dE, dt, state):
    """One radial return on a 21-double point state (see orc_radial_return)."""
    m = _abi.Material(*[float(mat[k]) for k, _ in _abi.Material._fields_])
    st = np.ascontiguousarray(state, dtype=np.float64).copy()
    de = np.ascontiguousarray(dE, dtype=np.float64)
    it = lib().orc_radial_return(ctypes.byref(m), _pd(de), float(dt), _pd(st))
    return it, st


def sym_eigen3(a6):
    a = np.ascontiguousarray(a6, dtype=np.float64)
    lam = np.zeros(3)
    vec = np.zeros((3, 3))
    lib().orc_sym_eigen3(_pd(a), _pd(lam), _pd(vec))
    return lam, vec


def polar_lnU(F):
    F = np.ascontiguousarray(F, dtype=np.float64).reshape(9)
    lnU = np.zeros(6)
    R = np.zeros(9)
    lib().orc_polar_lnU(_pd(F), _pd(lnU), _pd(R))
    return lnU, R.reshape(3, 3)


def polar_lnU_h(H):
    """The same decomposition of F = I + H from H (orc_polar_lnU_h)."""
    H = np.ascontiguousarray(H, dtype=np.float64).reshape(9)
    lnU = np.zeros(6)
    R = np.zeros(9)
    lib().orc_polar_lnU_h(_pd(H), _pd(lnU), _pd(R))
    return lnU, R.reshape(3, 3)


def jc_yield(mat, epsp, depsp, T):
    m = _abi.Material(*[float(mat[k]) for k, _ in _abi.Material._fields_])
    return lib().orc_jc_yield(ctypes.byref(m), epsp, depsp, T)


def jc_hardening(mat, epsp, depsp, T, dt):
    m = _abi.Material(*[float(mat[k]) for k, _ in _abi.Material._fields_])
    return lib().orc_jc_hardening(ctypes.byref(m), epsp, depsp, T, dt)
