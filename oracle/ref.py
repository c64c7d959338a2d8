"""ctypes binding of oracle/_ref/libdnlref.so: the DynELA reference compiled from
its own sources plus the C-ABI harness in ref_harness.cpp.

Test infrastructure only: the engine never imports this module.  Only one
reference model can be alive per process (the reference keeps its model in a
global); `RefModel.close()` releases it.
"""
import ctypes
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libdnlref.so")
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "dynela-v.-4.0_b200"))
from dnlPython import _abi  # noqa: E402

_lib = None


def available():
    return os.path.exists(LIB)


def reference_dir():
    """The reference checkout (its Samples/ and Sources/): the environment
    variable DNL_REFERENCE, else the default of oracle/Makefile.  None when
    the directory does not exist (the prebuilt oracle/_ref still works)."""
    import subprocess
    d = os.environ.get("DNL_REFERENCE")
    if not d:
        try:
            d = subprocess.run(["make", "-s", "-C", HERE, "ref-dir"], capture_output=True, text=True,
                               check=True).stdout.strip()
        except (OSError, subprocess.CalledProcessError):
            d = None
    return d if d and os.path.isdir(d) else None


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{LIB} is not built (make -C oracle ref)")
        L = ctypes.CDLL(LIB)
        vp, pd = ctypes.c_void_p, ctypes.POINTER(ctypes.c_double)
        L.ref_create.restype = vp
        L.ref_create.argtypes = [ctypes.POINTER(_abi.ModelDescC), ctypes.c_char_p]
        L.ref_last_error.restype = ctypes.c_char_p
        L.ref_init.argtypes = [vp]
        L.ref_run.restype = ctypes.c_long
        L.ref_run.argtypes = [vp, ctypes.c_double, ctypes.c_long]
        L.ref_solve_native.argtypes = [vp]
        L.ref_solver_seconds.restype = ctypes.c_double
        L.ref_solver_seconds.argtypes = [vp]
        L.ref_control.argtypes = [vp, pd]
        L.ref_get_nodes.argtypes = [vp, ctypes.c_int, pd]
        L.ref_set_nodes.argtypes = [vp, ctypes.c_int, pd]
        L.ref_get_ips.argtypes = [vp, pd]
        L.ref_set_ips.argtypes = [vp, pd]
        L.ref_element_pass.argtypes = [vp, ctypes.c_double]
        L.ref_courant.restype = ctypes.c_double
        L.ref_courant.argtypes = [vp]
        L.ref_element_lengths.argtypes = [vp, pd, pd]
        L.ref_timer.restype = ctypes.c_double
        L.ref_timer.argtypes = [vp, ctypes.c_char_p]
        L.ref_set_threads.argtypes = [ctypes.c_int]
        L.ref_point_kinematics.argtypes = [vp, ctypes.c_long, pd]
        L.ref_rotation_orthogonality.argtypes = [vp, pd]
        L.ref_enable_vtk.argtypes = [vp, ctypes.c_double, ctypes.c_double, ctypes.c_double]
        L.ref_write_final_vtk.argtypes = [vp]
        L.ref_destroy.argtypes = [vp]
        _lib = L
    return _lib


def _pd(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class RefModel:
    """The reference solver on one model description."""

    def __init__(self, desc, threads=None):
        L = lib()
        self.desc = desc
        self._c = desc.cstruct()
        self._tmp = tempfile.mkdtemp(prefix="dnlref_")
        self.h = L.ref_create(ctypes.byref(self._c), self._tmp.encode())
        if not self.h:
            raise RuntimeError("ref_create failed: " + L.ref_last_error().decode())
        if threads:
            L.ref_set_threads(int(threads))

    def init(self):
        rc = lib().ref_init(self.h)
        assert rc == 0, rc

    def run(self, t_stop=np.inf, max_incs=0):
        return lib().ref_run(self.h, float(t_stop), int(max_incs))

    def solve_native(self):
        return lib().ref_solve_native(self.h)

    def control(self):
        out = np.zeros(3)
        lib().ref_control(self.h, _pd(out))
        return dict(time=out[0], time_step=out[1], increment=int(out[2]))

    def nodes(self, field):
        out = np.zeros((self.desc.n_nodes, 3))
        rc = lib().ref_get_nodes(self.h, field, _pd(out))
        assert rc == 0
        return out

    def set_nodes(self, field, values):
        a = np.ascontiguousarray(values, dtype=np.float64).reshape(self.desc.n_nodes, 3)
        assert lib().ref_set_nodes(self.h, field, _pd(a)) == 0

    def ips(self):
        out = np.zeros((_abi.IP_NCOMP, self.desc.n_ips))
        assert lib().ref_get_ips(self.h, _pd(out)) == 0
        return out

    def set_ips(self, values):
        a = np.ascontiguousarray(values, dtype=np.float64).reshape(_abi.IP_NCOMP, self.desc.n_ips)
        assert lib().ref_set_ips(self.h, _pd(a)) == 0

    def element_pass(self, dt):
        assert lib().ref_element_pass(self.h, float(dt)) == 0

    def point_kinematics(self, q):
        """StrainInc (6) and R (3x3) of point q after the last element pass."""
        out = np.zeros(15)
        assert lib().ref_point_kinematics(self.h, int(q), _pd(out)) == 0
        return out[:6], out[6:].reshape(3, 3)

    def rotation_orthogonality(self):
        """(max |R^T R - I| over the points after the last element pass, that point)."""
        out = np.zeros(2)
        assert lib().ref_rotation_orthogonality(self.h, _pd(out)) == 0
        return out[0], int(out[1])

    def courant(self):
        return lib().ref_courant(self.h)

    def element_lengths(self):
        ln = np.zeros(self.desc.n_elems)
        wv = np.zeros(self.desc.n_elems)
        lib().ref_element_lengths(self.h, _pd(ln), _pd(wv))
        return ln, wv

    @property
    def workdir(self):
        """Directory where the reference writes its files (ref000.vtk, ...)."""
        return self._tmp

    def enable_vtk(self, start, end, inc):
        """The reference's own result files at its save times (written in
        `workdir` by its Explicit::endStep during run()), the initial one now.
        Their fields come from the reference's settings file when the model
        was created with DNL_REF_SETTINGS set."""
        assert lib().ref_enable_vtk(self.h, float(start), float(end), float(inc)) == 0

    def write_final_vtk(self):
        assert lib().ref_write_final_vtk(self.h) == 0

    def solver_seconds(self):
        return lib().ref_solver_seconds(self.h)

    def timer(self, name):
        return lib().ref_timer(self.h, name.encode())

    def close(self):
        if self.h:
            lib().ref_destroy(self.h)
            self.h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()
