"""The C ABI: the engine library loads and exports every entry point that
include/dnlgpu.h declares, the ctypes layout matches the header, invalid
descriptions are rejected on the host, and without a CUDA device the engine
refuses to run (there is no CPU fallback)."""
import ctypes
import subprocess

import numpy as np
import pytest

import helpers
from helpers import _abi, meshes
import oracle


def test_library_exports_header_symbols():
    lib = _abi.load_library()
    names = _abi.exported_symbols()
    assert len(names) >= 19
    for n in names:
        assert hasattr(lib, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", _abi.LIB_PATH], capture_output=True, text=True).stdout
    for n in names:
        assert f" T {n}" in out, n


def test_struct_layout_matches_header():
    assert ctypes.sizeof(_abi.ModelDescC) == oracle.abi_sizeof(0)
    assert ctypes.sizeof(_abi.Material) == oracle.abi_sizeof(1)
    assert ctypes.sizeof(_abi.Function) == oracle.abi_sizeof(2)
    assert ctypes.sizeof(_abi.Control) == oracle.abi_sizeof(3)


def _create(desc):
    lib = _abi.load_library()
    c = desc.cstruct()
    h = ctypes.c_void_p()
    rc = lib.dnl_engine_create(ctypes.byref(c), ctypes.byref(h))
    return rc, h, lib.dnl_engine_last_error(None).decode()


def test_invalid_descriptions_are_rejected():
    d = helpers.case_hex_small()
    bad = d.copy(conn=np.where(d.conn == 3, d.n_nodes + 5, d.conn))
    rc, h, msg = _create(bad)
    assert rc == -1 and "out of range" in msg
    rc, h, msg = _create(d.copy(t_end=0.0))
    assert rc == -1
    c = d.cstruct()
    c.elem_type = 7
    lib = _abi.load_library()
    h = ctypes.c_void_p()
    assert lib.dnl_engine_create(ctypes.byref(c), ctypes.byref(h)) == -1 and not h
    rc, h, msg = _create(d.copy(ts_method=7))
    assert rc == -6
    rc, h, msg = _create(d.copy(stress_method=5))
    assert rc == -6 and "stress computation" in msg
    rc, h, msg = _create(d.copy(node_order=9))
    assert rc == -1 and "node order" in msg
    # empty and ragged inputs: no elements, no nodes, no material, a material
    # index past the list, an unknown precision; each is refused on the host
    # before any device call and leaves no handle
    for field, value, text in (("n_elems", 0, "empty mesh"), ("n_nodes", 0, "empty mesh"),
                               ("n_materials", 0, "no material"), ("precision", 9, "unknown precision")):
        c = d.cstruct()
        setattr(c, field, value)
        h = ctypes.c_void_p()
        assert lib.dnl_engine_create(ctypes.byref(c), ctypes.byref(h)) == -1 and not h, field
        assert text in lib.dnl_engine_last_error(None).decode(), field
    # beyond the 32-bit point indices (the sizes are refused before the
    # arrays, which here are far shorter, are read)
    for field, value in (("n_elems", 200_000_000), ("n_nodes", 400_000_000)):
        c = d.cstruct()
        setattr(c, field, value)
        h = ctypes.c_void_p()
        assert lib.dnl_engine_create(ctypes.byref(c), ctypes.byref(h)) == -1 and not h, field
        assert "too large for 32-bit point indices" in lib.dnl_engine_last_error(None).decode(), field
    rc, h, msg = _create(d.copy(elem_mat=np.full(d.n_elems, 1, dtype=np.int32)))
    assert rc == -1 and "material index of element 0 out of range" in msg and not h
    rc, h, msg = _create(d.copy(conn=np.where(d.conn == 3, -1, d.conn)))
    assert rc == -1 and "out of range" in msg and not h


def test_no_device_means_no_engine():
    lib = _abi.load_library()
    if lib.dnl_device_count() > 0:
        pytest.skip("a CUDA device is visible")
    rc, h, msg = _create(helpers.case_hex_small())
    assert rc == -7
    from dnlPython.engine import Engine
    with pytest.raises(_abi.EngineUnavailable):
        Engine(helpers.case_hex_small())


def test_config_meshes():
    d = meshes.taylor_3d()
    assert d.n_elems == 153600
    assert d.conn.min() == 0 and d.conn.max() == d.n_nodes - 1
    small = meshes.taylor_3d(n_core=4, n_ring=3, n_axial=5, precision=_abi.PREC_FP64)
    with oracle.OracleModel(small) as o:
        o.init()  # negative Jacobians would fail here
        ips = o.ips()
        assert (ips[_abi.IP_DETJ0] > 0).all()
        vol = ips[_abi.IP_DETJ0].sum()
        assert abs(vol - np.pi * 3.2 ** 2 * 32.4) < 0.05 * vol
    a = meshes.taylor_axi()
    assert a.n_elems == 800 and a.n_nodes == 891
