"""The element pass that allocates no device memory (dnl_element_pass_static).

Callers whose device memory is owned by a memory manager of their own, or that
call between stream captures, cannot let a library call cudaMalloc; this entry
point takes every input and output as a caller-owned device array and keeps
its scratch in a static device array.  The test drives it through the C ABI
with device arrays the test allocates, and checks two calls in a row against
the engine's own element pass (dnl_engine_element_pass) on the same state.
This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

import helpers
from helpers import _abi, meshes

pytestmark = pytest.mark.gpu


def _reference_pass(desc, ips, u, dt):
    from dnlPython.engine import Engine
    with Engine(desc) as e:
        e.init()
        x = e.nodes(_abi.NODE_COORDS)
        e.set_ips(ips)
        e.set_nodes(_abi.NODE_U, u)
        e.element_pass(dt)
        return x, e.ips(), e.nodes(_abi.NODE_FORCE)


def _static_pass(desc, coords, u, ips, dt):
    import torch
    lib = _abi.load_library()
    dev = torch.device("cuda", 0)
    d_x = torch.as_tensor(np.ascontiguousarray(coords), device=dev)
    d_u = torch.as_tensor(np.ascontiguousarray(u), device=dev)
    d_conn = torch.as_tensor(np.ascontiguousarray(desc.conn, dtype=np.int32), device=dev)
    d_ip = torch.as_tensor(np.ascontiguousarray(ips), device=dev)
    d_f = torch.zeros((desc.n_nodes, 3), dtype=torch.float64, device=dev)
    keys = [f[0] for f in _abi.Material._fields_]
    mat = _abi.Material(*[float(desc.materials[0][k]) for k in keys])
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = lib.dnl_element_pass_static(desc.elem_type, desc.n_nodes, desc.n_elems, d_x.data_ptr(), d_u.data_ptr(),
                                     d_conn.data_ptr(), ctypes.byref(mat), float(dt), d_ip.data_ptr(),
                                     d_f.data_ptr(), stream)
    assert rc == 0, lib.dnl_engine_last_error(None).decode()
    torch.cuda.synchronize()
    return d_ip.cpu().numpy(), d_f.cpu().numpy()


@pytest.mark.parametrize("case", ["hex", "axi", "ogrid"])
def test_static_pass_matches_engine_pass_twice(case):
    if case == "hex":
        desc = helpers.case_hex_small()
    elif case == "axi":
        desc = helpers.case_axi_small()
    else:
        desc = meshes.taylor_3d(n_core=6, n_ring=4, n_axial=50, precision=_abi.PREC_FP64)
    assert desc.n_elems <= 16384
    from oracle import OracleModel
    u = helpers.random_increment(desc, seed=32, strain=3e-3)
    dt = 9e-9
    with OracleModel(desc) as o:
        o.init()
        ips = helpers.random_point_state(desc, o.ips(), seed=31, stress_scale=250.0)
        # the C oracle's element pass on the same state, increment and time step
        o.set_ips(ips)
        o.set_nodes(_abi.NODE_U, u)
        o.element_pass(dt)
        ip_orc, f_orc = o.ips(), o.nodes(_abi.NODE_FORCE)
    x, ip_ref, f_ref = _reference_pass(desc, ips, u, dt)
    # two calls in a row on the same inputs: the scratch keeps the first call's
    # contents, the second must not see them
    for _ in range(2):
        ip_s, f_s = _static_pass(desc, x, u, ips, dt)
        assert helpers.field_errors(ip_s, ip_ref).max() < 1e-9
        assert helpers.rel_err(f_s, f_ref) < 1e-9
        # and against the oracle, with the bounds of the engine's own parity tests
        assert helpers.field_errors(ip_s, ip_orc).max() < 1e-9
        assert helpers.rel_err(f_s, f_orc) < 1e-9


def test_static_pass_rejects_connectivity_out_of_range():
    """A connectivity entry outside [0, n_nodes) (here n_nodes itself, and -1)
    is caught on the device before any node is read through it: the call
    returns DNL_ERR_ARG and a following call on valid input works."""
    desc = helpers.case_hex_small()
    from oracle import OracleModel
    with OracleModel(desc) as o:
        o.init()
        ips = helpers.random_point_state(desc, o.ips(), seed=41)
    u = helpers.random_increment(desc, seed=42)
    x = desc.coords
    lib = _abi.load_library()
    for bad in (desc.n_nodes, -1):
        conn = desc.conn.copy()
        conn[desc.n_elems // 2, 3] = bad
        with pytest.raises(AssertionError, match="connectivity entry outside"):
            _static_pass(desc.copy(conn=conn), x, u, ips, 5e-9)
        assert "connectivity entry outside" in lib.dnl_engine_last_error(None).decode()
    ip_s, f_s = _static_pass(desc, x, u, ips, 5e-9)
    assert np.isfinite(ip_s).all() and np.abs(f_s).max() > 0


def test_static_pass_rejects_sizes_beyond_its_scratch():
    lib = _abi.load_library()
    mat = _abi.Material(*[1.0] * len(_abi.Material._fields_))
    rc = lib.dnl_element_pass_static(_abi.ELHEX8N3D, 1000, 16385, 1, 1, 1, ctypes.byref(mat), 1e-8, 1, 1, None)
    assert rc == -1
    assert "exceed the static scratch limit" in lib.dnl_engine_last_error(None).decode()
