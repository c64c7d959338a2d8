"""Node renumbering for gather locality (DNL_ORDER_*, csrc/mesh_order.cpp).

The engine may number its own copy of the nodes by reverse Cuthill-McKee;
every node index and node array of the C ABI stays in the caller's numbering.
The element order, and with it each node's assembly order (the reference's
element loop, Model.C:800-899), does not change, so the results are the same
bits up to the node permutation: only sums over all nodes (the energies) may
round differently.

CPU: the ordering is a permutation, recovers the span of a structured
numbering from a shuffled one, and rejects invalid meshes.  GPU: a shuffled
mesh run with the engine's renumbering, without it, and the unshuffled mesh
give identical nodal fields, point states, node averages, history items and
result files.
"""
import os

import numpy as np
import pytest

import helpers
from helpers import _abi, meshes


def shuffled(desc, seed):
    """The same model with its nodes renumbered at random: node i becomes p[i]."""
    p = np.random.default_rng(seed).permutation(desc.n_nodes).astype(np.int32)

    def perm(a):
        if a is None:
            return None
        out = np.empty_like(a)
        out[p] = a
        return out

    return desc.copy(coords=perm(desc.coords), conn=p[desc.conn], v_init=perm(desc.v_init),
                     bc_code=perm(desc.bc_code), bc_value=perm(desc.bc_value), bc_func=perm(desc.bc_func)), p


def test_rcm_is_a_permutation_that_restores_locality():
    d = meshes.hex_block(12, 10, 8, seed=3, distort=0.1)
    given = _abi.mesh_span(d.conn, d.n_nodes)
    s, _ = shuffled(d, 5)
    assert _abi.mesh_span(s.conn, s.n_nodes) > 5 * given
    order = _abi.mesh_order_rcm(s.conn, s.n_nodes)
    assert np.array_equal(np.sort(order), np.arange(s.n_nodes))
    rcm = _abi.mesh_span(s.conn, s.n_nodes, order)
    # a structured block's lexicographic span is about one cross-section; RCM's
    # level sets are diagonal cross-sections, somewhat wider
    assert rcm < 2.0 * given
    # the given numbering is the identity ordering
    assert _abi.mesh_span(d.conn, d.n_nodes, np.arange(d.n_nodes)) == given


def test_rcm_numbers_every_part_and_isolated_nodes():
    a = meshes.hex_block(3, 3, 3)
    b = meshes.hex_block(2, 2, 2)
    n = a.n_nodes + b.n_nodes + 2  # two nodes in no element
    conn = np.vstack([a.conn, b.conn + a.n_nodes])
    order = _abi.mesh_order_rcm(conn, n)
    assert np.array_equal(np.sort(order), np.arange(n))
    # each part is numbered as one contiguous run
    rank = np.empty(n, dtype=np.int64)
    rank[order] = np.arange(n)
    ra, rb = rank[: a.n_nodes], rank[a.n_nodes: a.n_nodes + b.n_nodes]
    assert ra.max() - ra.min() == a.n_nodes - 1 and rb.max() - rb.min() == b.n_nodes - 1


def test_invalid_meshes_are_rejected():
    d = meshes.hex_block(2, 2, 2)
    bad = d.conn.copy()
    bad[0, 0] = d.n_nodes
    with pytest.raises(_abi.EngineError):
        _abi.mesh_order_rcm(bad, d.n_nodes)
    with pytest.raises(_abi.EngineError):
        _abi.mesh_span(d.conn, d.n_nodes, np.zeros(d.n_nodes, dtype=np.int32))  # not a permutation


def _run(desc, incs, tmpdir, tag):
    from dnlPython.engine import Engine
    e = Engine(desc).init()
    e.run(max_incs=incs)
    out = {f: e.nodes(f) for f in (_abi.NODE_COORDS, _abi.NODE_DISP, _abi.NODE_U, _abi.NODE_SPEED,
                                   _abi.NODE_ACCEL, _abi.NODE_MASS, _abi.NODE_FORCE, _abi.NODE_SPEED_PREV)}
    out["ips"] = e.ips()
    out["avg"] = e.node_averages([_abi.IP_EPSP, _abi.NODE_AVG_VON_MISES, _abi.IP_PRESSURE])
    out["energies"] = np.array(e.energies())
    out["order"] = e.node_order()
    path = os.path.join(str(tmpdir), f"{tag}.vtk")
    e.write_vtk(path, ["speed", "vonMises", "Stress", "plasticStrain"])
    out["vtk"] = open(path).read()
    out["time"] = e.control()["time"]
    e.close()
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [_abi.PREC_FP64, _abi.PREC_MIXED])
def test_renumbered_engine_gives_the_same_bits(tmp_path, precision):
    base = meshes.hex_block(10, 12, 8, size=(0.9, 1.2, 0.9), speed=60000.0, seed=11, distort=0.1, t_end=5e-6,
                            precision=precision, ts_freq=3)
    d = helpers.case_hex_speed(precision)  # imposed speeds with a time function, restrained face
    for k, desc in enumerate((base, d)):
        s, p = shuffled(desc, 7 + k)
        ref = _run(desc, 40, tmp_path, f"ref{k}")
        plain = _run(s.copy(node_order=_abi.ORDER_GIVEN), 40, tmp_path, f"plain{k}")
        rcm = _run(s.copy(node_order=_abi.ORDER_RCM), 40, tmp_path, f"rcm{k}")
        auto = _run(s.copy(node_order=_abi.ORDER_AUTO), 40, tmp_path, f"auto{k}")
        assert ref["order"] == _abi.ORDER_GIVEN and plain["order"] == _abi.ORDER_GIVEN
        assert rcm["order"] == _abi.ORDER_RCM and auto["order"] == _abi.ORDER_RCM
        for r in (plain, rcm, auto):
            assert r["time"] == ref["time"]
            for f in (_abi.NODE_COORDS, _abi.NODE_DISP, _abi.NODE_U, _abi.NODE_SPEED, _abi.NODE_ACCEL,
                      _abi.NODE_MASS, _abi.NODE_FORCE, _abi.NODE_SPEED_PREV):
                assert np.array_equal(r[f][p], ref[f]), f
            assert np.array_equal(r["ips"], ref["ips"])
            assert np.array_equal(r["avg"][:, p], ref["avg"])
            np.testing.assert_allclose(r["energies"], ref["energies"], rtol=1e-12, atol=0)
        # the result files list the nodes in the caller's numbering, so the
        # shuffled runs write the same file whatever the engine's numbering
        assert rcm["vtk"] == plain["vtk"] == auto["vtk"]


@pytest.mark.gpu
def test_renumbered_engine_items_and_writes_follow_the_callers_numbering():
    from dnlPython.engine import Engine
    desc = meshes.hex_block(6, 8, 5, speed=60000.0, seed=2, distort=0.1, t_end=5e-6, ts_freq=3)
    s, p = shuffled(desc, 3)
    nodes = [0, 17, desc.n_nodes - 1]
    vals = []
    for order in (_abi.ORDER_GIVEN, _abi.ORDER_RCM):
        e = Engine(s.copy(node_order=order)).init()
        e.set_items([(_abi.ITEM_NODE, _abi.NODE_COORDS, int(p[n])) for n in nodes] +
                    [(_abi.ITEM_NODE, _abi.NODE_SPEED_PREV, int(p[n])) for n in nodes] +
                    [(_abi.ITEM_KINETIC, _abi.NODE_SPEED, 0)])
        # a write in the caller's numbering lands on the caller's node
        v = e.nodes(_abi.NODE_SPEED)
        v[p[nodes[1]]] = (1.0, 2.0, 3.0)
        e.set_nodes(_abi.NODE_SPEED, v)
        assert np.array_equal(e.nodes(_abi.NODE_SPEED), v)
        e.run(max_incs=10)
        vals.append(e.gather_items())
        e.close()
    np.testing.assert_array_equal(vals[0][:-1], vals[1][:-1])
    np.testing.assert_allclose(vals[0][-1], vals[1][-1], rtol=1e-12)
