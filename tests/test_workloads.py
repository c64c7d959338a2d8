"""The measured workloads as whole runs: the 3-D copper Taylor bar run to its
end time (mixed path against the FP64 path, the whole-run reference at a size
where the CPU oracle would take hours; the FP64 path itself is held to the
oracle on every smaller case), and batches of independent Taylor bars
(generator, instances that fail alone, finished instances skipped)."""
import numpy as np
import pytest

import helpers
from helpers import _abi, meshes


def engine(desc):
    from dnlPython.engine import Engine
    return Engine(desc)


def bar_results(desc, coords, ips):
    """Final bar length (highest node), foot radius (largest distance to the
    axis on the impact face) and maximum equivalent plastic strain."""
    face = desc.coords[:, 1] == 0.0
    if desc.elem_type == _abi.ELHEX8N3D:
        foot = np.sqrt(coords[face, 0] ** 2 + coords[face, 2] ** 2).max()
    else:
        foot = coords[face, 0].max()
    return coords[:, 1].max(), foot, ips[_abi.IP_EPSP].max()


def test_taylor_batch_generator():
    a = meshes.taylor_batch(n=32, seed=7)
    b = meshes.taylor_batch(n=32, seed=7)
    e = np.array([d.n_elems for d in a])
    assert np.array_equal(e, [d.n_elems for d in b])
    assert e.min() >= 1900 and e.max() <= 62000
    v = np.array([-d.v_init[0, 1] for d in a])
    assert v.min() >= 150000.0 and v.max() <= 300000.0
    for d in a:
        for k in ("A", "B", "n", "C", "m"):
            assert 0.8 - 1e-12 <= d.materials[0][k] / meshes.COPPER[k] <= 1.2 + 1e-12
        assert d.materials[0]["young"] == meshes.COPPER["young"]
    full = meshes.taylor_batch()
    tot = sum(d.n_elems for d in full)
    assert len(full) == 256 and 4.0e6 < tot < 5.2e6


@pytest.mark.gpu
@pytest.mark.parametrize("variant", [0, 2], ids=["plain", "bulk-copy"])
def test_batch_failed_instance_stops_alone(variant):
    """An instance whose element inverts stops with its status; the other
    instances of the batch run to their end exactly as they do alone."""
    good = meshes.hex_block(2, 3, 2, speed=90000.0, seed=4, distort=0.05, t_end=6e-6)
    bad = helpers.case_hex_small()
    with engine(good) as e:
        e.init()
        e.set_variant(variant)
        e.run()
        x_ref, ip_ref, c_ref = e.nodes(_abi.NODE_COORDS), e.ips(), e.control()
    with engine([bad, good]) as b:
        b.init()
        b.set_variant(variant)
        x = b.nodes(_abi.NODE_COORDS)
        k = bad.conn[0]
        x[k[6]] = x[k[0]] - (x[k[6]] - x[k[0]])
        b.set_nodes(_abi.NODE_COORDS, x)
        b.run(check=False)
        assert b.control(0)["status"] == _abi.DNL_ERR_NEG_JACOBIAN
        c = b.control(1)
        assert c["status"] == 0 and c["increment"] == c_ref["increment"] and c["time"] == c_ref["time"]
        n0, _, q0 = b.offsets(1)
        assert np.array_equal(b.nodes(_abi.NODE_COORDS)[n0:], x_ref)
        assert np.array_equal(b.ips()[:, q0:], ip_ref)
        with pytest.raises(_abi.EngineError):
            b.run()


@pytest.mark.gpu
@pytest.mark.parametrize("variant", [0, 2], ids=["plain", "bulk-copy"])
def test_batch_of_taylor_bars_matches_single_runs(variant):
    """Bars of uneven size, speed and material in one batch: every instance
    ends bit-identical to its own run (the bars finish at different
    increments, after which their tiles are skipped)."""
    descs = meshes.taylor_batch(n=5, seed=11, elems=(300, 1500), t_end=6e-6)
    with engine(descs) as b:
        b.init()
        b.set_variant(variant)
        b.run()
        X, IP = b.nodes(_abi.NODE_COORDS), b.ips()
        incs = []
        for i, d in enumerate(descs):
            with engine(d) as e:
                e.init()
                e.set_variant(variant)
                e.run()
                n0, _, q0 = b.offsets(i)
                assert np.array_equal(X[n0:n0 + d.n_nodes], e.nodes(_abi.NODE_COORDS))
                assert np.array_equal(IP[:, q0:q0 + d.n_ips], e.ips())
                assert b.control(i)["increment"] == e.control()["increment"]
                incs.append(e.control()["increment"])
    assert len(set(incs)) > 1


@pytest.mark.gpu
def test_taylor3d_whole_run_mixed_against_fp64():
    """The 153,600-element copper bar to 80 us: mixed path within 1e-4 of the
    FP64 path on final length and foot radius, 1e-3 on max plastic strain."""
    out = {}
    for prec in (_abi.PREC_FP64, _abi.PREC_MIXED):
        d = meshes.taylor_3d(precision=prec)
        with engine(d) as e:
            e.init()
            e.run()
            c = e.control()
            assert c["status"] == 0 and c["time"] == pytest.approx(80e-6, rel=1e-12)
            out[prec] = bar_results(d, e.nodes(_abi.NODE_COORDS), e.ips()) + (c["increment"],)
    L64, R64, ep64, n64 = out[_abi.PREC_FP64]
    L, R, ep, n = out[_abi.PREC_MIXED]
    assert abs(L - L64) <= 1e-4 * L64 and abs(R - R64) <= 1e-4 * R64
    assert abs(ep - ep64) <= 1e-3 * ep64
    assert L64 < 0.7 * 32.4 and R64 > 1.8 * 3.2  # a mushroomed bar
