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
@pytest.mark.parametrize("variant", [0, 2, 6], ids=["plain", "bulk-copy", "staged"])
def test_batch_failed_instance_stops_alone(variant):
    """An instance whose element inverts stops with its status; the other
    instances of the batch run to their end exactly as they do alone."""
    good = meshes.hex_block(2, 3, 2, speed=90000.0, seed=4, distort=0.05, t_end=6e-6)
    bad = helpers.case_hex_small()
    with engine(helpers.with_spare_material(good)) as e:
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
@pytest.mark.parametrize("variant", [0, 2, 6], ids=["plain", "bulk-copy", "staged"])
def test_batch_of_taylor_bars_matches_single_runs(variant):
    """Bars of uneven size, speed and material in one batch: every instance
    ends bit-identical to its own run on the same kernels (the bars finish at
    different increments, after which their tiles are skipped), and within
    the last bits of the point math of its run on the one-material kernels
    (material constants as kernel parameters)."""
    descs = meshes.taylor_batch(n=5, seed=11, elems=(300, 1500), t_end=6e-6)
    with engine(descs) as b:
        b.init()
        b.set_variant(variant)
        b.run()
        X, IP = b.nodes(_abi.NODE_COORDS), b.ips()
        incs = []
        for i, d in enumerate(descs):
            n0, _, q0 = b.offsets(i)
            with engine(helpers.with_spare_material(d)) as e:
                e.init()
                e.set_variant(variant)
                e.run()
                assert np.array_equal(X[n0:n0 + d.n_nodes], e.nodes(_abi.NODE_COORDS))
                assert np.array_equal(IP[:, q0:q0 + d.n_ips], e.ips())
                assert b.control(i)["increment"] == e.control()["increment"]
                incs.append(e.control()["increment"])
            with engine(d) as e:
                e.init()
                e.set_variant(variant)
                e.run()
                x1, ip1 = e.nodes(_abi.NODE_COORDS), e.ips()
                dx = np.abs(x1 - X[n0:n0 + d.n_nodes]).max() / np.abs(x1).max()
                ds = np.abs(ip1 - IP[:, q0:q0 + d.n_ips]).max(axis=1) / np.maximum(np.abs(ip1).max(axis=1), 1e-300)
                print(f"instance {i}: one-material kernels against the batch: coordinates {dx:.2e}, "
                      f"point state {ds.max():.2e} of the field's largest value")
                assert b.control(i)["increment"] == e.control()["increment"]
                assert dx <= 1e-9 and ds.max() <= 1e-4
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


def test_necking_generators():
    b = meshes.bar_necking(n_core=6, n_ring=8, n_axial=30)
    assert b.n_elems == (36 + 4 * 6 * 8) * 30
    face = b.coords[:, 1] == 0.0
    r0 = np.sqrt(b.coords[face, 0] ** 2 + b.coords[face, 2] ** 2).max()
    top = b.coords[:, 1] == b.coords[:, 1].max()
    r1 = np.sqrt(b.coords[top, 0] ** 2 + b.coords[top, 2] ** 2).max()
    assert abs(r0 - 0.99 * 6.413) < 1e-9 and abs(r1 - 6.413) < 1e-9
    assert np.all(b.bc_code[face, 1] == _abi.BC_RESTRAIN) and np.all(b.bc_code[top, 1] == _abi.BC_SPEED)
    # 7 mm of elongation at 5 m/s after a ramp over the first 10% of the run
    assert abs(b.t_end - 7.0 / (5000.0 * 0.95)) < 1e-15
    fx, fy = b.functions[0]
    assert np.interp(0.05 * b.t_end, fx, fy) == pytest.approx(0.5) and np.interp(0.5 * b.t_end, fx, fy) == 1.0
    p = meshes.plate_necking(nx=16, nz=2, ny=40)
    assert p.n_elems == 16 * 2 * 40
    pf = p.coords[:, 1] == 0.0
    assert abs(p.coords[pf, 0].max() - 0.99 * 5.0) < 1e-12
    assert abs(p.coords[:, 2].max() - 0.5) < 1e-12


def neck_radius(desc, coords):
    face = desc.coords[:, 1] == 0.0
    return np.sqrt(coords[face, 0] ** 2 + coords[face, 2] ** 2).max()


@pytest.mark.gpu
def test_bar_necking_matches_oracle():
    """The pulled bar (imposed speed ramped by a discrete function) against the
    oracle over its first increments, FP64."""
    import oracle
    d = meshes.bar_necking(n_core=4, n_ring=4, n_axial=20, precision=_abi.PREC_FP64)
    with oracle.OracleModel(d) as o, engine(d) as e:
        o.init()
        e.init()
        o.run(max_incs=40)
        e.run(max_incs=40)
        assert e.control()["increment"] == o.control()["increment"] == 40
        assert helpers.rel_err(e.nodes(_abi.NODE_COORDS), o.nodes(_abi.NODE_COORDS)) < 1e-12
        assert helpers.field_errors(e.ips(), o.ips()).max() < 1e-8


@pytest.mark.gpu
def test_bar_necking_whole_run_mixed_against_fp64():
    """A 13,680-element bar pulled by 7 mm: the mixed path's neck radius and
    maximum plastic strain against the FP64 path's."""
    out = {}
    for prec in (_abi.PREC_FP64, _abi.PREC_MIXED):
        d = meshes.bar_necking(n_core=6, n_ring=8, n_axial=60, precision=prec)
        with engine(d) as e:
            e.init()
            e.run()
            c = e.control()
            assert c["status"] == 0 and c["time"] == pytest.approx(d.t_end, rel=1e-12)
            out[prec] = (neck_radius(d, e.nodes(_abi.NODE_COORDS)), e.ips()[_abi.IP_EPSP].max())
    (r64, ep64), (r, ep) = out[_abi.PREC_FP64], out[_abi.PREC_MIXED]
    assert r64 < 0.99 * 6.413  # the bar has thinned at the notch
    assert abs(r - r64) <= 1e-4 * r64 and abs(ep - ep64) <= 1e-3 * ep64
