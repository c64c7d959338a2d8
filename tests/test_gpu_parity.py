"""Parity of the CUDA engine (through the C ABI) with the oracle and with the
reference's golden fixtures.

Tolerances: the FP64 path must agree with the FP64 oracle within 1e-6 relative
on internal forces and returned stresses of one element pass (we assert much
tighter bounds where the arithmetic allows); the mixed path (FP32 element math
and point state, FP64 positions/displacements/time/energy sums) is held to
MIXED_PASS_RTOL on one pass and to 1e-4 on final bar length / radius and 1e-3
on the maximum equivalent plastic strain of a whole Taylor run."""
import glob
import os

import numpy as np
import pytest

import helpers
from helpers import _abi, meshes
import oracle

pytestmark = pytest.mark.gpu

RUNS = sorted(glob.glob(os.path.join(helpers.GOLDEN, "*_run.npz")))
PASSES = sorted(glob.glob(os.path.join(helpers.GOLDEN, "*_pass.npz")))


def engine(desc):
    from dnlPython.engine import Engine
    return Engine(desc)


@pytest.mark.parametrize("path", PASSES, ids=[os.path.basename(p) for p in PASSES])
@pytest.mark.parametrize("precision", [_abi.PREC_FP64, _abi.PREC_MIXED], ids=["fp64", "mixed"])
def test_element_pass_matches_reference(path, precision):
    z = np.load(path)
    desc = helpers.desc_from_npz(z, precision=precision)
    with engine(desc) as e:
        e.init()
        e.set_ips(z["in_ips"])
        e.set_nodes(_abi.NODE_U, z["in_u"])
        e.element_pass(float(z["dt"]))
        errs = helpers.field_errors(e.ips(), z["out_ips"])
        ferr = helpers.rel_err(e.nodes(_abi.NODE_FORCE), z["out_force"])
    if precision == _abi.PREC_FP64:
        assert errs.max() < 1e-9, errs
        assert ferr < 1e-9
        assert max(errs[:6].max(), ferr) < helpers.FP64_PASS_RTOL
    else:
        assert errs.max() < helpers.MIXED_PASS_RTOL, errs
        assert ferr < helpers.MIXED_PASS_RTOL


@pytest.mark.parametrize("seed", [1, 2, 3])
@pytest.mark.parametrize("case", ["hex", "axi"])
def test_element_pass_random_states_vs_oracle(case, seed):
    desc = helpers.case_hex_small() if case == "hex" else helpers.case_axi_small()
    with oracle.OracleModel(desc) as o, engine(desc) as e:
        o.init()
        e.init()
        ips = helpers.random_point_state(desc, o.ips(), seed, stress_scale=150.0 * seed)
        u = helpers.random_increment(desc, seed + 7, strain=1e-3 * seed)
        dt = 4e-9 * seed
        for m in (o, e):
            m.set_ips(ips)
            m.set_nodes(_abi.NODE_U, u)
            m.element_pass(dt)
        assert helpers.field_errors(e.ips(), o.ips()).max() < 1e-9
        assert helpers.rel_err(e.nodes(_abi.NODE_FORCE), o.nodes(_abi.NODE_FORCE)) < 1e-9


@pytest.mark.parametrize("path", RUNS, ids=[os.path.basename(p) for p in RUNS])
def test_fp64_runs_match_reference(path):
    z = np.load(path)
    desc = helpers.desc_from_npz(z, precision=_abi.PREC_FP64)
    with engine(desc) as e:
        e.init()
        assert helpers.rel_err(e.nodes(_abi.NODE_MASS), z["init_mass"]) < 1e-13
        assert abs(e.control()["time_step"] - z["init_control"][1]) < 1e-12 * z["init_control"][1]
        # initial speeds, imposed-speed conditions applied as Model::initSolve does
        assert np.array_equal(e.nodes(_abi.NODE_SPEED), z["init_speed"])
        done = 0
        for k in z["checkpoints"]:
            n = e.run(max_incs=int(k) - done)
            assert n == int(z[f"inc{k}_control"][2]) - done  # the run may reach its end time first
            done = int(z[f"inc{k}_control"][2])
            c = e.control()
            assert c["increment"] == int(z[f"inc{k}_control"][2])
            assert abs(c["time"] - z[f"inc{k}_control"][0]) <= 1e-12 * z[f"inc{k}_control"][0]
            assert helpers.rel_err(e.nodes(_abi.NODE_COORDS), z[f"inc{k}_coords"]) < 1e-12
            assert helpers.rel_err(e.nodes(_abi.NODE_DISP), z[f"inc{k}_disp"]) < 1e-9
            assert helpers.rel_err(e.nodes(_abi.NODE_SPEED), z[f"inc{k}_speed"]) < 1e-8
            errs = helpers.field_errors(e.ips(), z[f"inc{k}_ips"])
            assert errs.max() < 1e-8, errs


@pytest.mark.parametrize("path", RUNS, ids=[os.path.basename(p) for p in RUNS])
def test_mixed_runs_track_reference(path):
    z = np.load(path)
    desc = helpers.desc_from_npz(z, precision=_abi.PREC_MIXED)
    k = int(z["checkpoints"][-1])
    with engine(desc) as e:
        e.init()
        e.run(max_incs=k)
        span = np.ptp(z[f"inc{k}_coords"], axis=0).max()
        assert np.abs(e.nodes(_abi.NODE_COORDS) - z[f"inc{k}_coords"]).max() < 1e-5 * span
        errs = helpers.field_errors(e.ips(), z[f"inc{k}_ips"])
        assert errs[:6].max() < 5e-3, errs
        assert errs[_abi.IP_EPSP] < 1e-3 and errs[_abi.IP_T] < 1e-4


def _taylor_summary(desc, m, nr):
    c = m.nodes(_abi.NODE_COORDS)
    ip = m.ips()
    return dict(radius=c[nr, 0], height=c[desc.n_nodes - 1 - nr, 1], epsp=ip[_abi.IP_EPSP].max(),
                energies=m.energies())


@pytest.fixture(scope="module")
def config0_oracle():
    """Copper Taylor impact, 10 x 80 ElQua4NAx, 227 m/s, 80 us (Courant, every 10 increments)."""
    desc = meshes.taylor_axi(precision=_abi.PREC_FP64)
    with oracle.OracleModel(desc) as o:
        o.init()
        n = o.run()
        return n, _taylor_summary(desc, o, 10), o.nodes(_abi.NODE_COORDS), o.ips()


def test_config0_fp64_whole_run(config0_oracle):
    n_o, s_o, x_o, ip_o = config0_oracle
    desc = meshes.taylor_axi(precision=_abi.PREC_FP64)
    with engine(desc) as e:
        e.init()
        n = e.run()
        s = _taylor_summary(desc, e, 10)
        assert n == n_o and e.control()["done"]
        assert helpers.rel_err(e.nodes(_abi.NODE_COORDS), x_o) < 1e-9
        assert helpers.field_errors(e.ips(), ip_o).max() < 1e-6
        assert abs(s["height"] - s_o["height"]) < 1e-9 * s_o["height"]
        assert np.allclose(s["energies"], s_o["energies"], rtol=1e-9)


def test_config0_mixed_whole_run(config0_oracle):
    n_o, s_o, x_o, ip_o = config0_oracle
    desc = meshes.taylor_axi(precision=_abi.PREC_MIXED)
    with engine(desc) as e:
        e.init()
        e.run()
        s = _taylor_summary(desc, e, 10)
        c = e.control()
    assert c["done"]
    assert abs(s["height"] - s_o["height"]) < 1e-4 * s_o["height"]
    assert abs(s["radius"] - s_o["radius"]) < 1e-4 * s_o["radius"]
    assert abs(s["epsp"] - s_o["epsp"]) < 1e-3 * s_o["epsp"]
    assert np.allclose(s["energies"], s_o["energies"], rtol=1e-3)


def test_batched_instances_match_single_runs():
    descs = [helpers.case_hex_small(), helpers.case_hex_small().copy(t_end=3e-6),
             meshes.hex_block(2, 3, 2, speed=90000.0, seed=4, distort=0.05, t_end=6e-6)]
    descs[1].materials[0]["A"] *= 1.1
    # the same element-pass variant alone and in the batch (a batch starts on
    # a persistent variant; the arithmetic of one variant is the same in both)
    with engine(descs) as b:
        variant = b.variant()[0]
    singles = []
    for d in descs:
        with engine(d) as e:
            e.init()
            e.set_variant(variant)
            e.run()
            singles.append((e.nodes(_abi.NODE_COORDS), e.ips(), e.control()))
    with engine(descs) as b:
        b.init()
        b.run()
        X, IP = b.nodes(_abi.NODE_COORDS), b.ips()
        for i, (x, ip, c) in enumerate(singles):
            n0, e0, q0 = b.offsets(i)
            n1, e1, q1 = b.offsets(i + 1) if i + 1 < len(descs) else (b.n_nodes, b.n_elems, b.n_ips)
            assert np.array_equal(X[n0:n1], x)
            assert np.array_equal(IP[:, q0:q1], ip)
            cb = b.control(i)
            assert cb["increment"] == c["increment"] and cb["time"] == c["time"]


@pytest.mark.parametrize("precision", [_abi.PREC_FP64, _abi.PREC_MIXED], ids=["fp64", "mixed"])
def test_history_items_equal_full_reads(precision):
    """dnl_engine_gather_items returns, item after item, exactly what the full
    reads of the nodal fields and the point state hold, and the kinetic
    energy of both speed fields; a batch's instances are kept apart."""
    descs = [helpers.case_hex_small(precision), helpers.case_hex_small(precision).copy(t_end=3e-6)]
    with engine(descs) as e:
        e.init()
        e.run(max_incs=25)
        n1, _, q1 = e.offsets(1)
        fields = (_abi.NODE_COORDS, _abi.NODE_DISP, _abi.NODE_U, _abi.NODE_SPEED, _abi.NODE_ACCEL,
                  _abi.NODE_MASS, _abi.NODE_SPEED_PREV)
        items = [(_abi.ITEM_NODE, f, i) for f in fields for i in (0, 3, n1, e.n_nodes - 1)]
        items += [(_abi.ITEM_POINT, 0, q) for q in (0, 7, q1 + 2, e.n_ips - 1)]
        items += [(_abi.ITEM_KINETIC, f, k) for f in (_abi.NODE_SPEED, _abi.NODE_SPEED_PREV) for k in (0, 1)]
        n = e.set_items(items)
        assert n == sum(_abi.ITEM_WIDTH[k] for k, _, _ in items)
        got = e.gather_items()
        ips = e.ips()
        want = []
        for kind, f, i in items:
            if kind == _abi.ITEM_NODE:
                want.extend(e.nodes(f)[i])
            elif kind == _abi.ITEM_POINT:
                want.extend(ips[:, i])
            else:
                n0, _, _ = e.offsets(i)
                n_end = e.offsets(i + 1)[0] if i + 1 < e.n_instances else e.n_nodes
                v, m = e.nodes(f)[n0:n_end], e.nodes(_abi.NODE_MASS)[n0:n_end, 0]
                want.append(np.sum(m * (v * v).sum(1) / 2.0))
        want = np.array(want)
        nk = 4
        assert np.array_equal(got[:-nk], want[:-nk])
        assert np.allclose(got[-nk:], want[-nk:], rtol=1e-13, atol=0)
        assert got[-nk] > 0
        with pytest.raises(_abi.EngineError):
            e.set_items([(_abi.ITEM_POINT, 0, e.n_ips)])


def test_runs_are_deterministic():
    d = helpers.case_hex_small(_abi.PREC_MIXED)
    out = []
    for _ in range(2):
        with engine(d) as e:
            e.init()
            e.run(max_incs=40)
            out.append((e.nodes(_abi.NODE_COORDS), e.ips()))
    assert np.array_equal(out[0][0], out[1][0]) and np.array_equal(out[0][1], out[1][1])


def test_pause_and_resume_equal_one_run():
    d = helpers.case_hex_speed()
    with engine(d) as a, engine(d) as b:
        a.init()
        b.init()
        a.run(max_incs=50)
        t_half = b.control()["time"] + 20 * b.control()["time_step"]
        b.run(t_pause=t_half)
        b.run(max_incs=50 - b.control()["increment"])
        assert a.control()["increment"] == b.control()["increment"] == 50
        assert np.array_equal(a.nodes(_abi.NODE_COORDS), b.nodes(_abi.NODE_COORDS))


@pytest.mark.parametrize("ts_freq,precision", [(10, _abi.PREC_FP64), (3, _abi.PREC_FP64), (2, _abi.PREC_MIXED),
                                                (1, _abi.PREC_FP64), (10, _abi.PREC_MIXED)])
def test_graph_replays_equal_kernel_by_kernel(ts_freq, precision):
    """Graph replays of several lengths, the graphs of the remaining
    increments of a counted run, and runs cut into uneven pieces (each piece
    starting at another increment of the time-step cycle) give the same bits
    as the same increments launched kernel by kernel."""
    d = helpers.case_hex_speed().copy(ts_freq=ts_freq, precision=precision)
    with engine(d) as ref:
        ref.init()
        ref.set_timing(True)
        ref.run(max_incs=61)
        want = (ref.nodes(_abi.NODE_COORDS), ref.ips(), ref.control()["time"])
    for graph_incs, pieces in ((8, [61]), (8, [1, 2, 3, 7, 9, 10, 11, 18]), (1, [5, 56]), (16, [13, 27, 21]),
                               (20, [30, 31])):
        with engine(d) as e:
            e.init()
            e.set_graph_increments(graph_incs)
            for n in pieces:
                assert e.run(max_incs=n) == n
            got = (e.nodes(_abi.NODE_COORDS), e.ips(), e.control()["time"])
            assert e.control()["increment"] == 61 and e.control()["status"] == 0
        assert np.array_equal(got[0], want[0]), (graph_incs, pieces)
        assert np.array_equal(got[1], want[1]), (graph_incs, pieces)
        assert got[2] == want[2]


def test_inverted_element_raises_status():
    d = helpers.case_hex_small()
    with engine(d) as e:
        e.init()
        x = e.nodes(_abi.NODE_COORDS)
        k = d.conn[0]
        x[k[6]] = x[k[0]] - (x[k[6]] - x[k[0]])  # fold element 0 through itself
        e.set_nodes(_abi.NODE_COORDS, x)
        with pytest.raises(_abi.EngineError) as ei:
            e.run(max_incs=3)
        assert ei.value.code == -3
        assert e.control()["status"] == -3


@pytest.mark.parametrize("precision", [_abi.PREC_FP64, _abi.PREC_MIXED], ids=["fp64", "mixed"])
def test_element_variants_agree_and_autotune_keeps_state(precision):
    """Every element-pass variant the autotuner may pick (register budgets,
    plain or bulk-copy-staged tiles) computes the same increments (to the
    rounding of the compiler's fused multiply-add choices), and autotuning
    leaves the simulation state untouched."""
    d = meshes.taylor_3d(n_core=4, n_ring=3, n_axial=40, precision=precision)
    results = []
    for v in range(_abi.NUM_VARIANTS):
        with engine(d) as e:
            e.init()
            e.set_variant(v)
            e.run(max_incs=25)
            results.append((e.nodes(_abi.NODE_COORDS), e.ips()))
    xtol, iptol = (1e-12, 1e-8) if precision == _abi.PREC_FP64 else (1e-7, 1e-3)
    for x, ip in results[1:]:
        ex, eip = helpers.rel_err(x, results[0][0]), helpers.field_errors(ip, results[0][1]).max()
        assert ex < xtol and eip < iptol, (ex, eip)
    with engine(d) as e:
        e.init()
        e.run(max_incs=5)
        before = (e.nodes(_abi.NODE_COORDS), e.ips(), e.control())
        v, ms = e.autotune(steps=3)
        assert 0 <= v < _abi.NUM_VARIANTS and (ms > 0).all()
        assert np.array_equal(e.nodes(_abi.NODE_COORDS), before[0]) and np.array_equal(e.ips(), before[1])
        assert e.control()["increment"] == before[2]["increment"]
        e.run(max_incs=20)
        assert helpers.rel_err(e.nodes(_abi.NODE_COORDS), results[0][0]) < xtol


@pytest.mark.parametrize("precision", [_abi.PREC_FP64, _abi.PREC_MIXED], ids=["fp64", "mixed"])
def test_power_iteration_taylor_axi_sample(precision):
    """The reference's Taylor-Axi sample with its power-iteration time step
    (Samples/Taylor/Taylor-Axi/Taylor.py:115-118) against the compiled
    reference's final height, radius and plastic strain."""
    rows = np.load(os.path.join(helpers.GOLDEN, "taylor_axi_sample.npz"))["rows"]
    row = rows[rows[:, 0] == _abi.TS_POWER_ITERATION][0]
    d = meshes.taylor_axi(nr=5, nz=50, radius=3.2, length=32.4, speed=287000.0, mat=meshes.STEEL_42CRMO4,
                          t_end=80e-6, ts_method=_abi.TS_POWER_ITERATION, ts_freq=1, precision=precision)
    with engine(d) as e:
        e.init()
        n = e.run()
        c = e.nodes(_abi.NODE_COORDS)
        epsp = e.ips()[_abi.IP_EPSP].reshape(-1, 4).mean(1).max()
    if precision == _abi.PREC_FP64:
        assert n == int(row[2])
        assert abs(c[5, 0] - row[3]) < 1e-9 * row[3] and abs(c[d.n_nodes - 6, 1] - row[4]) < 1e-9 * row[4]
        assert abs(epsp - row[5]) < 1e-8
    else:
        assert abs(c[5, 0] - row[3]) < 1e-4 * row[3] and abs(c[d.n_nodes - 6, 1] - row[4]) < 1e-4 * row[4]
        assert abs(epsp - row[5]) < 1e-3 * row[5]


@pytest.mark.parametrize("case", ["hex", "plane"])
def test_power_iteration_vs_oracle(case):
    base = helpers.case_hex_small() if case == "hex" else helpers.case_plane_small()
    desc = base.copy(ts_method=_abi.TS_POWER_ITERATION, ts_freq=2)
    with oracle.OracleModel(desc) as o, engine(desc) as e:
        o.init()
        e.init()
        assert abs(e.control()["time_step"] - o.control()["time_step"]) < 1e-12 * o.control()["time_step"]
        o.run(max_incs=30)
        e.run(max_incs=30)
        assert abs(e.control()["time_step"] - o.control()["time_step"]) < 1e-11 * o.control()["time_step"]
        assert helpers.rel_err(e.nodes(_abi.NODE_COORDS), o.nodes(_abi.NODE_COORDS)) < 1e-12


@pytest.mark.parametrize("precision", [_abi.PREC_FP64, _abi.PREC_MIXED], ids=["fp64", "mixed"])
def test_native_state_read_equals_widened(precision):
    """dnl_engine_get_ips_native gives the point state in the engine's own
    precision: widened, it equals dnl_engine_get_ips; the other word size is
    refused."""
    d = helpers.case_hex_small(precision)
    with engine(d) as e:
        e.init()
        e.run(max_incs=15)
        nat = e.ips_native()
        assert nat.dtype == (np.float32 if precision == _abi.PREC_MIXED else np.float64)
        assert np.array_equal(nat.astype(np.float64), e.ips())
        other = np.empty(nat.shape, np.float64 if precision == _abi.PREC_MIXED else np.float32)
        assert e._lib.dnl_engine_get_ips_native(e.h, other.ctypes.data, other.dtype.itemsize) == -1


def test_history_ring_equals_stopping_at_each_increment():
    """dnl_engine_set_history keeps the records on the device while the run
    goes on; they equal, bit for bit, what a run stopped after every
    increment gathers when the save rule of HistoryFile::save
    (HistoryFile.C:292-317) is due: same increments, times, masks, time steps
    and item values (nodes of both buffers, points, kinetic energies)."""
    d = helpers.case_hex_speed()
    t_end = d.t_end
    sched = [(0.0, 0.0, t_end / 7), (0.0, 0.0, 0.0), (0.3 * t_end, 0.3 * t_end, t_end / 5)]
    fields = (_abi.NODE_COORDS, _abi.NODE_SPEED, _abi.NODE_SPEED_PREV, _abi.NODE_U_PREV, _abi.NODE_ACCEL_PREV)
    items = [(_abi.ITEM_NODE, f, i) for f in fields for i in (0, 17, d.n_nodes - 1)]
    items += [(_abi.ITEM_POINT, 0, q) for q in (0, 33, d.n_ips - 1)]
    items += [(_abi.ITEM_KINETIC, f, 0) for f in (_abi.NODE_SPEED, _abi.NODE_SPEED_PREV)]
    with engine(d) as a:
        a.init()
        a.set_items(items)
        a.set_history(sched, capacity=16)
        a.run()
        rec = a.history_records()
    want = []
    nxt = [s[1] for s in sched]
    with engine(d) as b:
        b.init()
        b.set_items(items)
        while not b.control()["done"]:
            b.run(max_incs=1)
            c = b.control()
            mask = 0
            for j, (start, _, save) in enumerate(sched):
                if not (c["time"] > start and c["time"] < nxt[j]):
                    nxt[j] += save
                    mask |= 1 << j
            if mask:
                want.append((c["time"], c["increment"], c["last_time_step"], mask, b.gather_items()))
    assert len(rec) == len(want) > 20
    for (t, inc, dt, mask, vals), (wt, winc, wdt, wmask, wvals) in zip(rec, want):
        assert (t, inc, dt, mask) == (wt, winc, wdt, wmask)
        assert np.array_equal(vals, wvals)


def test_engine_rotation_accurate_at_nearly_repeated_stretches():
    """On the element where the reference's rotation is not orthogonal
    (tests/golden/polar_defect_element.npz, see test_oracle.py), the
    engine's FP64 element pass equals the C restatement's (accurate polar
    decomposition), not the reference's."""
    z = np.load(os.path.join(helpers.GOLDEN, "polar_defect_element.npz"))
    d = _abi.ModelDesc(_abi.ELHEX8N3D, z["coords"], np.arange(8)[None], [meshes.COPPER], t_end=1e-6)
    with oracle.OracleModel(d) as o, engine(d) as e:
        o.init()
        e.init()
        for m in (o, e):
            m.set_ips(z["ips"])
            m.set_nodes(_abi.NODE_U, z["u"])
            m.element_pass(float(z["dt"]))
        assert helpers.field_errors(e.ips(), o.ips()).max() < 1e-9
        assert helpers.rel_err(e.nodes(_abi.NODE_FORCE), o.nodes(_abi.NODE_FORCE)) < 1e-9
