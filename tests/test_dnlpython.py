"""The dnlPython model API (the drop-in front end): scripts written against
DynELA's SWIG module build the same model description as the generators the
engine is measured on; the reference's own sample scripts, where this checkout
has them, are parsed unchanged (their solve() is intercepted: solving needs a GPU)."""
import os
import runpy
import sys
import types

import numpy as np
import pytest

import helpers
from helpers import _abi, meshes
import dnlPython as dnl
import ref

# the reference's sample scripts (DNL_REFERENCE, else the oracle Makefile's default)
_REF_DIR = ref.reference_dir()
SAMPLES = os.path.join(_REF_DIR, "Samples") if _REF_DIR else ""


def taylor_axi_script(nr=5, nz=50, speed=287000.0, method=None, save_dir=None, precision=None):
    """The Taylor-Axi model written with the DynELA API (the usage of
    Samples/Taylor/Taylor-Axi/Taylor.py): 42CrMo4 steel bar, impact face
    restrained along y, axis restrained along x, initial speed -speed."""
    width, heigh, stop = 3.2, 32.4, 80.0e-6
    model = dnl.DynELA("Taylor")
    if precision:
        model.setPrecision(precision)
    allNS = dnl.NodeSet("NS_All")
    num = 1
    for j in range(nz + 1):
        for i in range(nr + 1):
            model.createNode(num, i * width / nr, j * heigh / nz, 0.0)
            model.add(allNS, num)
            num += 1
    nN = num - 1
    model.setDefaultElement(dnl.Element.ElQua4NAx)
    allES = dnl.ElementSet("ES_All")
    k = 1
    for j in range(nz):
        for i in range(nr):
            n1 = i + j * (nr + 1) + 1
            model.createElement(k, n1, n1 + 1, n1 + nr + 2, n1 + nr + 1)
            model.add(allES, k)
            k += 1
    bottom, axis = dnl.NodeSet("NS_Bottom"), dnl.NodeSet("NS_Axis")
    model.add(bottom, 1, nr + 1)
    model.add(axis, 1, nN, nr + 1)
    law = dnl.JohnsonCookLaw()
    law.setParameters(806.0, 614.0, 0.0089, 0.168, 1.1, 1.0, 1540.0, 20.0)
    steel = dnl.Material("Steel")
    steel.setHardeningLaw(law)
    steel.youngModulus, steel.poissonRatio, steel.density = 206000, 0.3, 7.83e-09
    steel.heatCapacity, steel.taylorQuinney, steel.T0 = 4.6e+08, 0.9, 20.0
    model.add(steel, allES)
    b = dnl.BoundaryRestrain("BC_bottom")
    b.setValue(0, 1, 1)
    model.attachConstantBC(b, bottom)
    a = dnl.BoundaryRestrain("BC_axis")
    a.setValue(1, 0, 1)
    model.attachConstantBC(a, axis)
    s = dnl.BoundarySpeed("BC_speed")
    s.setValue(0, -speed, 0)
    model.attachInitialBC(s, allNS)
    solver = dnl.Explicit("Solver")
    solver.setTimes(0, stop)
    model.add(solver)
    if method is not None:
        solver.setComputeTimeStepFrequency(1)
        solver.setTimeStepMethod(method)
    if save_dir is not None:
        # result files, as the sample script asks for them (Taylor.py:120)
        model.setSaveTimes(0, stop, stop / 10)
        hist = dnl.ElementSet("ES_Hist")
        model.add(hist, 1)
        rad, hei = dnl.NodeSet("NS_R"), dnl.NodeSet("NS_H")
        model.add(rad, 1 + nr)
        model.add(hei, nN - nr)
        for name, target, field in (("radius.plot", rad, dnl.Field.coordsX), ("height.plot", hei, dnl.Field.coordsY),
                                    ("plasticStrain.plot", hist, dnl.Field.plasticStrain)):
            h = dnl.HistoryFile(name)
            h.setFileName(os.path.join(save_dir, name))
            if isinstance(target, dnl.ElementSet):
                h.add(target, 0, field)
            else:
                h.add(target, field)
            h.setSaveTime(stop / 250)
            model.add(h)
        for name, field in (("dt.plot", dnl.Field.timeStep), ("ke.plot", dnl.Field.kineticEnergy)):
            h = dnl.HistoryFile(name)
            h.setFileName(os.path.join(save_dir, name))
            h.add(field)
            h.setSaveTime(stop / 250)
            model.add(h)
    return model, nN


def test_api_model_matches_generator():
    model, _ = taylor_axi_script(method=dnl.Explicit.PowerIteration)
    desc, nodes, elems = model._description()
    ref = meshes.taylor_axi(nr=5, nz=50, radius=3.2, length=32.4, speed=287000.0, mat=meshes.STEEL_42CRMO4,
                            t_end=80e-6, ts_method=_abi.TS_POWER_ITERATION, ts_freq=1)
    assert np.array_equal(desc.conn, ref.conn)
    assert np.allclose(desc.coords, ref.coords, rtol=0, atol=1e-12)
    # plane models carry two components; the z column of a restraint is not read
    assert np.array_equal(desc.bc_code[:, :2], ref.bc_code[:, :2])
    assert np.array_equal(desc.v_init, ref.v_init)
    assert desc.ts_method == ref.ts_method and desc.ts_freq == 1
    for k in ref.materials[0]:
        assert desc.materials[0][k] == pytest.approx(ref.materials[0][k])


def test_boundary_resolution_rules():
    """The last constant condition touching a component wins; a speed condition
    imposes only its non-zero components and, as a start condition, sets the
    whole speed vector (BoundaryCondition.C:131-190, BoundarySpeed.C:63-206)."""
    model = dnl.DynELA("bc")
    for n in range(1, 9):
        model.createNode(n, (n - 1) & 1, ((n - 1) >> 1) & 1, (n - 1) >> 2)
    model.setDefaultElement(dnl.Element.ElHex8N3D)
    model.createElement(1, 1, 2, 4, 3, 5, 6, 8, 7)
    es = dnl.ElementSet("E")
    model.add(es, 1)
    m = dnl.Material("m")
    law = dnl.JohnsonCookLaw()
    law.setParameters(1, 1, 0, 0.5, 1, 1, 1000, 0)
    m.setHardeningLaw(law)
    m.youngModulus, m.poissonRatio, m.density, m.heatCapacity, m.taylorQuinney = 1e5, 0.3, 1e-8, 1e8, 0.9
    model.add(m, es)
    ns = dnl.NodeSet("N")
    model.add(ns, 1, 2)
    r = dnl.BoundaryRestrain("r")
    r.setValue(1, 1, 0)
    sp = dnl.BoundarySpeed("s")
    sp.setValue(0, 5.0, 0)
    model.attachConstantBC(r, ns)
    model.attachConstantBC(sp, ns)
    init = dnl.BoundarySpeed("i")
    init.setValue(1.0, 2.0, 3.0)
    model.attachInitialBC(init, ns)
    solver = dnl.Explicit("S")
    solver.setTimes(0, 1e-6)
    model.add(solver)
    desc, _, _ = model._description()
    assert list(desc.bc_code[0]) == [_abi.BC_RESTRAIN, _abi.BC_SPEED, _abi.BC_FREE]
    assert desc.bc_value[0, 1] == 5.0
    assert list(desc.v_init[0]) == [0.0, 5.0, 0.0]  # the constant speed condition's vector, applied last
    assert list(desc.bc_code[4]) == [0, 0, 0]


def _one_hex(speed=True):
    model = dnl.DynELA("bc")
    for n in range(1, 9):
        model.createNode(n, (n - 1) & 1, ((n - 1) >> 1) & 1, (n - 1) >> 2)
    model.setDefaultElement(dnl.Element.ElHex8N3D)
    model.createElement(1, 1, 2, 4, 3, 5, 6, 8, 7)
    es = dnl.ElementSet("E")
    model.add(es, 1)
    m = dnl.Material("m")
    law = dnl.JohnsonCookLaw()
    law.setParameters(1, 1, 0, 0.5, 1, 1, 1000, 0)
    m.setHardeningLaw(law)
    m.youngModulus, m.poissonRatio, m.density, m.heatCapacity, m.taylorQuinney = 1e5, 0.3, 1e-8, 1e8, 0.9
    model.add(m, es)
    ns = dnl.NodeSet("N")
    model.add(ns, 1, 4)
    if speed:
        sp = dnl.BoundarySpeed("s")
        sp.setValue(0, 5.0, 0)
        model.attachConstantBC(sp, ns)
    solver = dnl.Explicit("S")
    solver.setTimes(0, 1e-6)
    model.add(solver)
    return model, ns


def _same_desc(a, b):
    for k in ("coords", "conn", "v_init", "bc_code", "bc_value", "bc_func"):
        assert np.array_equal(getattr(a, k), getattr(b, k)), k


def test_other_boundary_types():
    """The boundary types other than restraint and speed behave on the explicit
    path as in the reference: acceleration, temperature, convection and flux
    change nothing, as initial or constant conditions; displacement and force
    change nothing as initial conditions and stop the solve as constant ones
    (BoundaryAcceleration.C:54-70, BoundaryTemperature.C:73-93,
    BoundaryConvection.C:85-103, BoundaryFlux.C:73-95,
    BoundaryDisplacement.C:62-76, BoundaryForce.C:61-65, Boundary.h:62)."""
    plain, _ = _one_hex()
    ref = plain._description()[0]
    acc = dnl.BoundaryAcceleration("a")
    acc.setValue(1.0, 2.0, 3.0)
    temp = dnl.BoundaryTemperature("t")
    temp.setValue(500.0)
    conv = dnl.BoundaryConvection("c")
    conv.setValue(10.0, 300.0)
    flux = dnl.BoundaryFlux("f")
    flux.setValue(1e3)
    disp = dnl.BoundaryDisplacement("d")
    disp.setValue(0.1, 0.0, 0.0)
    force = dnl.BoundaryForce("F")
    force.setValue(dnl.Vec3D(0.0, 0.0, 7.0))
    for b in (acc, temp, conv, flux):
        for attach in ("attachConstantBC", "attachInitialBC"):
            model, ns = _one_hex()
            getattr(model, attach)(b, ns)
            _same_desc(model._description()[0], ref)
    for b in (disp, force):
        model, ns = _one_hex()
        model.attachInitialBC(b, ns)
        _same_desc(model._description()[0], ref)
        model, ns = _one_hex()
        model.attachConstantBC(b, ns)
        with pytest.raises(RuntimeError):
            model._description()
        # a condition on an empty set is never applied
        model, _ = _one_hex()
        empty = dnl.NodeSet("empty")
        model.attachConstantBC(b, empty)
        _same_desc(model._description()[0], ref)


@pytest.mark.skipif(not SAMPLES or not os.path.isdir(SAMPLES),
                    reason="the reference's Samples/ is not here (set DNL_REFERENCE to its checkout)")
@pytest.mark.parametrize("sample,etype,count", [
    ("Taylor/Taylor-Axi/Taylor.py", _abi.ELQUA4NAX, 250),
    ("Taylor/Taylor-3D/Taylor.py", _abi.ELHEX8N3D, 4455),
    ("BarNecking/BarNecking-Axi/BarNecking.py", _abi.ELQUA4NAX, None),
    ("BarNecking/BarNecking-3D/BarNecking.py", _abi.ELHEX8N3D, 3960),
    ("Element/Tensile/ElHex8N3D/Tensile.py", _abi.ELHEX8N3D, None),
    ("Element/Radial/ElQua4NAx/Radial.py", _abi.ELQUA4NAX, None),
    ("Element/Torus/ElQua4NAx/Torus.py", _abi.ELQUA4NAX, None),
    ("PlateNecking/PlateNecking.py", _abi.ELQUA4N2D, None),
    ("Element/Shear/ElQua4N2D/Shear.py", _abi.ELQUA4N2D, None),
    ("Element/Tensile/ElQua4N2D/Tensile.py", _abi.ELQUA4N2D, None),
])
def test_reference_samples_parse_unchanged(sample, etype, count, tmp_path, monkeypatch):
    captured = {}

    def fake_solve(self):
        captured["desc"] = self._description()[0]
        for n in self._nodes:  # results the script reads afterwards: the initial coordinates
            pass
        raise SystemExit(0)

    monkeypatch.setattr(dnl.DynELA, "solve", fake_solve)
    monkeypatch.setitem(sys.modules, "dnlPython", dnl)
    monkeypatch.setitem(sys.modules, "dnlCurves", types.ModuleType("dnlCurves"))
    monkeypatch.chdir(tmp_path)
    with pytest.raises(SystemExit):
        runpy.run_path(os.path.join(SAMPLES, sample), run_name="__main__")
    d = captured["desc"]
    assert d.elem_type == etype
    if count:
        assert d.n_elems == count
    with __import__("oracle").OracleModel(d.copy(ts_method=_abi.TS_COURANT)) as o:
        o.init()  # valid mesh: positive Jacobians, masses
        assert (o.nodes(_abi.NODE_MASS) > 0).all()


class OracleEngine:
    """The oracle behind the engine's handle interface (run / control / nodes /
    ips), so that the history writer of the model API can be checked on CPU."""

    def __init__(self, desc):
        from oracle import OracleModel
        self.o = OracleModel(desc)
        self.o.init()
        self.desc = desc
        self.t_end = desc.t_end
        self.last_dt = None

    def run(self, t_pause=np.inf, max_incs=0):
        n = 0
        while True:
            c = self.o.control()
            if c["status"] or c["time"] >= self.t_end or c["time"] >= t_pause or (max_incs and n >= max_incs):
                return n
            t0 = c["time"]
            self.o.run(max_incs=1)
            self.last_dt = self.o.control()["time"] - t0
            n += 1
            self._record()

    def control(self):
        c = self.o.control()
        c["done"] = c["time"] >= self.t_end
        c["last_time_step"] = self.last_dt if self.last_dt is not None else c["time_step"]
        return c

    def nodes(self, field):
        return self.o.nodes(field)

    def ips(self):
        return self.o.ips()

    def set_items(self, items):
        self.items = list(items)

    def set_history(self, schedules, capacity=0):
        """The device history records restated: after every increment, the
        save rule of HistoryFile::save per schedule, a record when one is due."""
        self.sched = [list(map(float, x)) for x in schedules]
        self.recs = []

    def _record(self):
        if not getattr(self, "sched", None):
            return
        c = self.control()
        mask = 0
        for j, sch in enumerate(self.sched):
            start, nxt, save = sch
            if not (c["time"] > start and c["time"] < nxt):
                sch[1] += save
                mask |= 1 << j
        if mask:
            self.recs.append((c["time"], c["increment"], self.last_dt, mask, self.gather_items()))

    def history_records(self):
        out, self.recs = self.recs, []
        return out

    def write_vtk(self, path, fields, prev=False, instance=0, title="DynELA FEM Code v.4.0"):
        """The engine's result file restated (oracle/vtk_ref.py)."""
        import vtk_ref
        pick = (lambda f: _abi.NODE_PREV[f]) if prev else (lambda f: f)
        nf = {"disp": self.o.nodes(_abi.NODE_DISP), "u": self.o.nodes(pick(_abi.NODE_U)),
              "speed": self.o.nodes(pick(_abi.NODE_SPEED)), "accel": self.o.nodes(pick(_abi.NODE_ACCEL)),
              "mass": self.o.nodes(_abi.NODE_MASS)}
        vtk_ref.write(path, self.o.control()["time"], self.o.nodes(_abi.NODE_COORDS), self.desc.conn,
                      12 if self.desc.nodes_per_element == 8 else 9, nf, self.o.ips(), fields, title)

    def gather_items(self):
        """The engine's item gather restated from the full arrays."""
        out = []
        for kind, field, index in self.items:
            if kind == _abi.ITEM_NODE:
                out.extend(self.o.nodes(field)[index])
            elif kind == _abi.ITEM_POINT:
                out.extend(self.o.ips()[:, index])
            else:
                v, m = self.o.nodes(field), self.o.nodes(_abi.NODE_MASS)[:, 0]
                out.append(float(np.sum(m * (v * v).sum(1) / 2.0)))
        return np.array(out)


def read_history(path):
    with open(path) as f:
        head = [f.readline(), f.readline()]
        rows = np.loadtxt(f, ndmin=2)
    return head, rows


def run_api_taylor(save_dir, **kw):
    model, n_nodes = taylor_axi_script(method=dnl.Explicit.PowerIteration, save_dir=str(save_dir), **kw)
    cwd = os.getcwd()
    os.chdir(save_dir)  # the result files go to the current directory, as the reference's
    try:
        model.solve()
    finally:
        os.chdir(cwd)
    out = {k: read_history(os.path.join(save_dir, k + ".plot")) for k in ("radius", "height", "plasticStrain", "dt", "ke")}
    return model, out


def test_history_files_through_oracle(tmp_path, monkeypatch):
    """History files written at the reference's save rule (HistoryFile.C:292-317):
    the first increment at or past each save time, values of that increment."""
    monkeypatch.setattr(dnl.DynELA, "_make_engine", staticmethod(lambda desc: OracleEngine(desc)))
    model, out = run_api_taylor(tmp_path)
    head, r = out["radius"]
    assert head[0] == "#DynELA FEM Code v. 4.0 history file\n"
    assert head[1].startswith("#plotted :coordsX")
    save = 80e-6 / 250
    t = r[:, 0]
    assert t[0] == 0.0 and r[0, 1] == pytest.approx(3.2)
    assert out["height"][1][0, 1] == pytest.approx(32.4)
    assert np.all(np.diff(t) > 0) and t[-1] == pytest.approx(80e-6, rel=1e-12)
    # a record per save time (an increment never spans two of them here)
    assert len(t) == 251 and np.all(t[1:] >= np.arange(1, 251) * save * (1 - 1e-12))
    rows = np.load(os.path.join(helpers.GOLDEN, "taylor_axi_sample.npz"))["rows"]
    row = rows[rows[:, 0] == _abi.TS_POWER_ITERATION][0]
    # the files hold 8 significant digits (%10.7E)
    assert abs(r[-1, 1] - row[3]) < 1e-7 * row[3]
    assert abs(out["height"][1][-1, 1] - row[4]) < 1e-7 * row[4]
    ke = out["ke"][1]
    v0 = 287000.0
    assert ke[0, 1] == pytest.approx(0.5 * model._engine.nodes(_abi.NODE_MASS)[:, 0].sum() * v0 * v0, rel=1e-7)
    # the impact turns nearly all kinetic energy into plastic work
    assert np.all(ke[:, 1] <= ke[0, 1] * (1 + 1e-7)) and ke[-1, 1] < 0.01 * ke[0, 1]
    np.savez_compressed(os.path.join(tmp_path, "hist.npz"), **{k: v[1] for k, v in out.items()})
    n = model.getNodeByNum(6)
    assert n.coords[0] == pytest.approx(row[3], rel=1e-9)
    # result files: the initial one, one per save time reached (the next
    # save time accumulates as DynELA::writeResultFile adds it), the final one
    nxt, saves = 80e-6 / 10, 0
    while nxt <= 80e-6:
        saves, nxt = saves + 1, nxt + 80e-6 / 10
    names = sorted(f for f in os.listdir(tmp_path) if f.endswith(".vtk"))
    assert names == [f"Taylor{k:03d}.vtk" for k in range(saves + 2)]
    import vtk_ref
    last = vtk_ref.parse(open(os.path.join(tmp_path, names[-1])).read())
    assert last["order"] == vtk_ref.DEFAULT_FIELDS and last["time"] == pytest.approx(80e-6)
    assert last["points"][5, 0] == pytest.approx(row[3], rel=1e-5)


@pytest.mark.gpu
def test_history_files_on_engine_match_oracle(tmp_path, monkeypatch):
    """The same script solved on the engine (FP64) writes the same history
    files as through the oracle: same save increments, values equal to the
    8 digits the files hold."""
    (tmp_path / "gpu").mkdir()
    _, gpu = run_api_taylor(tmp_path / "gpu")
    monkeypatch.setattr(dnl.DynELA, "_make_engine", staticmethod(lambda desc: OracleEngine(desc)))
    (tmp_path / "cpu").mkdir()
    _, cpu = run_api_taylor(tmp_path / "cpu")
    for k in cpu:
        a, b = gpu[k][1], cpu[k][1]
        assert a.shape == b.shape, k
        assert np.allclose(a[:, 0], b[:, 0], rtol=1e-12, atol=0), k
        scale = np.abs(b[:, 1:]).max() + 1e-300
        assert np.abs(a[:, 1:] - b[:, 1:]).max() <= 2e-7 * scale, k
    # the result files: written by the engine library, by the restatement on CPU
    import vtk_ref
    names = sorted(f for f in os.listdir(tmp_path / "cpu") if f.endswith(".vtk"))
    assert len(names) >= 11 and names == sorted(f for f in os.listdir(tmp_path / "gpu") if f.endswith(".vtk"))
    for n in names:
        g = vtk_ref.parse(open(tmp_path / "gpu" / n).read())
        c = vtk_ref.parse(open(tmp_path / "cpu" / n).read())
        assert g["header"] == c["header"]
        worst = vtk_ref.compare(g, c)
        assert max(worst.values()) < 2e-5, (n, worst)


@pytest.mark.gpu
def test_api_mixed_precision_taylor(tmp_path):
    """setPrecision('mixed') on the same script: final radius / height to 1e-4."""
    rows = np.load(os.path.join(helpers.GOLDEN, "taylor_axi_sample.npz"))["rows"]
    row = rows[rows[:, 0] == _abi.TS_POWER_ITERATION][0]
    _, out = run_api_taylor(tmp_path, precision="mixed")
    assert abs(out["radius"][1][-1, 1] - row[3]) < 1e-4 * row[3]
    assert abs(out["height"][1][-1, 1] - row[4]) < 1e-4 * row[4]


def test_stress_computation_method():
    """DynELA::setStressComputation (DynELA.C:1407-1431): "Direct" selects the
    one-step return, "NewtonRaphson" the iterated one, anything else is refused."""
    model, _ = taylor_axi_script(nr=2, nz=4)
    assert model._description()[0].stress_method == _abi.STRESS_NEWTON
    model.setStressComputation("Direct")
    assert model._description()[0].stress_method == _abi.STRESS_DIRECT
    model.setStressComputation("NewtonRaphson")
    assert model._description()[0].stress_method == _abi.STRESS_NEWTON
    with pytest.raises(ValueError):
        model.setStressComputation("Implicit")
