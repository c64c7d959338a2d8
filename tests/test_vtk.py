"""VTK result files (DynELA::setSaveTimes -> writeResultFile / writeVTKFile,
DynELA.C:479-504, 688-711; VtkInterface.C:68-242).

The fixtures hold the files the compiled reference wrote itself during a run
(tests/golden/make_golden.py, cases vtk_axi and vtk_hex), with the reference's
state when it wrote each one:

* on CPU, the restatement oracle/vtk_ref.py, fed that state, writes the same
  files: same layout, cells, field order and header, every number within
  2e-5 of its field's largest magnitude (the files hold 6 significant digits);
* on the GPU, the engine (FP64) runs the same model with the same save
  schedule and its writer (dnl_engine_write_vtk: nodal extraction on the
  device, formatting in the library) gives the same files within the same
  bound; the files of dnlPython's solve() with setSaveTimes equal those of the
  same script on the CPU stand-in engine.
"""
import os

import numpy as np
import pytest

import helpers
from helpers import _abi
import vtk_ref

CASES = [os.path.join(helpers.GOLDEN, f"vtk_{c}.npz") for c in ("axi", "hex")]
RTOL = 2e-5


def _files(z):
    return [vtk_ref.parse(str(t)) for t in z["vtk_text"]]


@pytest.mark.parametrize("path", CASES, ids=["axi", "hex"])
def test_restatement_writes_the_reference_files(path, tmp_path):
    z = np.load(path)
    desc = helpers.desc_from_npz(z)
    want = _files(z)
    assert len(want) >= 4 and want[0]["time"] == 0.0
    vt = 12 if desc.nodes_per_element == 8 else 9
    for k, w in enumerate(want):
        nf = {f: z["vtk_" + f][k] for f in ("disp", "u", "speed", "accel", "mass")}
        text = vtk_ref.write(str(tmp_path / "f.vtk"), float(z["vtk_time"][k]), z["vtk_coords"][k], desc.conn, vt, nf,
                             z["vtk_ips"][k], w["order"])
        got = vtk_ref.parse(text)
        assert got["header"] == w["header"]
        worst = vtk_ref.compare(got, w)
        assert max(worst.values()) < RTOL, (k, worst)
    # the reference's default fields (its settings file), in that order
    assert want[0]["order"] == vtk_ref.DEFAULT_FIELDS


def _engine_files(z, tmp_path):
    """The engine on the fixture's model with the reference's save rule:
    the initial file, then a file at the first increment whose end time
    reaches each save time (one more increment when an increment passed two),
    then the final file."""
    from dnlPython.engine import Engine
    desc = helpers.desc_from_npz(z, precision=_abi.PREC_FP64)
    n_saves = len(z["vtk_text"]) - 2
    inc = desc.t_end / n_saves
    fields = vtk_ref.parse(str(z["vtk_text"][0]))["order"]
    out, incs = [], []
    with Engine(desc) as e:
        e.init()

        def write(prev):
            p = str(tmp_path / f"e{len(out):03d}.vtk")
            e.write_vtk(p, fields, prev=prev)
            out.append(vtk_ref.parse(open(p).read()))
            incs.append(e.control()["increment"])

        write(False)
        nxt = inc
        while e.control()["time"] < desc.t_end:
            t = e.control()["time"]
            e.run(t_pause=desc.t_end, max_incs=1) if t >= nxt else e.run(t_pause=nxt)
            t = e.control()["time"]
            if t >= nxt and t <= desc.t_end:
                write(True)
                nxt += inc
        write(False)
    return out, incs


@pytest.mark.gpu
@pytest.mark.parametrize("path", CASES, ids=["axi", "hex"])
def test_engine_writes_the_reference_files(path, tmp_path):
    z = np.load(path)
    got, incs = _engine_files(z, tmp_path)
    want = _files(z)
    assert incs == list(z["vtk_increment"])
    assert len(got) == len(want)
    for k, (g, w) in enumerate(zip(got, want)):
        assert g["header"] == w["header"]
        worst = vtk_ref.compare(g, w)
        assert max(worst.values()) < RTOL, (k, worst)


@pytest.mark.gpu
def test_node_averages_match_restatement():
    """dnl_engine_node_averages against the restatement on a plastified state
    (every point-state component and the von Mises stress)."""
    from dnlPython.engine import Engine
    import oracle
    desc = helpers.case_hex_small()
    with oracle.OracleModel(desc) as o:
        o.init()
        ips = helpers.random_point_state(desc, o.ips(), seed=3)
    comps = list(range(_abi.IP_NCOMP)) + [_abi.NODE_AVG_VON_MISES]
    with Engine(desc) as e:
        e.init()
        e.set_ips(ips)
        got = e.node_averages(comps)
    want = vtk_ref.node_averages(desc.conn, desc.n_nodes, np.vstack([ips, vtk_ref.von_mises(ips)[None]]))
    assert np.allclose(got, want, rtol=1e-13, atol=1e-12 * np.abs(want).max())
