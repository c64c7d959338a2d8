"""Generate the golden fixtures of tests/golden/ from the DynELA reference
compiled from its own sources (oracle/_ref/libdnlref.so, built by
`make -C oracle ref`).  Run from the repository root:

    python tests/golden/make_golden.py

Each fixture stores the model description it was made from, so the tests
rebuild exactly the same model.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import helpers  # noqa: E402
from helpers import _abi, meshes  # noqa: E402
import ref  # noqa: E402  (oracle/ref.py)


def snapshot(r, prefix):
    out = {}
    for name, f in (("coords", _abi.NODE_COORDS), ("disp", _abi.NODE_DISP), ("speed", _abi.NODE_SPEED),
                    ("u", _abi.NODE_U), ("accel", _abi.NODE_ACCEL), ("mass", _abi.NODE_MASS)):
        out[prefix + name] = r.nodes(f)
    out[prefix + "ips"] = r.ips()
    c = r.control()
    out[prefix + "control"] = np.array([c["time"], c["time_step"], c["increment"]])
    return out


def run_case(name, desc, checkpoints):
    data = helpers.desc_to_npz(desc)
    with ref.RefModel(desc) as r:
        r.init()
        data.update(snapshot(r, "init_"))
        done = 0
        for k in checkpoints:
            r.run(max_incs=k - done)
            done = k
            data.update(snapshot(r, f"inc{k}_"))
    data["checkpoints"] = np.array(checkpoints)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **data)
    print(name, "ok", {k: v.shape for k, v in data.items() if k.startswith("inc")}.__len__())


def pass_case(name, desc, seed):
    """Element pass (strains -> forces, density) on a seeded random state."""
    data = helpers.desc_to_npz(desc)
    with ref.RefModel(desc) as r:
        r.init()
        ips = helpers.random_point_state(desc, r.ips(), seed)
        u = helpers.random_increment(desc, seed + 1)
        dt = 1.3e-8
        r.set_ips(ips)
        r.set_nodes(_abi.NODE_U, u)
        data["in_ips"], data["in_u"], data["in_coords"], data["dt"] = ips, u, r.nodes(_abi.NODE_COORDS), np.array(dt)
        r.element_pass(dt)
        data["out_ips"] = r.ips()
        data["out_force"] = r.nodes(_abi.NODE_FORCE)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **data)
    print(name, "ok")


def published_case():
    """The Taylor-Axi sample of the reference (Samples/Taylor/Taylor-Axi/Taylor.py:10-35,
    steel 42CrMo4, 287 m/s, 5 x 50 ElQua4NAx, 80 us) with the Courant and the
    power-iteration time step, final height / radius / max plastic strain."""
    rows = []
    for method, freq in ((_abi.TS_POWER_ITERATION, 1), (_abi.TS_COURANT, 1), (_abi.TS_COURANT, 10)):
        d = meshes.taylor_axi(nr=5, nz=50, radius=3.2, length=32.4, speed=287000.0, mat=meshes.STEEL_42CRMO4,
                              t_end=80e-6, ts_method=method, ts_freq=freq)
        with ref.RefModel(d) as r:
            r.init()
            n = r.run()
            c = r.nodes(_abi.NODE_COORDS)
            ip = r.ips()
            rows.append([method, freq, n, c[5, 0], c[d.n_nodes - 6, 1],
                         ip[_abi.IP_EPSP].reshape(-1, 4).mean(1).max(), ip[_abi.IP_EPSP].max()])
    np.savez_compressed(os.path.join(HERE, "taylor_axi_sample.npz"), rows=np.array(rows))
    print("taylor_axi_sample", rows)


# ---------------------------------------------------------------- full size
#
# The measured workloads at their full size.  Their arrays are too large to
# commit, so a fixture keeps (a) a seeded sample of nodes and integration
# points with every field of them, compared entry by entry, and (b) sums over
# every node and point of each field component (signed, absolute and the
# largest magnitude), which catch an error anywhere in the mesh.  The mesh is
# rebuilt by its generator (dnlPython.meshes) from the recorded arguments; a
# digest of the coordinates and connectivity guards against a generator change.

FULL_MESHES = {
    "taylor3d_153600": ("taylor_3d", {}),
    "bar_necking_1198080": ("bar_necking", {}),
    "plate_necking_491520": ("plate_necking", {}),
}
NODE_FIELDS = (("coords", _abi.NODE_COORDS), ("disp", _abi.NODE_DISP), ("speed", _abi.NODE_SPEED),
               ("u", _abi.NODE_U), ("accel", _abi.NODE_ACCEL), ("force", _abi.NODE_FORCE))


def full_desc(mesh):
    name, kw = FULL_MESHES[mesh]
    return getattr(meshes, name)(precision=_abi.PREC_FP64, **kw)


def full_sample(desc, n_nodes=4096, n_ips=8192, seed=20261204):
    rng = np.random.default_rng(seed)
    nodes = np.unique(np.concatenate([rng.choice(desc.n_nodes, min(n_nodes, desc.n_nodes), replace=False),
                                      [0, desc.n_nodes - 1, int(np.argmax(desc.coords[:, 1]))]]))
    ips = np.unique(np.concatenate([rng.choice(desc.n_ips, min(n_ips, desc.n_ips), replace=False),
                                    [0, desc.n_ips - 1]]))
    return nodes.astype(np.int64), ips.astype(np.int64)


def full_snapshot(r, prefix, nodes, ips):
    out = {}
    for name, f in NODE_FIELDS:
        a = r.nodes(f)
        out[prefix + name] = a[nodes]
        out[prefix + name + "_sums"] = helpers.field_sums(a)
    ip = r.ips()
    out[prefix + "ips"] = ip[:, ips]
    out[prefix + "ips_sums"] = helpers.field_sums(ip.T)
    c = r.control()
    out[prefix + "control"] = np.array([c["time"], c["time_step"], c["increment"]])
    return out


def full_run_case(mesh, checkpoints, threads=None):
    """The first increments of a full-size workload (FP64, from t = 0)."""
    desc = full_desc(mesh)
    nodes, ips = full_sample(desc)
    data = {"mesh": np.array(mesh), "digest": np.array(helpers.mesh_digest(desc)), "sample_nodes": nodes,
            "sample_ips": ips, "checkpoints": np.array(checkpoints)}
    with ref.RefModel(desc, threads=threads or os.cpu_count()) as r:
        r.init()
        data.update(full_snapshot(r, "init_", nodes, ips))
        done = 0
        for k in checkpoints:
            r.run(max_incs=k - done)
            done = k
            data.update(full_snapshot(r, f"inc{k}_", nodes, ips))
            print(f"fullsize_{mesh}_incs: increment {k}", flush=True)
    np.savez_compressed(os.path.join(HERE, f"fullsize_{mesh}_incs.npz"), **data)
    print(f"fullsize_{mesh}_incs ok")


def oracle_values(mesh):
    """The C restatement (oracle/dnl_oracle.c, FP64) on a full-size run
    fixture's model, stored in the fixture at every checkpoint, in three runs:

    * the reference's route (C = F^T F): its values at the sampled nodes and
      points and whole-field sums (`*_orc`, `*_orc_sums`), time and time step
      (`*_control_orc`), and its distance to the reference measured as the
      tests measure the engine's (`*_onoise`, `*_osums`).  The reference's
      rotation is inaccurate where two principal stretches nearly coincide
      (polar_defect_case), which moves its runs away from any accurate polar
      decomposition;
    * the same from H = F - I (orc_polar_lnU_h, the engine's route: no
      rounding of C's entries near 1, which is a relative error of 1e-16 over
      the strain increment in ln U, 1e-9 in the first increments of the
      quasi-static necking pulls): `*_orh`, `*_orh_sums`, `*_control_orh`,
      and its distance to the reference (`*_hnoise`, `*_hsums`);
    * the H route again from coordinates moved by one unit in the last place
      (seeded signs), measured against `*_orh` (`*_pnoise`, `*_psums`,
      `*_control_pnoise`): how far rounding alone carries two FP64 runs of
      the same algorithm apart.  The engine sums in other orders than the
      restatement, so its rounding differs by about as much.

    The H-route values are the strict yardstick of the engine's runs."""
    import oracle
    path = os.path.join(HERE, f"fullsize_{mesh}_incs.npz")
    derived = ("_onoise", "_osums", "_orc", "_orc_sums", "_pnoise", "_psums", "_control_orc", "_control_pnoise",
               "_orh", "_orh_sums", "_control_orh", "_hnoise", "_hsums")
    data = {k: v for k, v in np.load(path).items() if not k.endswith(derived)}
    desc = full_desc(mesh)
    nodes, ips = data["sample_nodes"], data["sample_ips"]
    names = [m for m, _ in helpers.FULL_NODE_FIELDS] + ["ips"]
    ref_only = dict(data)

    def run(model_desc, route, tag, noise_tag, against):
        with oracle.OracleModel(model_desc) as o:
            o.set_polar_route(route)
            o.init()
            done = 0
            for k in data["checkpoints"]:
                done += o.run(max_incs=int(k) - done)
                for name, (err, serr) in helpers.full_size_errors(o, against, f"inc{k}_").items():
                    data[f"inc{k}_{name}_{noise_tag}noise"] = err
                    data[f"inc{k}_{name}_{noise_tag}sums"] = serr
                c = o.control()
                ctl = np.array([c["time"], c["time_step"], c["increment"]], dtype=np.float64)
                if tag:
                    for name, f in helpers.FULL_NODE_FIELDS:
                        a = o.nodes(f)
                        data[f"inc{k}_{name}_{tag}"] = a[nodes]
                        data[f"inc{k}_{name}_{tag}_sums"] = helpers.field_sums(a)
                    ip = o.ips()
                    data[f"inc{k}_ips_{tag}"] = ip[:, ips]
                    data[f"inc{k}_ips_{tag}_sums"] = helpers.field_sums(ip.T)
                    data[f"inc{k}_control_{tag}"] = ctl
                else:
                    co = data[f"inc{k}_control_orh"]
                    data[f"inc{k}_control_pnoise"] = np.abs(ctl[:2] - co[:2]) / co[:2]
                print(f"oracle {mesh} route {route} {tag or 'perturbed'} increment {k}: distance ({noise_tag}) " +
                      " ".join(f"{n} {data[f'inc{k}_{n}_{noise_tag}noise'].max():.1e}" for n in names), flush=True)

    run(desc, 0, "orc", "o", ref_only)
    run(desc, 1, "orh", "h", ref_only)
    # the perturbed H-route run against the H-route values
    orh = {f"inc{k}_{n}": data[f"inc{k}_{n}_orh"] for k in data["checkpoints"] for n in names}
    orh.update({f"inc{k}_{n}_sums": data[f"inc{k}_{n}_orh_sums"] for k in data["checkpoints"] for n in names})
    orh.update(sample_nodes=nodes, sample_ips=ips)
    signs = np.random.default_rng(20261204).integers(-1, 2, size=desc.coords.shape)
    run(desc.copy(coords=desc.coords * (1.0 + 2.0 ** -52 * signs)), 1, None, "p", orh)
    np.savez_compressed(path, **data)


def polar_defect_case():
    """One element cut from the reference's own run of the 153,600-element
    bar at increment 17 (element 3090: its nodes' coordinates and increments,
    its points' state, the time step).  At its Gauss point 0 the two lateral
    principal stretches differ by ~1e-12 (uniaxial compression in the impact
    zone) and the reference's eigen-solver returns eigenvectors that are not
    orthonormal, so its U, and the rotation R = F U^-1 (Tensor2::
    polarExtractLnU, Tensor2.C:1237-1313), are off by ~2e-3."""
    desc = full_desc("taylor3d_153600")
    e = 3090
    with ref.RefModel(desc, threads=os.cpu_count()) as r:
        r.init()
        r.run(max_incs=17)
        x, u = r.nodes(_abi.NODE_COORDS), r.nodes(_abi.NODE_U)
        ips = r.ips()[:, e * 8:(e + 1) * 8]
        dt = r.control()["time_step"]
    nodes = desc.conn[e]
    np.savez_compressed(os.path.join(HERE, "polar_defect_element.npz"), coords=x[nodes], u=u[nodes], ips=ips,
                        dt=np.array(dt), element=np.array(e), increment=np.array(17))
    print("polar_defect_element ok")


def full_pass_case(mesh, seed, dt=4e-9, threads=None):
    """One element pass of a full-size mesh on a seeded plastic state and
    displacement increment (helpers.random_point_state / random_increment,
    regenerated by the test from the same seeds)."""
    desc = full_desc(mesh)
    nodes, ips = full_sample(desc)
    data = {"mesh": np.array(mesh), "digest": np.array(helpers.mesh_digest(desc)), "sample_nodes": nodes,
            "sample_ips": ips, "seed": np.array(seed), "dt": np.array(dt)}
    with ref.RefModel(desc, threads=threads or os.cpu_count()) as r:
        r.init()
        st = helpers.random_point_state(desc, r.ips(), seed)
        u = helpers.random_increment(desc, seed + 1)
        r.set_ips(st)
        r.set_nodes(_abi.NODE_U, u)
        del st, u
        r.element_pass(dt)
        f = r.nodes(_abi.NODE_FORCE)
        data["out_force"] = f[nodes]
        data["out_force_sums"] = helpers.field_sums(f)
        ip = r.ips()
        data["out_ips"] = ip[:, ips]
        data["out_ips_sums"] = helpers.field_sums(ip.T)
    np.savez_compressed(os.path.join(HERE, f"fullsize_{mesh}_elempass.npz"), **data)
    print(f"fullsize_{mesh}_elempass ok")


def config0_case():
    """The axisymmetric copper bar of 10 x 80 ElQua4NAx at 227 m/s run to
    80 us by the reference, with the power-iteration time step every
    increment (the method of the reference's Taylor-Axi sample) and with the
    Courant time step every 10 increments: the final nodal fields and point
    state whole (891 nodes, 3,200 points), and the increment count."""
    data = {}
    for tag, method, freq in (("pi1", _abi.TS_POWER_ITERATION, 1), ("courant10", _abi.TS_COURANT, 10)):
        d = meshes.taylor_axi(ts_method=method, ts_freq=freq, precision=_abi.PREC_FP64)
        if tag == "pi1":
            data.update(helpers.desc_to_npz(d))
        with ref.RefModel(d, threads=1) as r:
            r.init()
            n = r.run()
            for name, f in NODE_FIELDS[:5]:
                data[f"{tag}_{name}"] = r.nodes(f)
            data[f"{tag}_ips"] = r.ips()
            c = r.control()
            data[f"{tag}_control"] = np.array([c["time"], c["time_step"], c["increment"], n])
        x = data[f"{tag}_coords"]
        ep = data[f"{tag}_ips"][_abi.IP_EPSP].reshape(-1, 4).mean(1).max()
        print(f"config0 {tag}: {n} increments, height {x[d.n_nodes - 11, 1]:.4f}, radius {x[10, 0]:.4f}, "
              f"max element-mean eps_p {ep:.4f}", flush=True)
    np.savez_compressed(os.path.join(HERE, "config0_whole.npz"), **data)


def vtk_case(name, desc, n_saves):
    """The reference's own result files (its VtkInterface, fields from its
    settings file) for a run with setSaveTimes(0, t_end, t_end / n_saves):
    the text of every file, and the reference's state when it wrote each one
    (the run stops at the increment that writes a file), for the checks of
    the restatement oracle/vtk_ref.py and of the engine's writer."""
    sdir = os.path.join(ref.reference_dir(), "Sources", "dnlSettings")
    os.environ["DNL_REF_SETTINGS"] = sdir
    data = helpers.desc_to_npz(desc)
    inc = desc.t_end / n_saves
    snaps = []

    def snap(r, prev):
        pick = (lambda f: _abi.NODE_PREV[f]) if prev else (lambda f: f)
        snaps.append({"time": r.control()["time"], "coords": r.nodes(_abi.NODE_COORDS),
                      "disp": r.nodes(_abi.NODE_DISP), "u": r.nodes(pick(_abi.NODE_U)),
                      "speed": r.nodes(pick(_abi.NODE_SPEED)), "accel": r.nodes(pick(_abi.NODE_ACCEL)),
                      "mass": r.nodes(_abi.NODE_MASS), "ips": r.ips(), "increment": r.control()["increment"]})

    with ref.RefModel(desc) as r:
        r.init()
        r.enable_vtk(0.0, desc.t_end, inc)  # writes the initial file
        snap(r, False)
        nxt = inc
        while r.control()["time"] < desc.t_end:
            t = r.control()["time"]
            r.run(max_incs=1) if t >= nxt else r.run(t_stop=nxt)
            t = r.control()["time"]
            if t >= nxt and t <= desc.t_end:  # DynELA::writeResultFile's test
                snap(r, True)
                nxt += inc
        r.write_final_vtk()
        snap(r, False)
        files = sorted(f for f in os.listdir(r.workdir) if f.endswith(".vtk"))
        texts = [open(os.path.join(r.workdir, f)).read() for f in files]
    assert len(texts) == len(snaps), (len(texts), len(snaps))
    data["vtk_text"] = np.array(texts)
    data["vtk_increment"] = np.array([s_["increment"] for s_ in snaps])
    data["vtk_prev"] = np.array([0] + [1] * (len(snaps) - 2) + [0])
    for k in ("time", "coords", "disp", "u", "speed", "accel", "mass", "ips"):
        data["vtk_" + k] = np.array([s_[k] for s_ in snaps])
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **data)
    print(name, len(texts), "files")


CASES = {
    "axi_run": lambda: run_case("axi_run", helpers.case_axi_small(), [1, 10, 200]),
    "hex_run": lambda: run_case("hex_run", helpers.case_hex_small(), [1, 10, 60]),
    "hex_speed_run": lambda: run_case("hex_speed_run", helpers.case_hex_speed(), [1, 10, 60]),
    "axi_pass": lambda: pass_case("axi_pass", helpers.case_axi_small(), seed=5),
    "hex_pass": lambda: pass_case("hex_pass", helpers.case_hex_small(), seed=6),
    # Element::computeStressDirect (DynELA::setStressComputation("Direct"))
    "hex_direct_run": lambda: run_case("hex_direct_run", helpers.case_hex_small().copy(stress_method=_abi.STRESS_DIRECT),
                                       [1, 10, 60]),
    "hex_direct_pass": lambda: pass_case("hex_direct_pass",
                                         helpers.case_hex_small().copy(stress_method=_abi.STRESS_DIRECT), seed=7),
    # the round bar pulled by a ramped end speed (necking workload, small mesh)
    "bar_necking_run": lambda: run_case("bar_necking_run", helpers.case_bar_necking(), [1, 10, 60]),
    # plane-strain quads (ElQua4N2D)
    "plane_run": lambda: run_case("plane_run", helpers.case_plane_small(), [1, 10, 60]),
    "plane_pass": lambda: pass_case("plane_pass", helpers.case_plane_small(), seed=8),
    "taylor_axi_sample": published_case,
    "config0_whole": config0_case,
    # result files of the reference (VtkInterface) at its save times
    "vtk_axi": lambda: vtk_case("vtk_axi", helpers.case_axi_small(), 4),
    "vtk_hex": lambda: vtk_case("vtk_hex", helpers.case_hex_speed(), 4),
    "fullsize_taylor3d_153600_incs": lambda: full_run_case("taylor3d_153600", [1, 10, 50]),
    "fullsize_taylor3d_153600_elempass": lambda: full_pass_case("taylor3d_153600", seed=51),
    # the C oracle's values and distance to the reference at each checkpoint (added to the run fixtures)
    "oracle_values_taylor3d_153600": lambda: oracle_values("taylor3d_153600"),
    "oracle_values_plate_necking_491520": lambda: oracle_values("plate_necking_491520"),
    "oracle_values_bar_necking_1198080": lambda: oracle_values("bar_necking_1198080"),
    # the reference's inaccurate rotation at nearly repeated principal stretches
    "polar_defect_element": polar_defect_case,
    "fullsize_plate_necking_491520_incs": lambda: full_run_case("plate_necking_491520", [1, 5, 10]),
    "fullsize_plate_necking_491520_elempass": lambda: full_pass_case("plate_necking_491520", seed=53),
    "fullsize_bar_necking_1198080_incs": lambda: full_run_case("bar_necking_1198080", [1, 5, 10]),
    "fullsize_bar_necking_1198080_elempass": lambda: full_pass_case("bar_necking_1198080", seed=52),
}

if __name__ == "__main__":
    # python tests/golden/make_golden.py [case ...]   (all cases by default)
    names = sys.argv[1:] or list(CASES)
    if len(names) == 1:
        CASES[names[0]]()
    else:
        # one process per case: the reference keeps its model in process-wide
        # state, and a large model built after another one can crash it
        import subprocess
        for name in names:
            subprocess.run([sys.executable, os.path.abspath(__file__), name], check=True)
