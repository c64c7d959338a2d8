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
}

if __name__ == "__main__":
    # python tests/golden/make_golden.py [case ...]   (all cases by default)
    for name in (sys.argv[1:] or list(CASES)):
        CASES[name]()
