#!/usr/bin/env python3
"""bench.py - element-steps/s of DynELA's explicit hot path on B200.

Workload: 3-D Taylor impact of a copper bar (R 3.2 mm, L 32.4 mm) meshed as an
O-grid cylinder of 960 x 160 = 153,600 ElHex8N3D elements (158,585 nodes,
1,228,800 Gauss points), 227 m/s onto a rigid wall, Courant time step every 10
increments.  A step is one explicit increment of the whole mesh (element pass,
nodal gather + Chung-Hulbert update, time-step pass), run from t = 0 (the
impact phase, where the radial return works hardest).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--precision mixed|fp64]
    python bench.py --impl reference ...   # the DynELA reference on the host cores

Several GPUs (torchrun, one process per GPU): every rank runs its own replica
of the mesh (a single mesh does not shard without a halo exchange), value is
the sum over ranks, timed as the max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "dynela-v.-4.0_b200")
sys.path.insert(0, PKG)

METRIC = "elem-steps/s (3-D copper Taylor impact, 153,600 ElHex8N3D)"
UNIT = "elem-steps/s"
WORKLOAD = "taylor3d-copper-ogrid-153600-hex8"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=1000)
    p.add_argument("--warmup", type=int, default=10)
    p.add_argument("--impl", default="engine", choices=["engine", "reference"])
    p.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--no-fp64", action="store_true")
    p.add_argument("--variant", type=int, default=-1,
                   help="element-pass variant (0-11, names in dnl_variant_name); default: chosen by the autotuner")
    p.add_argument("--no-accuracy", action="store_true", help="skip the whole-run mixed/FP64 comparison")
    p.add_argument("--no-batch", action="store_true", help="skip the batch of 256 Taylor bars")
    p.add_argument("--guess", action="store_true",
                   help="also run the learned Newton initial guess block (harvest, training, comparison; ~1 min)")
    p.add_argument("--no-necking", action="store_true", help="skip the necking workloads block")
    p.add_argument("--no-config0", action="store_true", help="skip the axisymmetric Taylor bar block")
    p.add_argument("--necking-whole", action="store_true",
                   help="also run the 1,198,080-element round bar to its 7 mm elongation, mixed and FP64 (~7 min)")
    p.add_argument("--batch-fp64-sample", type=int, default=256,
                   help="instances of the batch timed one by one on the FP64 path (default: all 256)")
    p.add_argument("--axial", type=int, default=160,
                   help="axial element layers (160 = the measured workload; fewer for profiling captures)")
    return p.parse_args()


AXIAL = 160


def variant_names(precision):
    """Names of the element-pass variants the autotuner chooses from
    (dnl_variant_name): staging scheme / blocks of 128 threads per SM that
    the register budget allows."""
    from dnlPython import _abi
    lib = _abi.load_library()
    return [lib.dnl_variant_name(int(precision), v).decode() for v in range(_abi.NUM_VARIANTS)]


def workload(precision):
    from dnlPython import _abi, meshes
    prec = _abi.PREC_MIXED if precision == "mixed" else _abi.PREC_FP64
    return meshes.taylor_3d(n_axial=AXIAL, length=32.4 * AXIAL / 160, precision=prec)


# ----------------------------------------------------------------- roofline

def alg_bytes(desc, word):
    """Algorithmic bytes of one increment, counted once per persistent array:
    per Gauss point 28 state words read+written + detJ0 read (57 word accesses),
    per element 8 int32 of connectivity, per node x, disp, du (FP64, read+write),
    v, a (FP64, read+write) and the mass (FP64, read).  Transients (F, R, J,
    dN/dx, strain increment, element force slots) count 0.  Returns
    (element kernel bytes, whole increment bytes)."""
    nE, nN = desc.n_elems, desc.n_nodes
    ip = nE * 8 * 57 * word
    conn = nE * 8 * 4
    elem = ip + conn + nN * (3 * 8 + 3 * 8)        # element pass reads x and du once per node
    step = ip + conn + nN * (3 * 3 * 8 * 2 + 2 * 3 * 8 * 2 + 8)
    return elem, step


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic():
    """DRAM bytes (read + write) of one element-kernel launch on this
    workload, from a committed ncu capture (profiles/element_kernel_traffic.json):
    a counter bench.py cannot read while it times.  Returns (bytes, source)."""
    p = os.path.join(ROOT, "profiles", "element_kernel_traffic.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["traffic_bytes_per_launch_mixed"]), \
            f"committed ncu capture of {d['kernel']} ({d['workload']}), profiles/element_kernel_traffic.json"
    except (OSError, KeyError, ValueError):
        return None, None


# ------------------------------------------------------------------- clocks

def smi_index(fallback, uuid=None, listing=None):
    """nvidia-smi's index of the GPU this process computes on: its CUDA device
    0 (the launcher's assignment, through CUDA_VISIBLE_DEVICES), matched by
    UUID against `nvidia-smi --query-gpu=index,uuid`; `fallback` when either
    is unavailable.  uuid / listing: given by the tests, queried otherwise."""
    try:
        if uuid is None:
            import torch
            uuid = str(torch.cuda.get_device_properties(0).uuid)
        if listing is None:
            listing = subprocess.run(["nvidia-smi", "--query-gpu=index,uuid", "--format=csv,noheader"],
                                     capture_output=True, text=True, timeout=30).stdout
    except Exception:
        return fallback
    want = uuid.lower().removeprefix("gpu-")
    for line in listing.splitlines():
        parts = [x.strip() for x in line.split(",")]
        if len(parts) == 2 and parts[1].lower().removeprefix("gpu-") == want:
            return int(parts[0])
    return fallback


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.out = tempfile.NamedTemporaryFile(prefix="clk_", suffix=".csv", delete=False)

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=self.out, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        time.sleep(0.15)

    def stop(self):
        if self.proc is None:
            return None
        time.sleep(0.1)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.out.close()
        rows = []
        with open(self.out.name) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.out.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if "Active" in r[5 + k] and "Not" not in r[5 + k]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


# -------------------------------------------------------------- CPU baseline

class quiet_stdout:
    """Send the C-level stdout to /dev/null (the reference prints progress
    lines; the bench prints exactly one JSON line)."""

    def __enter__(self):
        sys.stdout.flush()
        self.saved = os.dup(1)
        self.null = os.open(os.devnull, os.O_WRONLY)
        os.dup2(self.null, 1)
        return self

    def __exit__(self, *a):
        os.dup2(self.saved, 1)
        os.close(self.null)
        os.close(self.saved)


def reference_rate(desc, steps, warmup, threads):
    """The DynELA reference (oracle/_ref) on the host cores: elem-steps/s of
    `steps` increments after `warmup` ones, from its own solver-loop clock.
    Returns (value, kind, cores, sample) or None when it is not built."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import ref
    if not ref.available():
        return None
    with quiet_stdout():
        r = ref.RefModel(desc.copy(precision=0), threads=threads)
        try:
            r.init()
            if warmup:
                r.run(max_incs=warmup)
            s0 = r.solver_seconds()
            n = r.run(max_incs=steps)
            sec = r.solver_seconds() - s0
        finally:
            r.close()
    return desc.n_elems * n / sec, "reference", threads, \
        f"{n} increments of the full {desc.n_elems}-element mesh from t=0 after {warmup} warm-up increments, " \
        f"FP64, OpenMP {threads} threads (model build and start of the solve excluded)"


def port_rate(desc, steps):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    o = oracle.OracleModel(desc.copy(precision=0))
    o.init()
    t0 = time.perf_counter()
    n = o.run(max_incs=steps)
    sec = time.perf_counter() - t0
    o.close()
    return desc.n_elems * n / sec, "port", 1, f"{n} increments of the full mesh on the C restatement, 1 thread"


def cpu_baseline(desc):
    threads = os.cpu_count() or 1
    got = reference_rate(desc, steps=10, warmup=0, threads=threads)
    if got is None:
        got = port_rate(desc, steps=1)
    v, kind, cores, sample = got
    return {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample}


# ------------------------------------------------- whole runs and batches

def bar_results(desc, coords, ips):
    """Final bar length (highest node), foot radius (largest distance to the
    axis on the impact face), maximum equivalent plastic strain."""
    import numpy as np
    from dnlPython import _abi
    face = desc.coords[:, 1] == 0.0
    foot = np.sqrt(coords[face, 0] ** 2 + coords[face, 2] ** 2).max()
    return float(coords[:, 1].max()), float(foot), float(ips[_abi.IP_EPSP].max())


def accuracy_run():
    """The measured bar run to its end time on the mixed and the FP64 path:
    final length, foot radius and max plastic strain, with the mixed path's
    relative error against the FP64 path."""
    from dnlPython import _abi
    from dnlPython.engine import Engine
    res = {}
    for name in ("fp64", "mixed"):
        d = workload(name)
        with Engine(d) as e:
            e.init()
            e.autotune(steps=6)
            e.run()
            c = e.control()
            L, R, ep = bar_results(d, e.nodes(_abi.NODE_COORDS), e.ips())
            res[name] = {"increments": c["increment"], "time_s": c["time"], "status": c["status"],
                         "run_ms": e.timings()["run_ms"], "length_mm": L, "foot_radius_mm": R, "max_epsp": ep,
                         "fp64_resolves": c["fp64_resolves"]}
    m, f = res["mixed"], res["fp64"]
    res["rel_err_mixed_vs_fp64"] = {"length": abs(m["length_mm"] - f["length_mm"]) / f["length_mm"],
                                    "foot_radius": abs(m["foot_radius_mm"] - f["foot_radius_mm"]) / f["foot_radius_mm"],
                                    "max_epsp": abs(m["max_epsp"] - f["max_epsp"]) / f["max_epsp"]}
    res["whole_run_mixed_over_fp64"] = f["run_ms"] / m["run_ms"]
    res["reference"] = "FP64 GPU path (held to the FP64 oracle on the smaller cases of the test suite)"
    return res


def batch_run(sample, dist=None, world=1, rank=0):
    """256 independent copper Taylor bars (element counts log-uniform in
    2k-60k, speed U(150,300) m/s, Johnson-Cook A, B, n, C, m scaled by
    U(0.8,1.2), seed 20261203) advanced together to 80 us on the mixed path,
    against a size-stratified sample of the same bars run one by one on the
    FP64 path.  On several GPUs the bars are partitioned over the ranks
    (dnlPython.parallel.shard_instances, no exchange during the run) and the
    time is the slowest rank's."""
    import numpy as np
    from dnlPython import meshes, _abi, parallel
    from dnlPython.engine import Engine
    all_descs = meshes.taylor_batch()
    mine = parallel.shard_instances([parallel.instance_cost(d) for d in all_descs], world)[rank]
    descs = [all_descs[i] for i in mine]
    elems = np.array([d.n_elems for d in descs], dtype=np.float64)
    t0 = time.perf_counter()
    with Engine(descs) as b:
        b.init()
        variant, _ = b.autotune(steps=6)
        setup = time.perf_counter() - t0
        if dist is not None:
            dist.barrier()
        replays = b.run(check=False)
        ms_rank = b.timings()["run_ms"]
        launches = b.launch_count()
        ctl = [b.control(i) for i in range(len(descs))]
    incs = np.array([c["increment"] for c in ctl], dtype=np.float64)
    steps_rank = float((elems * incs).sum())
    ms = parallel.reduce_max(ms_rank, dist)
    steps = parallel.reduce_sum(steps_rank, dist)
    # one gather of the per-instance records at the end (every rank ran its own bars)
    rec = parallel.gather_records({mine[i]: {"increments": int(c["increment"]), "status": int(c["status"]),
                                             "time": float(c["time"])} for i, c in enumerate(ctl)}, dist)
    all_incs = np.array([rec[i]["increments"] for i in sorted(rec)], dtype=np.float64)
    n_all = len(all_descs)
    out = {"instances": n_all, "elements": int(sum(d.n_elems for d in all_descs)), "seed": 20261203,
           "precision": "mixed", "ranks": world, "replays_rank0": int(replays), "run_ms": ms,
           "sims_per_s": n_all / (ms / 1e3), "elem_steps_per_s": steps / (ms / 1e3),
           "increments_min_median_max": [int(all_incs.min()), int(np.median(all_incs)), int(all_incs.max())],
           "stopped_on_error": {str(i): _abi.ERRORS.get(r["status"], "error") + f" at t={r['time']:.3e}"
                                for i, r in sorted(rec.items()) if r["status"] != 0},
           "element_variant_rank0": int(variant), "gpu_launches_rank0": launches, "setup_s_rank0": setup}
    if sample > 0:
        order = np.argsort(elems, kind="stable")
        pick = order[np.linspace(0, len(order) - 1, min(sample, len(order))).astype(int)]
        t_ms, s_steps, s_elems = 0.0, 0.0, 0.0
        for i in pick:
            d = descs[i].copy(precision=_abi.PREC_FP64)
            with Engine(d) as e:
                e.init()
                n = e.run(check=False)
                t_ms += e.timings()["run_ms"]
                s_steps += d.n_elems * e.control()["increment"]
        rate = s_steps / (t_ms / 1e3)
        est_s = steps / rate
        every = len(pick) == len(descs)
        out["fp64_one_by_one"] = {"instances_timed": int(len(pick)), "elem_steps_per_s": rate,
                                  "seconds_all" if every else "est_seconds_all": est_s if not every else t_ms / 1e3,
                                  "sims_per_s" if every else "est_sims_per_s":
                                      len(descs) / (t_ms / 1e3 if every else est_s),
                                  "how": "every instance of the batch run alone to its end time on the FP64 path, "
                                         "device time of each run summed" if every else
                                         "every instance of a size-ordered stride timed alone to its end time; "
                                         "all-instance time extrapolated by elem-steps"}
        out["batched_mixed_over_one_by_one_fp64"] = out["elem_steps_per_s"] / rate
    return out


def necking_run(incs=300):
    """Throughput of the two tension workloads on the mixed path (FP64 beside
    it): the round bar (1,198,080 elements) and the plate (491,520 elements),
    each pulled by its ramped end speed, `incs` increments after 20, device
    time of the run."""
    from dnlPython import _abi, meshes
    from dnlPython.engine import Engine
    out = {}
    for name, make in (("bar_necking_1198080", meshes.bar_necking), ("plate_necking_491520", meshes.plate_necking)):
        res = {}
        for prec, pname in ((_abi.PREC_MIXED, "mixed"), (_abi.PREC_FP64, "fp64")):
            d = make(precision=prec)
            with Engine(d) as e:
                e.init()
                v, _ = e.autotune(steps=4)
                e.run(max_incs=20)
                e.run(max_incs=incs)
                ms = e.timings()["run_ms"]
                res[pname] = {"elem_steps_per_s": d.n_elems * incs / (ms / 1e3), "ms_per_step": ms / incs,
                              "variant": int(v)}
        res["mixed_over_fp64"] = res["mixed"]["elem_steps_per_s"] / res["fp64"]["elem_steps_per_s"]
        res["elements"] = d.n_elems
        out[name] = res
    return out


def necking_whole_run():
    """The round bar of 1,198,080 ElHex8N3D pulled to its 7 mm elongation (end
    speed ramped to 5 m/s over the first 10 % of the run) on the mixed and the
    FP64 path: increments, device time, and the results the mixed path is held
    to against the FP64 one (the FP64 GPU path stands in for the FP64 oracle,
    which is held to the reference on the first increments of this mesh): the
    elongation, the radius of the neck (the smallest distance to the axis in
    the symmetry plane y = 0) and the largest equivalent plastic strain."""
    import numpy as np
    from dnlPython import _abi, meshes
    from dnlPython.engine import Engine
    out = {}
    for prec, pname in ((_abi.PREC_MIXED, "mixed"), (_abi.PREC_FP64, "fp64")):
        d = meshes.bar_necking(precision=prec)
        plane = np.abs(d.coords[:, 1]) < 1e-12
        with Engine(d) as e:
            e.init()
            v, _ = e.autotune(steps=4)
            e.set_timing(False)
            t0 = time.perf_counter()
            n = e.run()
            wall = time.perf_counter() - t0
            c = e.control()
            x = e.nodes(_abi.NODE_COORDS)
            disp = e.nodes(_abi.NODE_DISP)
            ep = e.ips()[_abi.IP_EPSP]
        out[pname] = {"increments": int(n), "run_s": wall, "elem_steps_per_s": d.n_elems * n / wall,
                      "time": c["time"], "elongation_mm": float(disp[:, 1].max()),
                      "neck_radius_mm": float(np.hypot(x[plane, 0], x[plane, 2]).max()),
                      "max_epsp": float(ep.max()), "fp64_resolves": c["fp64_resolves"], "variant": int(v)}
    m, f = out["mixed"], out["fp64"]
    out["mixed_over_fp64"] = f["run_s"] / m["run_s"]
    out["mixed_vs_fp64"] = {k: abs(m[k] - f[k]) / abs(f[k]) for k in ("elongation_mm", "neck_radius_mm", "max_epsp")}
    out["elements"] = 1198080
    out["how"] = ("whole run to the end time, host wall time around dnl_engine_run (graph replays polled every 64 "
                  "increments); neck radius: largest distance to the axis of the nodes of the plane y = 0 (the "
                  "O-grid's outer ring) after the pull")
    return out


def config0_run():
    """The reference's own CPU-scale case: the axisymmetric copper Taylor bar
    (10 x 80 ElQua4NAx, 227 m/s, 80 us), run whole on the GPU with the Courant
    time step (every 10 increments) and with the power iteration of the
    Taylor-Axi sample (every increment), mixed and FP64; beside it the
    reference on the host cores for a bounded sample of its increments."""
    from dnlPython import _abi, meshes
    from dnlPython.engine import Engine
    out = {}
    for ts, tname, freq in ((_abi.TS_COURANT, "courant_every_10", 10), (_abi.TS_POWER_ITERATION, "power_iteration_every_1", 1)):
        res = {}
        for prec, pname in ((_abi.PREC_MIXED, "mixed"), (_abi.PREC_FP64, "fp64")):
            d = meshes.taylor_axi(ts_method=ts, ts_freq=freq, precision=prec)
            with Engine(d) as e:
                e.init()
                n = e.run()
                ms = e.timings()["run_ms"]
                c = e.nodes(_abi.NODE_COORDS)
                res[pname] = {"increments": int(n), "run_s": ms / 1e3, "elem_steps_per_s": d.n_elems * n / (ms / 1e3),
                              "height_mm": float(c[d.n_nodes - 1 - 10, 1]), "foot_radius_mm": float(c[10, 0])}
        d = meshes.taylor_axi(ts_method=ts, ts_freq=freq, precision=_abi.PREC_FP64)
        got = reference_rate(d, steps=1000, warmup=0, threads=os.cpu_count() or 1)
        if got is not None:
            v, kind, cores, sample = got
            res["reference"] = {"elem_steps_per_s": v, "cores": cores, "sample": sample,
                                "est_run_s": d.n_elems * res["fp64"]["increments"] / v}
        out[tname] = res
    out["elements"] = 800
    return out


def guess_run():
    """The learned Newton initial guess: pairs harvested from the first-yield
    returns of the 256-bar batch (its first 1,500 increments), the network
    trained on ln(gamma / gamma_max) by the engine's tensor-core kernels, then
    the same increments run from the same state with the reference's start
    and with the network's, on the first-yield window of the 3-D bar
    (increments 0-400) and of the necking plate (491,520 elements,
    increments 6,000-8,000)."""
    from dnlPython import _abi, guess, meshes
    t0 = time.perf_counter()
    cap, info = 10_000_000, {}
    pairs, st = guess.harvest(meshes.taylor_batch(), capacity=cap, stride=1, max_incs=1500,
                              scope=_abi.GUESS_FIRST_YIELD, info=info)
    stride = 1
    if info["candidates"] > cap:
        # more candidates than room: harvest again one in `stride`, a set that
        # fits and so does not depend on the order of the appends
        stride = -(-info["candidates"] // cap)
        del pairs
        pairs, st = guess.harvest(meshes.taylor_batch(), capacity=cap, stride=stride, max_incs=1500,
                                  scope=_abi.GUESS_FIRST_YIELD, info=info)
    t1 = time.perf_counter()
    net, hist = guess.train(pairs, epochs=20, batch_tiles=128, learning_rate=1e-3, log_target=True)
    t2 = time.perf_counter()
    out = {"pairs": int(pairs.shape[0]), "harvest_stride": stride, "harvest_s": t1 - t0, "train_s": t2 - t1,
           "loss_first_last": [hist[0], hist[-1]], "scope": "first yield (eps_p = 0)",
           "harvest_plain_evals_per_first_yield_point": st[3] / max(st[2], 1)}
    del pairs
    for name, desc, warm, incs in (("taylor3d_153600", workload("mixed"), 0, 400),
                                   ("plate_necking_491520", meshes.plate_necking(), 6000, 2000)):
        out[name] = guess.compare(desc, net, warm, incs, scope=_abi.GUESS_FIRST_YIELD)
        out[name]["window"] = [warm, warm + incs]
    return out


# ------------------------------------------------------------------ arms

# The reference runs an increment of the measured mesh in about 0.75 s on 16
# host threads: its arm runs the GPU arm's steps and warm-up as long as they
# stay within this many increments (a few minutes), and fewer beyond.
REF_MAX_INCREMENTS = 200


def bench_config(desc, args, world):
    """The `config` of the JSON line, the same on both arms."""
    return {"workload": WORKLOAD, "elements": desc.n_elems, "nodes": desc.n_nodes, "gauss_points": desc.n_ips,
            "time_step": "courant every 10", "increments_from_t0": [args.warmup, args.warmup + args.steps],
            "parallelism": f"replicas{world}" if world > 1 else "single",
            "l2": "inputs larger than L2 (point state 143 MB mixed / 285 MB FP64 > 126 MB)"}


def run_reference_arm(args, rank, world):
    if rank != 0:
        return
    desc = workload("fp64")
    threads = os.cpu_count() or 1
    steps, warmup = args.steps, args.warmup
    if steps + warmup > REF_MAX_INCREMENTS:
        steps = max(1, min(steps, REF_MAX_INCREMENTS // 2))
        warmup = min(warmup, REF_MAX_INCREMENTS - steps)
    got = reference_rate(desc, steps=steps, warmup=warmup, threads=threads)
    if got is None:
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libdnlref.so is not built"}))
        return
    v, kind, cores, sample = got
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": steps,
        "warmup": warmup, "ms_per_step": desc.n_elems / v * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "precision": "fp64", "data": "synthetic",
        "config": bench_config(desc, args, world),
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": kind, "sample": sample},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }))


def run_engine_arm(args, rank, world, dist):
    import numpy as np
    from dnlPython import _abi
    from dnlPython.engine import Engine

    def barrier():
        if dist is not None:
            dist.barrier()

    def max_over_ranks(x):
        from dnlPython import parallel
        return parallel.reduce_max(x, dist)

    desc = workload(args.precision)
    word = 4 if args.precision == "mixed" else 8
    eng = Engine(desc).init()
    if args.variant >= 0:
        eng.set_variant(args.variant)
        variant, variant_ms = eng.variant()
    else:
        variant, variant_ms = eng.autotune(steps=6)  # leaves the state unchanged
    if args.warmup:
        eng.run(max_incs=args.warmup)

    # ---- timed region: K increments, device time on the engine stream
    barrier()
    sampler = ClockSampler(smi_index(int(os.environ.get("LOCAL_RANK", "0")) if world > 1 else 0))
    sampler.start()
    done = eng.run(max_incs=args.steps)
    run_ms = eng.timings()["run_ms"]
    launches = eng.launch_count()
    clocks = sampler.stop()
    barrier()
    assert done == args.steps, f"ran {done} of {args.steps} increments"
    ms = max_over_ranks(run_ms)
    value = world * desc.n_elems * args.steps / (ms / 1e3)
    ctl = eng.control()

    # ---- roofline of the element kernel (per-kernel CUDA events on the engine
    # stream) over the same increments as the timed region: a second engine on
    # the same model replays them (the solve is deterministic) kernel by kernel
    eng.close()
    eng = Engine(desc).init()
    eng.set_variant(variant)
    if args.warmup:
        eng.run(max_incs=args.warmup)
    eng.set_timing(True)
    kt = args.steps
    eng.run(max_incs=kt)
    tim = eng.timings()
    eng.set_timing(False)
    elem_ms = tim["element_ms"] / kt
    eb, sb = alg_bytes(desc, word)
    peak, peak_kind = measured_peak()
    achieved = eb / (elem_ms / 1e3) / 1e9
    traffic, traffic_source = profiled_traffic() if args.precision == "mixed" else (None, None)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "traffic_source": traffic_source, "kernel": "k_element",
                "peak_source": peak_kind,
                "alg_bytes_per_launch": eb, "ms_per_launch": elem_ms}
    step_roofline = {"achieved": sb / (ms / args.steps / 1e3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": sb / (ms / args.steps / 1e3) / 1e9 / peak, "alg_bytes_per_step": sb,
                     "phase_ms_per_step": {"element": elem_ms, "nodal": tim["nodal_ms"] / kt,
                                           "timestep_and_control": tim["timestep_ms"] / kt}}
    eng.close()

    # ---- the FP64 path on the same workload (the mixed/FP64 ratio of the metric)
    fp64 = None
    if args.precision == "mixed" and not args.no_fp64:
        d64 = workload("fp64")
        e64 = Engine(d64).init()
        e64.autotune(steps=6)
        if args.warmup:
            e64.run(max_incs=args.warmup)
        k64 = min(args.steps, 500)
        e64.run(max_incs=k64)
        ms64 = e64.timings()["run_ms"]
        e64.close()
        fp64 = {"value": d64.n_elems * k64 / (ms64 / 1e3), "steps": k64, "ms_per_step": ms64 / k64}

    # ---- end to end through the public API, host buffers in and out
    e2e = None
    if not args.no_e2e:
        # the caller's result buffers, page-locked and allocated once (outside the timing)
        import torch
        # the point state in the engine's own precision (FP32 on the mixed path: nothing widened)
        ips_host = torch.empty((_abi.IP_NCOMP, desc.n_ips), pin_memory=True,
                               dtype=torch.float32 if args.precision == "mixed" else torch.float64).numpy()
        coords_host = torch.empty((desc.n_nodes, 3), dtype=torch.float64, pin_memory=True).numpy()

        def pinned(a):
            if a is None:
                return None
            p = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True).numpy().view(a.dtype).reshape(a.shape)
            p[...] = a
            return p

        # the caller's model arrays (the step's inputs) in page-locked host memory too
        desc_in = desc.copy(coords=pinned(desc.coords), conn=pinned(desc.conn), v_init=pinned(desc.v_init),
                            bc_code=pinned(desc.bc_code), bc_value=pinned(desc.bc_value),
                            bc_func=pinned(desc.bc_func))
        # three repetitions, the median reported (host-side times vary from
        # one run to the next with the state of the host's memory)
        reps = []
        for _ in range(3):
            barrier()
            t0 = time.perf_counter()
            e = Engine(desc_in)
            ta = time.perf_counter()
            e.init()
            e.set_variant(variant)
            tb = time.perf_counter()
            e.run(max_incs=args.steps)
            tc = time.perf_counter()
            coords = e.nodes(_abi.NODE_COORDS, out=coords_host)
            ips = e.ips_native(out=ips_host)
            t1 = time.perf_counter()
            e.close()
            reps.append((max_over_ranks(t1 - t0),
                         {"create_upload": ta - t0, "start": tb - ta, "increments": tc - tb, "read_back": t1 - tc}))
        reps.sort(key=lambda r: r[0])
        wall, secs = reps[len(reps) // 2]
        h2d = desc.coords.nbytes + desc.conn.nbytes + desc.v_init.nbytes + desc.bc_code.nbytes
        d2h = coords.nbytes + ips.nbytes
        e2e = {"value": world * desc.n_elems * args.steps / wall, "unit": UNIT,
               "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps,
               "what": "model upload from page-locked host arrays and build + start of the solve + K increments + "
                       "coordinates (FP64) and point state (in the path's own precision) read back into page-locked "
                       "host arrays allocated before the timing; median of 3 runs",
               "seconds": secs, "walls_s": [r[0] for r in reps]}

    batched = None
    if not args.no_batch:
        # partitioned over the ranks (collective timing: every rank takes part);
        # the one-by-one FP64 sample on a single GPU only
        batched = batch_run(args.batch_fp64_sample if world == 1 else 0, dist, world, rank)

    if rank != 0:
        return
    out = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64" if args.precision == "mixed" else "f64",
        "precision": args.precision, "data": "synthetic",
        "config": bench_config(desc, args, world),
        "roofline": roofline,
        "step_roofline": step_roofline,
        "gpu_launches": launches,
        "fp64_resolves": ctl["fp64_resolves"],
        "element_variant": {"chosen": int(variant), "autotune_ms": [round(float(x), 5) for x in variant_ms],
                            "names": variant_names(desc.precision), "how": (
                                "the autotuner times every variant (staging scheme x register budget) over "
                                "increments run from a saved copy of the state and keeps the fastest")},
    }
    if fp64:
        out["fp64_path"] = fp64
        # the like-for-like figure beside the reference (both FP64), at the top level
        out["fp64_value"] = fp64["value"]
        out["mixed_over_fp64"] = (desc.n_elems * args.steps / (run_ms / 1e3)) / fp64["value"]
    if clocks:
        out["clocks"] = clocks
    if e2e:
        out["e2e"] = e2e
    if world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(desc)
        if fp64:
            out["fp64_over_cpu_baseline"] = fp64["value"] / out["cpu_baseline"]["value"]
    # whole runs and the batch hold one GPU for a few minutes: single-GPU runs only
    if world == 1 and AXIAL == 160 and not args.no_accuracy:
        out["accuracy_whole_run"] = accuracy_run()
    if batched:
        out["batched"] = batched
    if world == 1 and not args.no_necking:
        out["necking"] = necking_run()
    if world == 1 and not args.no_config0:
        out["taylor_axi_800"] = config0_run()
    if world == 1 and args.necking_whole:
        out["necking_whole_run"] = necking_whole_run()
    if world == 1 and AXIAL == 160 and args.guess:
        out["learned_guess"] = guess_run()
    print(json.dumps(out))


def rank_device(visible, local):
    """The CUDA_VISIBLE_DEVICES of local rank `local`: the local-th of the
    devices the launcher gave the job (`visible`, indices or UUIDs), or
    device `local` when the launcher set none.  ValueError when the list is
    shorter than the ranks."""
    if visible is None or not visible.strip():
        return str(local)
    ids = [x.strip() for x in visible.split(",") if x.strip()]
    if local >= len(ids):
        raise ValueError(f"local rank {local} but CUDA_VISIBLE_DEVICES lists {len(ids)} devices")
    return ids[local]


def spawn_ranks(n):
    """Run this command again as n ranks under torch.distributed.run (local
    rendezvous on 127.0.0.1, a free port, a hard time limit well above the
    process group's own timeout) and exit with its status."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = ["timeout", "-k", "60", "3600", sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={n}", "--master-addr", "127.0.0.1", "--master-port", str(port),
           os.path.abspath(__file__)] + sys.argv[1:]
    sys.exit(subprocess.run(cmd).returncode)


def main():
    global AXIAL, WORKLOAD
    args = parse()
    AXIAL = args.axial
    if AXIAL != 160:
        WORKLOAD = f"taylor3d-copper-ogrid-{960 * AXIAL}-hex8"
    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        # --gpus N without a launcher: start the N ranks here (one process per GPU)
        spawn_ranks(args.gpus)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus:
        sys.exit(f"bench.py: --gpus {args.gpus} but the launcher started {world} ranks")
    if args.impl == "reference":
        run_reference_arm(args, rank, world)
        return
    dist = None
    if world > 1:
        # one process per GPU: this rank sees only its own device (the engine
        # creates its handles on the current device, device 0 of what it sees)
        try:
            os.environ["CUDA_VISIBLE_DEVICES"] = rank_device(os.environ.get("CUDA_VISIBLE_DEVICES"), local)
        except ValueError as e:
            sys.exit(f"bench.py: {e}")
        import datetime
        import torch
        import torch.distributed as tdist
        torch.cuda.set_device(0)
        tdist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = tdist
    try:
        run_engine_arm(args, rank, world, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
