"""bench.py's host logic, run on the CPU: which GPU a rank computes on and
whose clocks it samples under a launcher, and the reference arm's JSON line
(the reference compiled from its sources, timed on the host cores)."""
import os

import pytest

import helpers


def test_clock_sampler_follows_the_assigned_gpu():
    """The bench samples the clocks of the GPU its rank computes on: the one
    whose UUID matches its CUDA device 0, wherever that lies in nvidia-smi's
    list (a launcher may hand a job GPUs 4 and 5); the rank's index when no
    match can be made."""
    import sys
    sys.path.insert(0, helpers.ROOT)
    import bench
    listing = ("0, GPU-aaaa-0000\n1, GPU-bbbb-1111\n4, GPU-cccc-4444\n5, GPU-dddd-5555\n")
    assert bench.smi_index(1, uuid="dddd-5555", listing=listing) == 5
    assert bench.smi_index(0, uuid="GPU-CCCC-4444", listing=listing) == 4
    assert bench.smi_index(1, uuid="eeee-9999", listing=listing) == 1
    assert bench.smi_index(3, uuid="aaaa-0000", listing="") == 3


def test_each_rank_takes_its_own_assigned_gpu():
    """Under a launcher every rank runs on the local-rank-th of the GPUs the
    job was given, never on a GPU outside that list."""
    import sys
    sys.path.insert(0, helpers.ROOT)
    import bench
    assert bench.rank_device("4,5", 0) == "4" and bench.rank_device("4,5", 1) == "5"
    assert bench.rank_device(" 6 , 7 ", 1) == "7"
    assert bench.rank_device("GPU-aaaa,GPU-bbbb", 1) == "GPU-bbbb"
    assert bench.rank_device(None, 3) == "3" and bench.rank_device("", 2) == "2"
    with pytest.raises(ValueError, match="lists 2 devices"):
        bench.rank_device("4,5", 2)


def test_reference_arm_prints_one_contract_line():
    """`bench.py --impl reference` times the reference compiled from its
    sources on the host cores and prints one JSON line with the metric,
    config and unit of the engine arm, impl "reference", a cpu_baseline
    describing the run and an e2e figure equal to its value with no
    host-device bytes (a reduced mesh keeps the test short)."""
    import json
    import subprocess
    import sys
    sys.path.insert(0, os.path.join(helpers.ROOT, "oracle"))
    import ref
    if not ref.available():
        pytest.skip("oracle/_ref is not built")
    out = subprocess.run([sys.executable, os.path.join(helpers.ROOT, "bench.py"), "--impl", "reference",
                          "--steps", "2", "--warmup", "1", "--axial", "8"],
                         capture_output=True, text=True, timeout=600, cwd=helpers.ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [x for x in out.stdout.splitlines() if x.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better", "scaling",
              "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert k in d, k
    assert d["impl"] == "reference" and d["unit"] == "elem-steps/s" and d["higher_is_better"] is True
    assert d["value"] > 0 and d["steps"] == 2 and d["warmup"] == 1
    assert d["config"]["elements"] == 960 * 8
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["value"] == d["value"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}
