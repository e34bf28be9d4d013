"""bench.py --impl reference: the reference's own CPU advance, timed on the host cores, on
the JSON contract of the B200 arm (same metric and unit, impl "reference", a cpu_baseline
that describes the run, an e2e with no device copies).  Runs without a GPU."""
import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def run_arm(workload):
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--workload", workload, "--steps", "1", "--warmup", "1"],
                       capture_output=True, text=True, timeout=600, env=env, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 1, r.stdout
    return json.loads(lines[0])


@pytest.mark.parametrize("workload", ["turb64_plm_hlld_rk2"])
def test_reference_arm_json_contract(workload):
    import bench
    d = run_arm(workload)
    assert d["impl"] == "reference"
    assert d["metric"] == bench.METRIC and d["unit"] == bench.UNIT
    assert d["higher_is_better"] is True
    assert d["steps"] == 1 and d["warmup"] == 1 and d["n_gpus"] == 1
    assert d["config"]["workload"] == workload
    assert d["value"] > 0
    cb = d["cpu_baseline"]
    assert cb["value"] == d["value"] and cb["unit"] == d["unit"]
    assert cb["kind"] in ("reference", "port") and cb["cores"] >= 1 and cb["sample"]
    assert d["e2e"] == {"value": d["value"], "unit": d["unit"], "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


def test_default_workload_is_the_512_plm_hlld_rk3_box():
    import bench
    n, ic, kw = bench.WORKLOADS[bench.DEFAULT_WORKLOAD]
    assert n == (512, 512, 512) and ic == "turbulence"
    assert kw == dict(extrap="plm", riemann="hlld", advance="rk3")


def test_ghost_correction_and_linf():
    import numpy as np
    import bench
    assert bench.ghost_factor(64, (64, 64, 64)) == 1.0
    # 64^3 sample (70^3 guarded) against a 512^3 box (518^3 guarded)
    want = (70 / 64) ** 3 / (518 / 512) ** 3
    assert abs(bench.ghost_factor(64, (512, 512, 512)) - want) < 1e-12
    a = np.ones((10, 10, 10, 8))
    b = a.copy()
    b[5, 5, 5, 0] = 1.5            # interior zone
    b[0, 0, 0, 1] = 9.0            # guard zone: not counted
    r = bench.rel_linf(a, b, 3)
    assert abs(r["rho"] - 0.5 / 1.5) < 1e-15 and r["pre"] == 0.0


def test_tiled_block_is_a_window_of_the_periodic_repetition():
    """--decompose builds each rank's block from a small turbulence box repeated periodically:
    a block is exactly the window of the repeated box, guards included."""
    import numpy as np
    import bench
    from ctf_b200 import ics
    t = ics.turbulence_box((8, 8, 8), seed=3)
    assert np.array_equal(bench.tiled_block(t, (0, 0, 0), (8, 8, 8)), t)
    whole = bench.tiled_block(t, (0, 0, 0), (16, 16, 16))
    blk = bench.tiled_block(t, (8, 0, 4), (8, 16, 4))
    assert np.array_equal(whole[8:8 + 14, :, 4:4 + 10], blk)
