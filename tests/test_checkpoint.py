"""Checkpoint files: the reference drivers' content (one dataset per primitive name over the
global interior, JSON status) as raw .bin + JSON; round trip back to a guarded array."""
import json
import os

import numpy as np

from ctf_b200 import checkpoint, ics


def test_round_trip_3d(tmp_path):
    P = ics.turbulence_box((12, 10, 8), seed=3)
    path = str(tmp_path / "chkpt.0007")
    checkpoint.write(path, P, 3, status={"iteration": 7, "time": 0.25}, measure_log=[{"t": 0.0}],
                     model_parameters={"vrms": 0.3})
    Q, meta = checkpoint.read(path)
    assert Q.shape == (18, 16, 14, 8)
    assert np.array_equal(Q, P)                   # the generator's guards are periodic too
    assert meta["status"]["iteration"] == 7 and meta["prim_names"][0] == "rho"
    assert sorted(os.listdir(os.path.join(path, "prim"))) == sorted(n + ".bin" for n in checkpoint.PRIM_NAMES)
    rho = np.fromfile(os.path.join(path, "prim", "rho.bin")).reshape(12, 10, 8)
    assert np.array_equal(rho, P[3:-3, 3:-3, 3:-3, 0])
    assert json.load(open(os.path.join(path, "checkpoint.json")))["model_parameters"] == {"vrms": 0.3}


def test_round_trip_2d_solver_layout(tmp_path):
    P = ics.kh_box((16, 12), seed=4)              # the Solver layout (22, 18, 1, 8)
    path = str(tmp_path / "c")
    checkpoint.write(path, P, 2)
    Q, _ = checkpoint.read(path)
    assert Q.shape == (22, 18, 1, 8) and np.array_equal(Q, P)
    assert np.fromfile(os.path.join(path, "prim", "vy.bin")).size == 16 * 12
