"""Driven turbulence on the GPU against the reference: the same OU field (serialized by the
reference's Mara.new_ou_field), the same sequence of Mara.advance / driving.Advance /
driving.Resample, states compared after every step."""
import numpy as np
import pytest

from ctf_b200 import ics
from ctf_b200.mara import Scheme, Solver, new_ou_field

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("fp32", 5e-3)])   # FP32: the L-inf bound of test_gpu_fp32
def test_driven_box_matches_the_reference(precision, tol):
    from oracle import RefOracle, Scheme as OScheme
    n = (12, 12, 12)
    P = ics.turbulence_box(n, seed=91, vrms=0.1)
    field = new_ou_field(3, 0.5, 1.0, 3, 12345)          # strong forcing: visible in 6 steps
    ref = RefOracle(OScheme(n=n, extrap="plm", riemann="hlld", advance="rk2"))
    g = Solver(Scheme(extrap="plm", riemann="hlld", advance="rk2", precision=precision), n)
    import os
    import tempfile
    d = tempfile.mkdtemp()
    open(os.path.join(d, "f.bin"), "wb").write(field)
    ref.dostring(f"local f = io.open('{d}/f.bin', 'rb'); Mara.set_driving(f:read('*a')); f:close()")
    g.set_driving(field)
    Pr = P.copy()
    g.upload(P.copy())
    assert ref.advance(Pr, 0.0) == 0 and g.advance(0.0) == 0
    for step in range(6):
        dt = ref.get_timestep(0.3)
        # OU step of the modes, resample every other step, then the driven advance
        ref.dostring(f"Mara.driving.Advance({dt!r})")
        g.driving_advance(dt)
        if step % 2 == 0:
            ref.dostring("Mara.driving.Resample()")
            g.driving_resample()
        assert ref.advance(Pr, dt) == 0 and g.advance(dt) == 0
        Pg = g.download()
        err = np.abs(Pg - Pr).max() / np.abs(Pr).max()
        assert err <= tol, (step, err)
    assert g.driving_serialize() != field                  # the modes moved
    ref.dostring(f"local f = io.open('{d}/p.txt', 'w'); f:write(string.format('%.17g', Mara.driving.Power())); f:close()")
    ref.close()
    pr = float(open(os.path.join(d, "p.txt")).read())
    assert pr > 0 and abs(g.driving_power() - pr) <= 1e-10 * pr


def test_driving_kicks_only_committed_advances(golden):
    """A failing advance (the HLLC failure fixture) leaves the state undriven and unchanged."""
    gd = golden("step_hllc_fail_12.npz")
    n = (12, 12, 12)
    s = Solver(Scheme(extrap="plm", riemann="hllc", advance="rk3"), n)
    field = new_ou_field(3, 0.5, 1.0, 3, 5)
    s.set_driving(field)
    s.driving_advance(0.01)
    s.driving_resample()
    s.upload(gd["P0"].copy())
    assert s.advance(0.0) == 0
    for k, dt in enumerate(gd["dts"]):
        s.upload(np.ascontiguousarray(gd["states"][k - 1]) if k else gd["P0"].copy())
        before = s.download()
        e = s.advance(float(dt))
        if e:
            assert np.array_equal(s.download(), before)
            return
    pytest.fail("the fixture's failing step did not fail")
