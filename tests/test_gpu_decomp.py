"""The decomposed advance on one GPU: every rank's block in this process (the blocks' stream
plus a side stream for the slabs, copied directly), phase by phase with the guard exchange
between c2p and the sweeps -- overlapped with the cores' c2p, or after the whole c2p --
against the single-box solver of the whole domain.  Power-of-two boxes on the unit cube keep
each block's spacing (local extent / local zones, as the reference's decomposed domain
computes it) bitwise equal to the whole box's, so the comparison is exact."""
import numpy as np
import pytest

from ctf_b200 import ics
from ctf_b200.decomp import DecomposedSolver, Layout
from ctf_b200.mara import Scheme, Solver

pytestmark = pytest.mark.gpu


def single(scheme, n, P0, dts):
    s = Solver(scheme, n)
    s.upload(P0.copy())
    errs = [s.advance(0.0)] + [s.advance(dt) for dt in dts]
    out = s.download()
    s.close()
    return out, errs


def decomposed(scheme, n, dims, P0, dts, overlap=True):
    L = Layout(N=n, dims=dims, x0=(0.0,) * len(n), x1=(1.0,) * len(n))
    D = DecomposedSolver(scheme, L, ranks=range(dims[0] * dims[1] * dims[2]), overlap=overlap)
    D.upload_global(P0)
    D.advance(dt=0.0)
    errs = [D.errors()]
    for dt in dts:
        D.advance(dt=dt)
        errs.append(D.errors())
    out = D.download_global()
    return D, out, errs


@pytest.mark.parametrize("overlap", [True, False])
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("dims", [(2, 1, 1), (1, 2, 1), (2, 2, 1), (1, 2, 2), (2, 2, 2)])
def test_decomposed_3d_matches_the_whole_box(dims, precision, overlap):
    n = (16, 16, 16)
    scheme = Scheme(extrap="plm", riemann="hlld", advance="rk2", precision=precision)
    P0 = ics.turbulence_box(n, seed=81)
    s = Solver(scheme, n)
    s.upload(P0.copy())
    s.advance(0.0)
    dt = s.get_timestep(0.3)
    s.close()
    ref, e1 = single(scheme, n, P0, [dt] * 4)
    D, got, e2 = decomposed(scheme, n, dims, P0, [dt] * 4, overlap)
    assert e1 == e2 == [0] * 5
    assert np.array_equal(got, ref), np.abs(got - ref).max()
    D.close()


@pytest.mark.parametrize("dims", [(2, 1, 1), (1, 2, 2), (2, 2, 2)])
@pytest.mark.parametrize("learned", [False, True])
def test_decomposed_lean_layout_matches_the_whole_box(dims, learned):
    """The lean layout (FP32 bulk; the layout of the 1024^3 boxes) decomposed: each block's
    stage primitives get their split guards from the exchange at every stage (the first
    stage's are the committed ones), the corner EMFs read the face fields of one halo row, and
    the blocks together give the whole lean box bit for bit, MaxLambda included."""
    from ctf_b200.train_c2p import load as load_net
    n = (16, 16, 16)
    scheme = Scheme(extrap="weno5", riemann="hlld", advance="rk3", precision="fp32", layout="lean",
                    learned_c2p=learned)
    P0 = ics.turbulence_box(n, seed=84)
    s = Solver(scheme, n)
    if learned:
        s.set_c2p_network(load_net())
    s.upload(P0.copy())
    assert s.advance(0.0) == 0
    dt = s.get_timestep(0.3)
    errs = [s.advance(dt) for _ in range(3)]
    ml = s.max_lambda
    ref = s.download()
    s.close()
    L = Layout(N=n, dims=dims, x0=(0.0,) * 3, x1=(1.0,) * 3)
    D = DecomposedSolver(scheme, L, ranks=range(dims[0] * dims[1] * dims[2]))
    if learned:
        for b in D.blocks:
            b.solver.set_c2p_network(load_net())
    D.upload_global(P0)
    D.advance(dt=0.0)
    assert D.errors() == 0
    for _ in range(3):
        D.advance(dt=dt)
        assert D.errors() == 0
    assert errs == [0, 0, 0]
    got = D.download_global()
    assert np.array_equal(got, ref), np.abs(got - ref).max()
    assert all(b.solver.max_lambda == ml for b in D.blocks)
    D.close()


def test_decomposed_2d_weno5_hllc_rk3():
    n = (32, 16)
    scheme = Scheme(extrap="weno5", riemann="hllc", advance="rk3")
    P0 = ics.kh_box(n, seed=82)
    ref, _ = single(scheme, n, P0, [2e-3] * 3)
    D, got, errs = decomposed(scheme, n, (4, 2, 1), P0, [2e-3] * 3)
    assert errs == [0] * 4
    assert np.array_equal(got, ref)
    D.close()


def test_global_cfl_step_uses_the_maximum_over_ranks():
    n = (16, 16, 16)
    scheme = Scheme()
    P0 = ics.turbulence_box(n, seed=83)
    L = Layout(N=n, dims=(2, 2, 1), x0=(0.0,) * 3, x1=(1.0,) * 3)
    D = DecomposedSolver(scheme, L, ranks=range(4))
    D.upload_global(P0)
    D.advance(dt=0.0)
    assert D.errors() == 0
    mls = [b.solver.max_lambda for b in D.blocks]
    assert len(set(mls)) == 1 and mls[0] > 0
    dt = D.get_timestep(0.3)
    assert dt == pytest.approx(0.3 * (1.0 / 16) / mls[0], rel=1e-15)
    for _ in range(3):
        D.advance(cfl=0.3)
        assert D.errors() == 0
    D.close()


def test_a_failure_anywhere_aborts_every_block(golden):
    """The reference's HLLC failure case split over two blocks: the third step fails, every
    block reports the same summed count, and no block commits."""
    g = golden("step_hllc_fail_12.npz")
    n = (12, 12, 12)
    scheme = Scheme(extrap="plm", riemann="hllc", advance="rk3")
    L = Layout(N=n, dims=(2, 1, 1), x0=(0.0,) * 3, x1=(1.0,) * 3)
    D = DecomposedSolver(scheme, L, ranks=range(2))
    D.upload_global(g["P0"])
    D.advance(dt=0.0)
    assert D.errors() == 0
    for k, dt in enumerate(g["dts"]):
        before = D.download_global()
        D.advance(dt=float(dt))
        e = D.errors()
        if g["errors"][k + 1]:
            assert e > 0
            assert all(int(b.errs.cpu()[k]) == e for b in D.blocks) or all(
                b.solver.stats()["errors"] == e for b in D.blocks)
            assert all(b.solver.stats()["committed"] == 0 for b in D.blocks)
            assert np.array_equal(D.download_global(), before)
            break
        assert e == 0
    else:
        pytest.fail("the fixture's failing step did not fail")
    D.close()
