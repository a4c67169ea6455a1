"""Failure detection on the GPU without any GPU fault.

Faults are made on the host: a NaN element density in one cell of a batch, a
non-finite or a garbage initial iterate (a broken learned guess), an iteration
cap.  The tests check the per-cell status words, the plain-FP64 fallback of a
mixed-precision breakdown and that the other cells of the batch are untouched
(bit-for-bit the result of solving them alone)."""
import numpy as np
import pytest
import torch

from oracle import ihd_oracle as O

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
R_CELL = 16
CONV, BRK, MAXIT, FB = 1, 2, 4, 8


def _rho(seeds):
    x = np.stack([O.seed_density(s, R_CELL, 2.0, 0.3).reshape(-1) for s in seeds])
    return 1e-9 + (1.0 - 1e-9) * x ** 3


def _solve(rho, prec, phys="elastic", guess=None, maxit=300):
    from maple_b200.core import HomogenizationContext
    c = HomogenizationContext(R_CELL, ncells=len(rho), device=DEV)
    c.set_density(phys, torch.tensor(rho, dtype=torch.float64, device=DEV).contiguous(), prec)
    if guess is not None:
        c.set_solution(phys, guess)
    info = c.solve(phys, prec, rtol=1e-10, maxit=maxit, warm=guess is not None)
    H = c.homogenize(phys).cpu().numpy()
    c.close()
    return info, H


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
@pytest.mark.parametrize("phys", ["elastic", "thermal"])
def test_nan_density_is_reported_and_isolated(lib, prec, phys):
    rho = _rho((0, 1))
    rho[1, 123] = np.nan
    info, H = _solve(rho, prec, phys)
    assert info.status[0] == CONV
    assert info.status[1] & BRK and not info.status[1] & CONV
    assert bool(info.status[1] & FB) == (prec == "mixed")  # the FP64 retry breaks down as well
    alone, H0 = _solve(rho[:1], prec, phys)
    assert alone.status[0] == CONV and info.iters[0] == alone.iters[0]
    np.testing.assert_array_equal(H[0], H0[0])


def test_nonfinite_guess_falls_back_to_fp64(lib):
    from maple_b200.core import HomogenizationContext
    rho = _rho((2, 3))
    shape = (2, 6, 3, R_CELL ** 3)
    guess = torch.zeros(shape, dtype=torch.float64, device=DEV)
    guess[1, 2, 1, 77] = float("nan")
    info, H = _solve(rho, "mixed", guess=guess)
    assert info.status[0] == CONV
    assert info.status[1] == CONV | FB, info.status
    ref0, Hm = _solve(rho[:1], "mixed")
    np.testing.assert_array_equal(H[0], Hm[0])
    ref1, H64 = _solve(rho[1:], "fp64")
    assert _rel(H[1], H64[0]) < 1e-12
    assert info.iters[1] > ref1.iters[0]  # the broken mixed attempt counts too
    del HomogenizationContext


def test_garbage_finite_guess_recovers(lib):
    """A finite but wild initial iterate (1e6 x N(0,1)) puts rtol 1e-10 beyond
    the attainable accuracy from it: the mixed solve and the FP64 retry from
    the same iterate break down, the FP64 retry from zero converges."""
    rho = _rho((4, 5))
    g = torch.zeros((2, 3, 1, R_CELL ** 3), dtype=torch.float64, device=DEV)
    g[1] = torch.randn((3, 1, R_CELL ** 3), dtype=torch.float64, device=DEV, generator=torch.Generator(DEV).manual_seed(0)) * 1e6
    info, H = _solve(rho, "mixed", phys="thermal", guess=g)
    assert info.status[0] == CONV
    assert info.status[1] == CONV | FB, info.status
    _, Hz = _solve(rho, "mixed", phys="thermal")
    np.testing.assert_array_equal(H[0], Hz[0])
    _, H64 = _solve(rho[1:], "fp64", phys="thermal")
    assert _rel(H[1], H64[0]) < 1e-12


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_iteration_cap_reports_maxit(lib, prec):
    info, _ = _solve(_rho((6, 7)), prec, maxit=2)
    assert list(info.status) == [MAXIT, MAXIT] and list(info.iters) == [2, 2]


def _oc_inputs(B, N, seed=3):
    rng = np.random.default_rng(seed)
    x = np.clip(0.25 + 0.2 * rng.standard_normal((B, N)), 1e-3, 1.0)
    dJ = np.abs(rng.standard_normal((B, N))) * 1e-2
    return (torch.tensor(x, device=DEV), torch.tensor(dJ, device=DEV),
            torch.tensor(np.full(B, 0.25), device=DEV))


def test_oc_barrier_wait_runs_out_and_is_reported(lib):
    """The OC bisection runs as one cooperative launch whose blocks meet at grid
    barriers, each wait bounded by a poll limit.  A phantom block that never
    arrives (maple_test_wait_limit) makes every wait run out: maple_oc_update
    and maple_oc_step must return MAPLE_E_TIMEOUT instead of hanging or
    reporting success, and the context must give the normal result afterwards."""
    from maple_b200 import _lib
    from maple_b200.core import HomogenizationContext
    r, B = 8, 2
    N = r ** 3
    ctx = HomogenizationContext(r, ncells=B, device=DEV)
    x, dJ, vf = _oc_inputs(B, N)
    good, good_stats = ctx.oc_update(x, dJ, vf, move=0.2, xmin=1e-3)
    good, good_stats = good.cpu().numpy(), good_stats.cpu().numpy()
    w = torch.tensor([[0.5, 0.0, 0.5]] * B, dtype=torch.float64, device=DEV)
    _lib.check(lib.maple_test_wait_limit(1 << 12, 1))
    try:
        with pytest.raises(_lib.MapleError) as e:
            ctx.oc_update(x, dJ, vf, move=0.2, xmin=1e-3)
        assert e.value.code == _lib.MAPLE_E_TIMEOUT
        assert "grid barrier" in str(e.value)
        with pytest.raises(_lib.MapleError, match="grid barrier") as e:
            ctx.oc_step(x, w, vf, precision="fp64", rtol=1e-8)
        assert e.value.code == _lib.MAPLE_E_TIMEOUT
    finally:
        _lib.check(lib.maple_test_wait_limit(0, 0))
    again, again_stats = ctx.oc_update(x, dJ, vf, move=0.2, xmin=1e-3)
    np.testing.assert_array_equal(again.cpu().numpy(), good)
    np.testing.assert_array_equal(again_stats.cpu().numpy(), good_stats)
    ctx.close()
