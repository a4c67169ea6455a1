"""Parity at the benchmark configurations, against fixtures recorded from the
reference (tests/golden/make_golden.py --only=config0 / config1).

* 32^3, plain FP64 method (seed 0, sigma 2, vf 0.25, J = 0.5 E + 0.5 kappa,
  move 0.2, 3^3 filter): 50 OC iterations follow the oracle trajectory, and
  the reference's own solvers at iterations 0, 1, 10, 25 and 49, to 1e-9.
* 64^3, precision configuration (seed 0, sigma 4, J = (E + G + kappa)/3):
  the mixed-precision path tracks the plain FP64 path over 20 OC iterations
  with every C^H, kappa^H and J within 1e-6 (relative), and meets the
  reference's C^H, kappa^H and J at iterations 0 and 1.
"""
import numpy as np
import pytest
import torch

from oracle import ihd_oracle as O

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
TOL = 1e-9      # the plain path against the reference
TOL_MIX = 1e-6  # the mixed path against the FP64 path and the reference
RTOL0 = 1e-12   # solver tolerance of the 50-iteration comparison


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / np.abs(np.asarray(b)).max())


def _run(ctx, x, w, vf, iters, precision, rtol, record=None):
    out = []
    for it in range(iters):
        o = ctx.oc_step(x, w, vf, penal=3.0, rho_min=1e-9, move=0.2, xmin=1e-3, filter_k=3, precision=precision,
                        rtol=rtol, maxit=1000, warm=True)
        out.append((o["CH"][0].cpu().numpy(), o["kappa"][0].cpu().numpy(), float(o["J"][0])))
        x = o["x_next"].clone()
        if record is not None:
            record[it + 1] = x[0].cpu().numpy()
    return out


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_config0_trajectory_matches_reference(lib, golden, precision):
    from maple_b200.core import HomogenizationContext
    g = golden("traj_r32.npz")
    r, iters = int(g["r"]), int(g["iters"])
    ctx = HomogenizationContext(r, ncells=1, device=DEV)
    x = torch.tensor(g["x0"][None], dtype=torch.float64, device=DEV)
    w = torch.tensor([[0.5, 0.0, 0.5]], dtype=torch.float64, device=DEV)
    vf = torch.tensor([float(g["vf"])], dtype=torch.float64, device=DEV)
    xs = {}
    traj = _run(ctx, x, w, vf, iters, precision, RTOL0, xs)
    ctx.close()
    eJ = max(abs(t[2] - J) / abs(J) for t, J in zip(traj, g["J"]))
    eC = max(rel(t[0], C) for t, C in zip(traj, g["CH"]))
    eK = max(rel(t[1], K) for t, K in zip(traj, g["kappa"]))
    assert max(eJ, eC, eK) < TOL, (eJ, eC, eK)
    for it in (1, 10, 25, 49, 50):
        assert np.abs(xs[it] - g[f"x{it}"]).max() < 1e-8, it
    for it in (0, 1, 10, 25, 49):  # the reference's own solvers at the oracle's designs
        assert abs(traj[it][2] - float(g[f"ref_J_{it}"])) < TOL * abs(float(g[f"ref_J_{it}"])), it
        assert rel(traj[it][0], g[f"ref_CH_{it}"]) < TOL, it
        assert rel(traj[it][1], g[f"ref_kappa_{it}"]) < TOL, it


def _config1_inputs():
    x0 = O.seed_density(0, 64, 4.0, 0.25).reshape(1, -1)
    w = torch.tensor([[1 / 3, 1 / 3, 1 / 3]], dtype=torch.float64, device=DEV)
    vf = torch.tensor([0.25], dtype=torch.float64, device=DEV)
    return torch.tensor(x0, dtype=torch.float64, device=DEV), w, vf


def test_config1_mixed_tracks_fp64_over_20_iterations(lib):
    from maple_b200.core import HomogenizationContext
    x, w, vf = _config1_inputs()
    runs = {}
    for prec in ("fp64", "mixed"):
        ctx = HomogenizationContext(64, ncells=1, device=DEV)
        runs[prec] = _run(ctx, x, w, vf, 20, prec, 1e-10)
        ctx.close()
    for it, (m, d) in enumerate(zip(runs["mixed"], runs["fp64"])):
        err = max(rel(m[0], d[0]), rel(m[1], d[1]), abs(m[2] - d[2]) / abs(d[2]))
        assert err <= TOL_MIX, (it, err)


def test_config1_spot_checks_against_reference(lib, golden):
    from maple_b200.core import HomogenizationContext
    g = golden("spot_r64.npz")
    x, w, vf = _config1_inputs()
    ctx = HomogenizationContext(64, ncells=1, device=DEV)
    xs = {}
    traj = _run(ctx, x, w, vf, 2, "mixed", 1e-10, xs)
    ctx.close()
    assert np.abs(xs[1] - g["x1"]).max() < 1e-8
    for it in (0, 1):
        assert abs(traj[it][2] - float(g[f"ref_J_{it}"])) <= TOL_MIX * abs(float(g[f"ref_J_{it}"])), it
        assert rel(traj[it][0], g[f"ref_CH_{it}"]) <= TOL_MIX, it
        assert rel(traj[it][1], g[f"ref_kappa_{it}"]) <= TOL_MIX, it
        assert rel(traj[it][0], g["CH"][it]) <= TOL_MIX, it  # the oracle at the same designs


def test_config0_batched_cell_follows_the_fixture(lib, golden):
    """The batching path: the 32^3 fixture cell advanced in one batch with two
    other cells (their own volume fractions and objective weights) follows
    the reference-pinned trajectory as the single-cell run does."""
    from maple_b200.batch import oc_run
    g = golden("traj_r32.npz")
    r, iters = int(g["r"]), 10
    x = np.stack([g["x0"], O.seed_density(7, r, 2.0, 0.1).reshape(-1), O.seed_density(8, r, 2.0, 0.35).reshape(-1)])
    w = np.array([[0.5, 0.0, 0.5], [0.2, 0.5, 0.3], [0.0, 1.0, 0.0]])
    vf = np.array([float(g["vf"]), 0.1, 0.35])
    res = oc_run(x, w, vf, r=r, precision="mixed", rtol=RTOL0, maxit=1000, dx_tol=-1.0, max_iters=iters,
                 record=True, device=DEV)
    assert list(res.iters_run) == [iters] * 3
    J0 = np.array([h["J"][0] for h in res.history])
    assert np.abs(J0 - g["J"][:iters]).max() < TOL * np.abs(g["J"][:iters]).max()
    assert np.abs(res.x[0].cpu().numpy() - g["x10"]).max() < 1e-8
