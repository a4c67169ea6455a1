"""The reference-facing surface (IHD, GMGSolver, _utils, main_IHD_v3 functions,
objectives) run on the GPU and checked against the reference's golden vectors."""
import csv
import json
import os
from types import SimpleNamespace

import numpy as np
import pytest
import torch

from oracle import ihd_oracle as O

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def cfg(r):
    return SimpleNamespace(resolution=r, GMG=SimpleNamespace(smooth_iter=[2, 2, 3, 4, 5], max_cycle=1))


@pytest.fixture(scope="module")
def ihd8(lib):
    from maple_b200.model import IHD
    return IHD(cfg(8), DEV, rtol=1e-12)


def test_ihd_forward_matches_reference(ihd8, golden):
    from maple_b200.optimize import build_unitcell_batch
    from maple_b200.utils import assemble_F_fast, assemble_F_fast_scalar
    g = golden("homog_r8_s0.npz")
    rho = torch.tensor(1e-9 + (1 - 1e-9) * g["x"] ** 3, dtype=torch.float64, device=DEV).reshape(-1, 1)
    batch = build_unitcell_batch(DEV, 8, rho.reshape(8, 8, 8))
    batch["rho"] = rho
    Fm = assemble_F_fast(batch["node_index"], ihd8.Fe_3d, 512, rho)
    Ft = assemble_F_fast_scalar(batch["node_index"], ihd8.Fe_1d, 512, rho)
    assert rel(Fm.cpu().numpy(), g["F_elastic"]) < 1e-13
    assert rel(Ft.cpu().numpy(), g["F_thermal"]) < 1e-13
    CH = ihd8.TO_homo_3d(batch, ihd8.Ke_3d, Fm, ihd8.X0_3d, batch_size=1)
    kap = ihd8.TO_homo_1d(batch, ihd8.Ke_1d, Ft, ihd8.X0_1d, batch_size=1)
    assert CH.shape == (6, 6) and kap.shape == (3, 3)
    assert rel(CH.cpu().numpy(), g["CH"]) < 1e-10
    assert rel(kap.cpu().numpy(), g["kappa"]) < 1e-10


@pytest.mark.parametrize("tag,spec", [("bi", "stiffness:0.5,thermal:0.5"),
                                      ("tri", "stiffness:0.3333333333333333,shear:0.3333333333333333,"
                                              "thermal:0.3333333333333333")])
def test_ihd_autograd_matches_reference(ihd8, golden, tag, spec):
    """dJ/dx through IHD.TO_homo_* (analytic adjoint in backward) equals the
    reference's autograd through converged solves (main_IHD_v3.py:622-688)."""
    from maple_b200.objective import objective_from_spec
    from maple_b200.optimize import build_unitcell_batch
    g = golden("homog_r8_s0.npz")
    x = torch.tensor(g["x"], dtype=torch.float64, device=DEV).reshape(-1, 1).requires_grad_(True)
    rho = 1e-9 + (1 - 1e-9) * x.clamp(1e-3, 1.0) ** 3
    batch = build_unitcell_batch(DEV, 8, torch.zeros(8, 8, 8, device=DEV))
    batch["rho"] = rho
    kap = ihd8.TO_homo_1d(batch, ihd8.Ke_1d, None, ihd8.X0_1d, batch_size=1)
    CH = ihd8.TO_homo_3d(batch, ihd8.Ke_3d, None, ihd8.X0_3d, batch_size=1)
    J = objective_from_spec(obj=spec, CH=CH, kappa=kap)
    (dJdx,) = torch.autograd.grad(J, x)
    assert abs(J.item() - float(g[f"J_{tag}"])) / abs(J.item()) < 1e-10
    assert rel(dJdx.cpu().numpy().reshape(-1), g[f"dJdx_{tag}"]) < 1e-8


def test_evaluate_terms_and_J(ihd8, golden):
    from maple_b200.optimize import build_unitcell_batch, evaluate_homogenized_terms, evaluate_J
    g = golden("homog_r8_s1.npz")
    rho = torch.tensor(1e-9 + (1 - 1e-9) * g["x"] ** 3, dtype=torch.float64, device=DEV).reshape(-1, 1)
    batch = build_unitcell_batch(DEV, 8, rho.reshape(8, 8, 8))
    terms = evaluate_homogenized_terms(ihd8, batch, rho)
    assert abs(terms["stiffness"] - O.stiffness_objective(g["CH"])) < 1e-10 * abs(terms["stiffness"])
    assert abs(terms["shear"] - O.shear_objective(g["CH"])) < 1e-10 * abs(terms["shear"])
    assert abs(terms["thermal"] - O.thermal_objective(g["kappa"])) < 1e-10 * abs(terms["thermal"])
    J = evaluate_J(ihd8, batch, rho, "0.4*stiffness+0.6*thermal")
    ref = 0.4 * O.stiffness_objective(g["CH"]) + 0.6 * O.thermal_objective(g["kappa"])
    assert abs(J - ref) < 1e-10 * abs(ref)


@pytest.mark.parametrize("solver,d", [("GMGSolver", 3), ("GMGSolverScalar", 1)])
def test_gmg_solver_dropin(lib, golden, solver, d):
    """GMGSolver.solve with the reference's arguments (fine_ke = rho_e Ke0)."""
    from maple_b200 import gmg
    from maple_b200.optimize import build_unitcell_batch
    from maple_b200.utils import hexahedron, hexahedron_scalar, isotropic_elastic_tensor
    g = golden("homog_r8_s0.npz")
    rho = torch.tensor(1e-9 + (1 - 1e-9) * g["x"] ** 3, dtype=torch.float64, device=DEV)
    batch = build_unitcell_batch(DEV, 8, rho.reshape(8, 8, 8))
    if d == 3:
        Ke, Fe, _ = hexahedron(8, isotropic_elastic_tensor(1.0, 0.3).double().to(DEV))
        f = torch.tensor(g["F_elastic"][:, :, 2], device=DEV)          # load case 2, (N,3)
    else:
        Ke, Fe, _ = hexahedron_scalar(8, torch.tensor(1.0, dtype=torch.float64, device=DEV))
        f = torch.tensor(g["F_thermal"][:, 1], device=DEV)             # load case 1, (N,)
    fine_ke = Ke.unsqueeze(0).expand(512, -1, -1) * rho.reshape(-1, 1, 1)
    u, r = getattr(gmg, solver)().solve(fine_ke, f, batch["coord"].int(), batch["elem_coords"], batch["node_index"],
                                        max_iter=1, smooth_iter=[2, 2, 3, 4, 5], max_levels=5, dtype=torch.float64)
    assert u.shape == (512, d) and r.shape == (512, d)
    assert float(r.norm() / f.norm()) < 1e-9
    if d == 3:
        ug = g["u_elastic"][:, :, 2]
    else:
        ug = g["u_thermal"][:, 1:2]
    un = u.cpu().numpy()
    du = (un - un.mean(0)) - (ug - ug.mean(0))
    assert np.abs(du).max() / np.abs(ug).max() < 1e-8
    with pytest.raises(ValueError):
        bad = fine_ke.clone()
        bad[0, 0, 1] += 1.0
        getattr(gmg, solver)().solve(bad, f, batch["coord"].int(), batch["elem_coords"], batch["node_index"])


def test_filter_and_oc_dropins(lib, golden):
    from maple_b200.optimize import avg_filter3d_x_periodic, build_unitcell_batch, oc_update
    g = golden("ops.npz")
    batch = build_unitcell_batch(DEV, 8, torch.zeros(8, 8, 8, device=DEV))
    v = torch.tensor(g["filter_r8_k3_in"], device=DEV).reshape(-1, 1)
    out = avg_filter3d_x_periodic(v, batch["elem_coords"], 8, 3)
    assert out.shape == (512, 1)
    assert rel(out.cpu().numpy().reshape(-1), g["filter_r8_k3_out"]) < 1e-14
    with pytest.raises(ValueError):
        avg_filter3d_x_periodic(v, batch["elem_coords"], 8, 2)
    for i in range(3):
        vf, move, xmin = g[f"oc{i}_params"]
        xn = oc_update(torch.tensor(g[f"oc{i}_x"], device=DEV).reshape(-1, 1),
                       torch.tensor(g[f"oc{i}_dJ"], device=DEV).reshape(-1, 1), volfrac=vf, move=move, xmin=xmin)
        assert np.abs(xn.cpu().numpy().reshape(-1) - g[f"oc{i}_xnew"]).max() < 1e-10


def test_optimize_inverse_homogenization(ihd8, golden, tmp_path):
    """Three OC iterations through the reference's optimizer signature follow
    the reference trajectory, with the reference's output files."""
    from maple_b200.optimize import build_unitcell_batch, optimize_inverse_homogenization
    g = golden("traj_r8.npz")
    batch = build_unitcell_batch(DEV, 8, torch.zeros(8, 8, 8, device=DEV))
    res = optimize_inverse_homogenization(
        ihd8, batch, res=8, objective="stiffness:0.5,thermal:0.5", init_mode="noise", volfrac=0.25, penal=3.0,
        rho_min=1e-9, move=0.2, xmin=1e-3, iters=3, seed=0, symmetry="none", lambda_print=0.0, overhang_deg=45.0,
        lambda_cavity=0.0, cavity_thresh=0.5, cavity_beta=20.0, min_channel_rad=0, cavity_rad=1,
        cavity_seed_faces="all", cavity_iters=128, cavity_tiles=1, cavity_tiles_xyz=None, cavity_focus_center=True,
        filter_k=3, output_dir=str(tmp_path), mesh_every=0, mesh_res=32, mesh_iso=0.3, mesh_pad=2,
        save_initial_mesh=False, verbose=False, x_init=torch.tensor(g["x0"]), rtol=1e-12)
    assert res.iters_run == 3
    rows = list(csv.reader(open(os.path.join(tmp_path, "iter_log.csv"))))
    assert rows[0] == ["iter", "J_total", "J_raw", "P_print", "P_cavity", "mean_x", "mean_rho", "dx_max", "dx_mean",
                       "time_sec"]
    for it in range(3):
        assert abs(float(rows[1 + it][2]) - float(g[f"J{it}"])) / float(g[f"J{it}"]) < 1e-9
    summary = json.load(open(os.path.join(tmp_path, "summary.json")))
    assert summary["iters_run"] == 3 and summary["resolution"] == 8
    rho_final = np.load(os.path.join(tmp_path, "rho_final.npy"))
    ref = (1e-9 + (1 - 1e-9) * g["x3"] ** 3).reshape(8, 8, 8).astype(np.float32)
    assert rho_final.shape == (8, 8, 8) and np.abs(rho_final - ref).max() < 1e-6


def test_batched_cells_match_single_cell_runs(lib):
    """B cells with different volume fractions and weights advanced together
    follow the same trajectories as one-cell runs, and stop independently."""
    from maple_b200.batch import oc_run, seeded_design
    r, B = 8, 4
    rng = np.random.default_rng(5)
    vf = np.array([0.1, 0.2, 0.3, 0.35])
    w = rng.dirichlet((1, 1, 1), B)
    x0 = np.stack([seeded_design(b, r, 1.5, vf[b]).reshape(-1) for b in range(B)])
    res = oc_run(x0, w, vf, precision="fp64", rtol=1e-12, max_iters=3, dx_tol=0.0)
    assert (res.iters_run == 3).all()
    for b in range(B):
        one = oc_run(x0[b:b + 1], w[b:b + 1], vf[b:b + 1], precision="fp64", rtol=1e-12, max_iters=3, dx_tol=0.0)
        assert abs(one.J[0] - res.J[b]) <= 1e-10 * abs(one.J[0])
        assert np.abs(one.x.cpu().numpy() - res.x[b:b + 1].cpu().numpy()).max() < 1e-9
    # independent stopping: a loose tolerance stops cells at different iterations
    res2 = oc_run(x0, w, vf, precision="mixed", rtol=1e-8, max_iters=40, dx_tol=0.02)
    assert res2.converged.any()
    assert (res2.iters_run <= 40).all() and (res2.iters_run >= 1).all()


def test_optimize_with_symmetry_follows_reference(ihd8, golden, tmp_path):
    """optimize_inverse_homogenization with symmetry "iso" (the cube group)
    runs the reference's projected OC loop."""
    from maple_b200.optimize import build_unitcell_batch, optimize_inverse_homogenization
    g = golden("sym.npz")
    batch = build_unitcell_batch(DEV, 8, torch.zeros(8, 8, 8, device=DEV))
    res = optimize_inverse_homogenization(
        ihd8, batch, res=8, objective="stiffness:0.5,thermal:0.5", init_mode="noise", volfrac=0.25, penal=3.0,
        rho_min=1e-9, move=0.2, xmin=1e-3, iters=3, seed=0, symmetry="iso", lambda_print=0.0, overhang_deg=45.0,
        lambda_cavity=0.0, cavity_thresh=0.5, cavity_beta=20.0, min_channel_rad=0, cavity_rad=1,
        cavity_seed_faces="all", cavity_iters=128, cavity_tiles=1, cavity_tiles_xyz=None, cavity_focus_center=True,
        filter_k=3, output_dir=str(tmp_path), mesh_every=0, mesh_res=32, mesh_iso=0.3, mesh_pad=2,
        save_initial_mesh=False, verbose=False, x_init=torch.tensor(g["traj_cubic_x0"]), rtol=1e-12)
    rows = list(csv.reader(open(os.path.join(tmp_path, "iter_log.csv"))))
    for it in range(3):
        ref = float(g[f"traj_cubic_J{it}"])
        assert abs(float(rows[1 + it][2]) - ref) < 1e-8 * ref
    assert res.iters_run == 3
    assert ihd8.homog_ctx is not None


def test_checkpoint_resume_repeats_the_run(lib, tmp_path):
    """A batched OC run interrupted after 3 iterations and resumed from its
    checkpoint (with the solver fields) ends exactly where the uninterrupted
    6-iteration run ends; without the fields the resumed solves start from
    zero and agree to the solver tolerance."""
    import os
    from maple_b200.batch import oc_run, seeded_design
    r = 16
    x0 = np.stack([seeded_design(s, r, 2.0, 0.3).reshape(-1) for s in (0, 1)])
    w = np.array([[0.5, 0.0, 0.5], [0.2, 0.3, 0.5]])
    vf = np.array([0.3, 0.3])
    kw = dict(precision="mixed", rtol=1e-10, stop_rule="reference", move=0.2)
    full = oc_run(x0, w, vf, max_iters=6, **kw)
    for fields in (True, False):
        path = os.path.join(tmp_path, f"ck_{fields}.npz")
        part = oc_run(x0, w, vf, max_iters=3, checkpoint=path, checkpoint_every=1, checkpoint_fields=fields, **kw)
        assert list(part.iters_run) == [3, 3]
        res = oc_run(x0, w, vf, max_iters=6, checkpoint=path, checkpoint_every=2, resume=True,
                     checkpoint_fields=fields, **kw)
        assert list(res.iters_run) == list(full.iters_run) == [6, 6]
        if fields:
            np.testing.assert_array_equal(res.x.cpu().numpy(), full.x.cpu().numpy())
            np.testing.assert_array_equal(res.J, full.J)
        else:
            np.testing.assert_allclose(res.x.cpu().numpy(), full.x.cpu().numpy(), rtol=0, atol=1e-7)
            np.testing.assert_allclose(res.J, full.J, rtol=1e-8)


@pytest.mark.parametrize("solver,d,R", [("GMGSolver", 3, 6), ("GMGSolverScalar", 1, 3)])
def test_gmg_solver_load_cases_share_one_solve(lib, golden, solver, d, R):
    """The reference's homogenization calls GMGSolver.solve once per load case
    (utils/model.py:111-124).  The first call solves every load case of the
    density; the others return the stored columns (one kernel launch, the
    right-hand side check), each equal to the reference's solution.  Any other
    right-hand side is still solved."""
    from maple_b200 import gmg
    from maple_b200.core import launch_count
    from maple_b200.optimize import build_unitcell_batch
    from maple_b200.utils import hexahedron, hexahedron_scalar, isotropic_elastic_tensor
    g = golden("homog_r8_s0.npz")
    rho = torch.tensor(1e-9 + (1 - 1e-9) * g["x"] ** 3, dtype=torch.float64, device=DEV)
    batch = build_unitcell_batch(DEV, 8, rho.reshape(8, 8, 8))
    if d == 3:
        Ke, _, _ = hexahedron(8, isotropic_elastic_tensor(1.0, 0.3).double().to(DEV))
        Fs = [torch.tensor(g["F_elastic"][:, :, i], device=DEV) for i in range(R)]
        Us = [g["u_elastic"][:, :, i] for i in range(R)]
    else:
        Ke, _, _ = hexahedron_scalar(8, torch.tensor(1.0, dtype=torch.float64, device=DEV))
        Fs = [torch.tensor(g["F_thermal"][:, i], device=DEV) for i in range(R)]
        Us = [g["u_thermal"][:, i:i + 1] for i in range(R)]
    fine_ke = Ke.unsqueeze(0).expand(512, -1, -1) * rho.reshape(-1, 1, 1)
    s = getattr(gmg, solver)()
    args = (batch["coord"].int(), batch["elem_coords"], batch["node_index"])
    launches = []
    for i in range(R):
        l0 = launch_count()
        u, r = s.solve(fine_ke, Fs[i], *args, dtype=torch.float64)
        torch.cuda.synchronize()
        launches.append(launch_count() - l0)
        un = u.cpu().numpy().reshape(512, d)
        du = (un - un.mean(0)) - (Us[i] - Us[i].mean(0))
        assert np.abs(du).max() / np.abs(Us[i]).max() < 1e-8, i
        assert float(r.norm() / Fs[i].norm()) < 1e-9
    assert launches[0] > 10 and all(n == 1 for n in launches[1:]), launches
    other = 0.5 * Fs[0] + 0.25 * Fs[R - 1]
    u, r = s.solve(fine_ke, other, *args, dtype=torch.float64)
    assert float(r.norm() / other.norm()) < 1e-9


def test_gmg_solver_per_level_init_list(lib, golden):
    """The reference's init_list hook: per-level fields ordered coarse to fine,
    as sparse tensors (.indices [b,x,y,z], .features) aligned by coordinates.
    A field at the fine level is the initial iterate; a coarse level's is
    prolonged to the fine grid first.  Either way the solve reaches the
    reference's solution."""
    import types
    from maple_b200 import gmg
    from maple_b200.optimize import build_unitcell_batch
    from maple_b200.utils import hexahedron, isotropic_elastic_tensor
    g = golden("homog_r8_s0.npz")
    rho = torch.tensor(1e-9 + (1 - 1e-9) * g["x"] ** 3, dtype=torch.float64, device=DEV)
    batch = build_unitcell_batch(DEV, 8, rho.reshape(8, 8, 8))
    Ke, _, _ = hexahedron(8, isotropic_elastic_tensor(1.0, 0.3).double().to(DEV))
    fine_ke = Ke.unsqueeze(0).expand(512, -1, -1) * rho.reshape(-1, 1, 1)
    f = torch.tensor(g["F_elastic"][:, :, 4], device=DEV)
    ug = g["u_elastic"][:, :, 4]
    args = (batch["coord"].int(), batch["elem_coords"], batch["node_index"])

    def sparse(n, field):
        xyz = torch.stack(torch.meshgrid(*[torch.arange(n, device=DEV)] * 3, indexing="ij"), -1).reshape(-1, 3)
        idx = torch.cat([torch.zeros((n ** 3, 1), dtype=torch.long, device=DEV), xyz], 1)
        feats = torch.cat([torch.as_tensor(field, device=DEV).reshape(n ** 3, 3),
                           torch.zeros((n ** 3, 2), dtype=torch.float64, device=DEV)], 1)  # extra channels
        return types.SimpleNamespace(indices=idx, features=feats)

    def check(u):
        un = u.cpu().numpy()
        du = (un - un.mean(0)) - (ug - ug.mean(0))
        assert np.abs(du).max() / np.abs(ug).max() < 1e-8

    s = gmg.GMGSolver()
    u, r = s.solve(fine_ke, f, *args, init_list=[None, sparse(8, ug)], dtype=torch.float64)
    check(u)
    coarse = ug.reshape(8, 8, 8, 3)[::2, ::2, ::2]  # injection to the 4^3 level
    u, r = s.solve(fine_ke, f, *args, init_list=[sparse(4, coarse), None], init_is_solution=True,
                   dtype=torch.float64)
    check(u)
    with pytest.raises(ValueError):
        s.solve(fine_ke, f, *args, init_list=[torch.zeros(10, dtype=torch.float64, device=DEV), None])
