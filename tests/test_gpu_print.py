"""Manufacturability penalties on the GPU against the reference's own
penalties and autograd gradients (tests/golden/print.npz): every case on two
8^3 fields (one full of exact ties), the autograd drop-ins, a penalised fused
OC trajectory and the optimizer drop-in with the experiment scripts' weights."""
import csv
import json
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


def _settings(kind, kw):
    if kind == "over":
        return dict(lambda_print=1.0, overhang_deg=kw.get("overhang_deg", 45.0),
                    overhang_periodic=kw.get("periodic_xy", True))
    common = dict(lambda_cavity=1.0, void_thresh=kw.get("void_thresh", 0.5), beta=kw.get("beta", 20.0),
                  min_channel_rad=kw.get("min_channel_rad", 0), rad=kw.get("rad", 1), iters=kw.get("iters", 0),
                  seed_faces=kw.get("seed_faces", "all"))
    if kind == "closed":
        return dict(common, tiles=(1, 1, 1), periodic=kw.get("periodic_xyz", True))
    return dict(common, tiles=tuple(kw["tiles_xyz"]), focus_center=kw.get("focus_center", True), periodic=False)


def test_penalties_match_reference_autograd(lib, golden):
    from maple_b200.core import HomogenizationContext
    g = golden("print.npz")
    cases = [json.loads(c) for c in g["cases"]]
    ctx = HomogenizationContext(8, ncells=2, device=DEV)
    rho = torch.tensor(np.stack([g["field_cont"], g["field_simp"]]), dtype=torch.float64, device=DEV)
    for i, (kind, kw) in enumerate(cases):
        ctx.set_penalties(**_settings(kind, kw))
        over = kind == "over"
        out = ctx.penalties(rho, overhang=over, cavity=not over)
        P = (out["P_print"] if over else out["P_cavity"]).cpu().numpy()
        dP = (out["dP_print"] if over else out["dP_cavity"]).cpu().numpy()
        for b, f in enumerate(("cont", "simp")):
            ref_P, ref_g = g[f"{f}_{i}_P"], g[f"{f}_{i}_grad"]
            assert abs(P[b] - ref_P) <= 1e-13 * max(1.0, abs(ref_P)), (i, kind, kw, f)
            assert np.abs(dP[b] - ref_g).max() <= 1e-12 * max(1e-300, np.abs(ref_g).max()), (i, kind, kw, f)
    ctx.close()


def test_penalty_dropins_autograd(lib, golden):
    from maple_b200 import printability as Pr
    g = golden("print.npz")
    cases = [json.loads(c) for c in g["cases"]]
    for f in ("cont", "simp"):
        for i, (kind, kw) in enumerate(cases):
            rho = torch.tensor(g[f"field_{f}"].reshape(8, 8, 8), device=DEV, requires_grad=True)
            if kind == "over":
                P = Pr.printability_penalty_overhang(rho, **kw)
            elif kind == "closed":
                P = Pr.cavity_penalty_closed_void(rho, **kw)
            else:
                P = Pr.cavity_penalty_periodic_array(rho, **{k: tuple(v) if k == "tiles_xyz" else v
                                                             for k, v in kw.items()})
            (gr,) = torch.autograd.grad(3.0 * P, rho)
            assert abs(P.item() - g[f"{f}_{i}_P"]) <= 1e-13 * max(1.0, abs(g[f"{f}_{i}_P"]))
            ref = 3.0 * g[f"{f}_{i}_grad"]
            assert np.abs(gr.cpu().numpy().reshape(-1) - ref).max() <= 1e-12 * max(1e-300, np.abs(ref).max())
    with pytest.raises(ValueError):
        Pr.printability_penalty_overhang(torch.zeros(8, 8, 6, device=DEV))


TRAJ = dict(lambda_print=0.9, overhang_deg=45.0, lambda_cavity=0.9, void_thresh=0.5, beta=20.0, min_channel_rad=1,
            rad=1, iters=0, tiles=(2, 2, 2), focus_center=True, seed_faces="all")


def test_penalised_oc_step_trajectory(lib, golden):
    """Three fused OC steps with both penalties (the experiment scripts'
    weights) follow the reference: J_total, J_raw, both penalties, x."""
    from maple_b200.core import HomogenizationContext
    g = golden("print.npz")
    ctx = HomogenizationContext(8, ncells=1, device=DEV)
    ctx.set_penalties(**TRAJ)
    x = torch.tensor(g["traj_x0"].reshape(1, -1), device=DEV)
    w = torch.tensor([[0.5, 0.0, 0.5]], dtype=torch.float64, device=DEV)
    vf = torch.tensor([0.25], dtype=torch.float64, device=DEV)
    for it in range(3):
        out = ctx.oc_step(x, w, vf, precision="fp64", rtol=1e-12, warm=True)
        assert abs(float(out["J"][0]) - g[f"traj_J{it}"]) < 1e-8 * abs(g[f"traj_J{it}"]), it
        assert abs(float(out["J_raw"][0]) - g[f"traj_Jraw{it}"]) < 1e-8 * abs(g[f"traj_Jraw{it}"]), it
        assert abs(float(out["P_print"][0]) - g[f"traj_Pp{it}"]) < 1e-10, it
        assert abs(float(out["P_cavity"][0]) - g[f"traj_Pc{it}"]) < 1e-10, it
        assert np.abs(out["x_next"].cpu().numpy().reshape(-1) - g[f"traj_x{it + 1}"]).max() < 1e-7, it
        x = out["x_next"].clone()
    ctx.set_penalties(0.0, 45.0, 0.0)
    out = ctx.oc_step(x, w, vf, precision="fp64", rtol=1e-12, warm=True)
    assert float(out["P_print"][0]) == 0.0 or float(out["J"][0]) == float(out["J_raw"][0])
    ctx.close()


def test_optimize_with_penalties_follows_reference(golden, tmp_path, lib):
    from maple_b200.model import IHD
    from maple_b200.optimize import build_unitcell_batch, optimize_inverse_homogenization

    class Cfg:
        resolution = 8

        class GMG:
            smooth_iter = [2, 2, 3]
            max_cycle = 1

    g = golden("print.npz")
    ihd = IHD(Cfg, DEV, precision="fp64", rtol=1e-12)
    batch = build_unitcell_batch(DEV, 8, torch.zeros(8, 8, 8, device=DEV))
    res = optimize_inverse_homogenization(
        ihd, batch, res=8, objective="stiffness:0.5,thermal:0.5", init_mode="noise", volfrac=0.25, penal=3.0,
        rho_min=1e-9, move=0.2, xmin=1e-3, iters=3, seed=0, symmetry="none", lambda_print=0.9, overhang_deg=45.0,
        lambda_cavity=0.9, cavity_thresh=0.5, cavity_beta=20.0, min_channel_rad=1, cavity_rad=1,
        cavity_seed_faces="all", cavity_iters=0, cavity_tiles=2, cavity_tiles_xyz=None, cavity_focus_center=True,
        filter_k=3, output_dir=str(tmp_path), mesh_every=0, mesh_res=32, mesh_iso=0.3, mesh_pad=2,
        save_initial_mesh=False, verbose=False, x_init=torch.tensor(g["traj_x0"]), rtol=1e-12)
    rows = list(csv.reader(open(os.path.join(tmp_path, "iter_log.csv"))))
    for it in range(3):
        row = [float(v) for v in rows[1 + it][1:5]]
        ref = [g[f"traj_J{it}"], g[f"traj_Jraw{it}"], g[f"traj_Pp{it}"], g[f"traj_Pc{it}"]]
        assert abs(row[0] - ref[0]) < 1e-8 * abs(ref[0]) and abs(row[1] - ref[1]) < 1e-8 * abs(ref[1])
        assert abs(row[2] - ref[2]) < 1e-10 and abs(row[3] - ref[3]) < 1e-10
    summary = json.load(open(os.path.join(tmp_path, "summary.json")))
    assert summary["P_print_init"] > 0 and summary["P_cavity_init"] >= 0
    assert abs(summary["J_total_init"] - (summary["J_raw_init"] - 0.9 * summary["P_print_init"]
                                          - 0.9 * summary["P_cavity_init"])) < 1e-12
    assert res.iters_run == 3


@pytest.mark.parametrize("r,tiles,periodic", [(6, (1, 1, 1), True), (6, (1, 1, 1), False), (10, (2, 1, 1), False),
                                              (6, (3, 3, 3), False), (10, (1, 1, 1), True)])
def test_cavity_odd_grids_match_oracle(lib, r, tiles, periodic):
    """Cavity penalty and gradient on (super)cells that are not multiples of
    the 8^3 tile of the fused radius-1 flood fill, periodic or not, on a field
    of exact ties and a continuous one, against the oracle: radius 1 with and
    without the opening (fused kernels) and radius 2 (separable passes)."""
    from maple_b200.core import HomogenizationContext
    from oracle import ihd_oracle as O
    rng = np.random.default_rng(r + sum(tiles))
    fields = np.stack([rng.choice([0.0, 0.3, 0.5, 1.0], size=r ** 3), rng.random(r ** 3)])
    rho = torch.tensor(fields, dtype=torch.float64, device=DEV)
    ctx = HomogenizationContext(r, ncells=2, device=DEV)
    for rad, mcr, iters in ((1, 0, 0), (1, 1, 5), (2, 0, 3)):
        if periodic and tiles == (1, 1, 1) and (2 * rad + 1 > r or 2 * mcr + 1 > r):
            continue
        ctx.set_penalties(0.0, 45.0, 1.0, min_channel_rad=mcr, rad=rad, iters=iters, tiles=tiles, focus_center=True,
                          periodic=periodic)
        out = ctx.penalties(rho, overhang=False, cavity=True)
        P, dP = out["P_cavity"].cpu().numpy(), out["dP_cavity"].cpu().numpy()
        for b in range(2):
            P0, g0 = O.cavity_penalty(fields[b], r, min_channel_rad=mcr, rad=rad, iters=iters, tiles=tiles,
                                      periodic=periodic)
            assert abs(P[b] - P0) <= 1e-13 * max(1.0, abs(P0)), (rad, mcr, b, P[b], P0)
            np.testing.assert_allclose(dP[b], np.asarray(g0).reshape(-1), rtol=0, atol=1e-12)
    ctx.close()
