"""Optimizer entry points with the call surface of the reference's
``maple/core/main_IHD_v3.py``: ``setup_seed``, ``build_unitcell_batch``,
``avg_filter3d_x_periodic``, ``oc_update``, ``make_random_x_init``,
``evaluate_J``, ``evaluate_homogenized_terms``, ``RunResult`` and
``optimize_inverse_homogenization``.

The OC loop runs each iteration as one fused device step (SIMP map, both
solves, C^H / kappa^H, objective, analytic sensitivities, box filter and the
60-step OC bisection; ``maple_oc_step``).  Output files keep the reference's
names and columns: ``iter_log.csv``, ``summary.json``, ``rho_final.npy``.
Mesh export (marching cubes to OBJ) is not part of this package.
"""
from __future__ import annotations

import csv
import json
import os
import random
import time
from dataclasses import dataclass
from typing import Dict, Optional, Tuple

import numpy as np
import torch

from .core import box_filter, symmetrize
from .model import IHD
from .objective import (objective_from_spec, objective_requires, objective_weights, shear_objective,
                        stiffness_objective, thermal_objective)
from .utils import cached_context, cube_root

HEX8 = ((0, 0, 0), (1, 0, 0), (1, 1, 0), (0, 1, 0), (0, 0, 1), (1, 0, 1), (1, 1, 1), (0, 1, 1))


def setup_seed(seed: int = 0) -> None:
    """Seeds python, numpy and torch RNGs (main_IHD_v3.py:62-68)."""
    random.seed(seed)
    np.random.seed(seed)
    torch.manual_seed(seed)
    torch.cuda.manual_seed_all(seed)
    torch.backends.cudnn.deterministic = True
    torch.backends.cudnn.benchmark = False


def build_unitcell_batch(device: torch.device, res: int, rho_grid: torch.Tensor) -> Dict[str, torch.Tensor]:
    """Periodic unit-cell batch dict (main_IHD_v3.py:162-215): coord, feature,
    node_index, elem_coords, rho, voxel_batch_id."""
    if tuple(rho_grid.shape) != (res, res, res):
        raise ValueError(f"rho_grid must be {(res, res, res)}, got {tuple(rho_grid.shape)}")
    ar = torch.arange(res, device=device)
    grid = torch.stack(torch.meshgrid(ar, ar, ar, indexing="ij"), dim=-1).reshape(-1, 3).long()
    hex8 = torch.tensor(HEX8, dtype=torch.int64, device=device)
    corners = (grid[:, None, :] + hex8[None]) % res                       # (N,8,3)
    node_index = (corners[..., 0] * res + corners[..., 1]) * res + corners[..., 2]
    rg = rho_grid.to(device)
    feats = rg[corners[..., 0], corners[..., 1], corners[..., 2]].reshape(-1, 8).to(torch.float32)
    b0 = torch.zeros((grid.shape[0], 1), dtype=torch.long, device=device)
    coord = torch.cat([b0, grid], dim=1)
    return {
        "coord": coord,
        "feature": feats.contiguous(),
        "node_index": node_index,
        "elem_coords": coord.clone(),
        "rho": rg.reshape(-1, 1).to(torch.float32),
        "voxel_batch_id": torch.zeros((grid.shape[0],), dtype=torch.long, device=device),
    }


def _canonical_order(elem_coords: torch.Tensor, res: int) -> torch.Tensor:
    xyz = elem_coords[:, 1:4].long() if elem_coords.shape[1] == 4 else elem_coords.long()
    return (xyz[:, 0] * res + xyz[:, 1]) * res + xyz[:, 2]


def avg_filter3d_x_periodic(x_vec: torch.Tensor, elem_coords: torch.Tensor, res: int, k: int = 3) -> torch.Tensor:
    """Periodic k^3 box filter of an (N,1) vector laid out by elem_coords
    (main_IHD_v3.py:342-359), as a CUDA kernel."""
    if int(k) <= 0:
        raise ValueError(f"filter size must be positive, got {k}")
    if int(k) % 2 == 0:
        raise ValueError(f"filter size must be odd, got {k}")
    order = _canonical_order(elem_coords, res).to(x_vec.device)
    vol = torch.empty(res ** 3, dtype=torch.float64, device=x_vec.device)
    vol[order] = x_vec.reshape(-1).to(torch.float64)
    out = box_filter(vol.reshape(1, -1).contiguous(), res, int(k)).reshape(-1)
    return out[order].reshape(-1, 1).to(x_vec.dtype)


def _parse_tiles_xyz(tiles_xyz, tiles: int):
    """(tx, ty, tz) from "tx,ty,tz" / "tx ty tz" or a single count (main_IHD_v3.py:101-115)."""
    if tiles_xyz is None:
        t = max(1, int(tiles))
        return t, t, t
    parts = [p for p in str(tiles_xyz).replace(" ", ",").split(",") if p != ""]
    if len(parts) != 3:
        raise ValueError("--cavity_tiles_xyz must have 3 integers, e.g. 3,3,3")
    return tuple(max(1, int(p)) for p in parts)


def parse_symmetry(symmetry: str):
    """(kind, axes) of a symmetry spec, as main_IHD_v3.py:221-256: "none";
    "mirror" with the x/y/z letters present ("octant", "1/8", "one_eighth" =
    all three); "cubic" for "cubic", "iso", "isotropic"."""
    sym = (symmetry or "none").lower().strip()
    if sym in ("none", ""):
        return "none", []
    if sym in ("octant", "1/8", "one_eighth"):
        sym = "xyz"
    if sym in ("cubic", "iso", "isotropic"):
        return "cubic", [0, 1, 2]
    axes = sorted({i for i, ch in enumerate("xyz") if ch in sym})
    return ("mirror", axes) if axes else ("none", [])


def symmetrize_vec(x_vec: torch.Tensor, elem_coords: torch.Tensor, res: int, kind: str, axes) -> torch.Tensor:
    """Symmetry projection of an (N,1) design laid out by elem_coords
    (main_IHD_v3.py:329-337), as a CUDA kernel."""
    if kind == "none":
        return x_vec.reshape(-1, 1)
    if kind not in ("mirror", "cubic"):
        raise ValueError(f"Unknown symmetry kind: {kind}")
    if kind == "mirror" and not axes:
        return x_vec.reshape(-1, 1)
    order = _canonical_order(elem_coords, res).to(x_vec.device)
    vol = torch.empty(res ** 3, dtype=torch.float64, device=x_vec.device)
    vol[order] = x_vec.reshape(-1).to(torch.float64)
    out = symmetrize(vol.reshape(1, -1).contiguous(), res, kind, axes).reshape(-1)
    return out[order].reshape(-1, 1).to(x_vec.dtype)


@torch.no_grad()
def oc_update(x: torch.Tensor, dJdx: torch.Tensor, volfrac: float, move: float = 0.1,
              xmin: float = 1e-3) -> torch.Tensor:
    """OC step with 60 bisections on lambda in [1e-12, 1e6] (main_IHD_v3.py:362-380),
    as a CUDA kernel; returns the x of the last bisection step."""
    n = x.numel()
    r = cube_root(n)
    if r < 6 or r % 2:
        raise ValueError(f"oc_update runs on periodic r^3 cells with even r >= 6; got {n} entries")
    ctx = cached_context(r, x.device)
    x64 = x.detach().reshape(1, n).to(torch.float64).contiguous()
    d64 = dJdx.detach().reshape(1, n).to(device=x.device, dtype=torch.float64).contiguous()
    vf = torch.full((1,), float(volfrac), dtype=torch.float64, device=x.device)
    xn, _ = ctx.oc_update(x64, d64, vf, move=float(move), xmin=float(xmin))
    return xn.reshape(x.shape).to(x.dtype)


@torch.no_grad()
def make_random_x_init(res: int, volfrac: float, xmin: float, device: torch.device, iters: int = 5) -> torch.Tensor:
    """Uniform random x in [xmin,1] with mean(x)=volfrac (main_IHD_v3.py:383-402)."""
    N = res ** 3
    x = torch.rand((N, 1), device=device, dtype=torch.float32)
    for _ in range(int(iters)):
        x = x - x.mean() + float(volfrac)
        x = torch.clamp(x, xmin, 1.0)
    x = x - x.mean() + float(volfrac)
    return torch.clamp(x, xmin, 1.0)


@torch.no_grad()
def evaluate_J(ihd_module: IHD, batch: Dict[str, torch.Tensor], rho: torch.Tensor, obj: str) -> float:
    """J of a fixed rho (main_IHD_v3.py:406-428)."""
    batch["rho"] = rho
    need_CH, need_kappa = objective_requires(obj)
    kappa = ihd_module.TO_homo_1d(batch, ihd_module.Ke_1d, None, ihd_module.X0_1d, batch_size=1) if need_kappa \
        else None
    CH = ihd_module.TO_homo_3d(batch, ihd_module.Ke_3d, None, ihd_module.X0_3d, batch_size=1) if need_CH else None
    return float(objective_from_spec(obj=obj, CH=CH, kappa=kappa).item())


@torch.no_grad()
def evaluate_homogenized_terms(ihd_module: IHD, batch: Dict[str, torch.Tensor], rho: torch.Tensor, *,
                               terms: Tuple[str, ...] = ("stiffness", "shear", "thermal")) -> Dict[str, float]:
    """Selected homogenized metrics of a fixed rho (main_IHD_v3.py:431-466)."""
    wanted = {str(t).lower() for t in terms}
    batch["rho"] = rho
    out: Dict[str, float] = {}
    if "thermal" in wanted:
        kappa = ihd_module.TO_homo_1d(batch, ihd_module.Ke_1d, None, ihd_module.X0_1d, batch_size=1)
        out["thermal"] = float(thermal_objective(kappa).item())
    if "stiffness" in wanted or "shear" in wanted:
        CH = ihd_module.TO_homo_3d(batch, ihd_module.Ke_3d, None, ihd_module.X0_3d, batch_size=1)
        if "stiffness" in wanted:
            out["stiffness"] = float(stiffness_objective(CH).item())
        if "shear" in wanted:
            out["shear"] = float(shear_objective(CH).item())
    return {k: out[k] for k in ("stiffness", "shear", "thermal") if k in out}


@dataclass
class RunResult:
    J_raw_init: float
    J_raw_final: float
    J_total_init: float
    J_total_final: float
    P_print_init: float
    P_print_final: float
    P_cavity_init: float
    P_cavity_final: float
    iters_run: int
    converged: bool
    rho_final: np.ndarray
    log_csv: Optional[str]
    summary_json: Optional[str]
    meshes_dir: str
    rho_final_npy: str
    final_obj: str


def optimize_inverse_homogenization(ihd_module: IHD, batch: Dict[str, torch.Tensor], *, res: int, objective: str,
                                    init_mode: str, volfrac: float, penal: float, rho_min: float, move: float,
                                    xmin: float, iters: int, seed: int, symmetry: str, lambda_print: float,
                                    overhang_deg: float, lambda_cavity: float, cavity_thresh: float,
                                    cavity_beta: float, min_channel_rad: int, cavity_rad: int,
                                    cavity_seed_faces: str, cavity_iters: int, cavity_tiles: int,
                                    cavity_tiles_xyz: str | None, cavity_focus_center: bool, filter_k: int,
                                    output_dir: str, mesh_every: int, mesh_res: int, mesh_iso: float,
                                    mesh_pad: int, save_iter_log: bool = True, save_summary: bool = True,
                                    save_initial_mesh: bool = True, verbose: bool = True,
                                    x_init: Optional[torch.Tensor] = None, precision: Optional[str] = None,
                                    rtol: Optional[float] = None, stop_rule: str = "reference",
                                    dx_tol: float = 0.01) -> RunResult:
    """OC loop of main_IHD_v3.py:492-891 on the GPU.

    Same arguments and outputs as the reference, including every symmetry
    ("none", mirror axes, "cubic"/"iso") and the overhang / cavity penalties
    (computed on the GPU with the gradients of the reference's autograd).  Extra keywords: ``x_init`` (an (N,1) design to
    start from, bypassing ``init_mode``), ``precision``/``rtol`` (default: the
    IHD module's), ``stop_rule`` "reference" (stall test of
    main_IHD_v3.py:611-618, 711-714) or "dx" (stop when max|dx| < dx_tol).
    """
    sym_kind, sym_axes = parse_symmetry(symmetry)
    device = ihd_module.device
    setup_seed(seed)
    os.makedirs(output_dir, exist_ok=True)
    meshes_dir = os.path.join(output_dir, "meshes")
    os.makedirs(meshes_dir, exist_ok=True)
    log_csv = os.path.join(output_dir, "iter_log.csv") if save_iter_log else None
    summary_json = os.path.join(output_dir, "summary.json") if save_summary else None
    final_rho_npy = os.path.join(output_dir, "rho_final.npy")
    final_obj = os.path.join(meshes_dir, "final.obj")
    precision = precision or ihd_module.precision
    rtol = float(rtol if rtol is not None else ihd_module.rtol)

    if x_init is not None:
        x = x_init.detach().reshape(-1, 1).to(device=device, dtype=torch.float64)
    elif init_mode == "noise":
        x = make_random_x_init(res=res, volfrac=volfrac, xmin=xmin, device=device, iters=5).double()
    else:
        rho0 = batch["rho"].double().reshape(-1, 1).clamp(rho_min, 1.0)
        x = ((rho0 - rho_min) / (1.0 - rho_min)).clamp(0.0, 1.0).pow(1.0 / penal).clamp(xmin, 1.0)
        if volfrac <= 0:
            volfrac = float(x.mean().item())
    x = x.clamp(xmin, 1.0).reshape(1, -1).contiguous()
    if sym_kind != "none":
        x = symmetrize(x, res, sym_kind, sym_axes).clamp(xmin, 1.0).contiguous()

    def simp(xv):
        return (rho_min + (1.0 - rho_min) * (xv.clamp(xmin, 1.0) ** penal)).reshape(-1, 1).clamp(rho_min, 1.0)

    hc = ihd_module.homog_ctx
    use_print, use_cavity = float(lambda_print) > 0.0, float(lambda_cavity) > 0.0
    if use_print or use_cavity:
        hc.set_penalties(float(lambda_print), float(overhang_deg), float(lambda_cavity), void_thresh=float(cavity_thresh),
                         beta=float(cavity_beta), min_channel_rad=int(min_channel_rad), rad=int(cavity_rad),
                         iters=int(cavity_iters or 0), tiles=_parse_tiles_xyz(cavity_tiles_xyz, cavity_tiles),
                         focus_center=bool(cavity_focus_center), seed_faces=str(cavity_seed_faces), periodic=True)

    def penalties(rho_col):
        if not (use_print or use_cavity):
            return 0.0, 0.0
        o = hc.penalties(rho_col.reshape(1, -1).contiguous(), overhang=use_print, cavity=use_cavity, grad=False)
        return (float(o["P_print"][0]) if use_print else 0.0, float(o["P_cavity"][0]) if use_cavity else 0.0)

    J_raw_init = evaluate_J(ihd_module, batch, simp(x), obj=objective)
    P_print_init, P_cavity_init = penalties(simp(x))
    J_total_init = float(J_raw_init) - float(lambda_print) * P_print_init - float(lambda_cavity) * P_cavity_init
    if save_iter_log and log_csv is not None:
        with open(log_csv, "w", newline="") as f:
            csv.writer(f).writerow(["iter", "J_total", "J_raw", "P_print", "P_cavity", "mean_x", "mean_rho", "dx_max",
                                    "dx_mean", "time_sec"])

    hc.set_symmetry(sym_kind, sym_axes)
    w = torch.tensor([objective_weights(objective)], dtype=torch.float64, device=device)
    vf = torch.tensor([float(volfrac)], dtype=torch.float64, device=device)
    t0 = time.time()
    J_prev: Optional[float] = None
    stall, converged, it_run = 0, False, 0
    tol_x, tol_J, patience, min_iters = 1e-3, 1e-4, 10, 10
    for it in range(iters):
        it_run = it + 1
        out = hc.oc_step(x, w, vf, penal=penal, rho_min=rho_min, move=move, xmin=xmin,
                         filter_k=int(filter_k) if filter_k and int(filter_k) > 1 else 0, precision=precision,
                         rtol=rtol, maxit=ihd_module.maxit, warm=ihd_module.warm_start)
        J_val = float(out["J"].item())
        J_raw_val = float(out["J_raw"].item())
        P_print_val, P_cavity_val = float(out["P_print"].item()), float(out["P_cavity"].item())
        dx_max, dx_mean = (float(v) for v in out["stats"][0].tolist())
        x_mean = float(x.clamp(xmin, 1.0).mean().item())
        rho_mean = float(simp(x).mean().item())
        dJ_rel = float("inf") if J_prev is None else abs(J_val - J_prev) / max(abs(J_prev), 1e-12)
        if stop_rule == "reference":
            stall = stall + 1 if (it >= min_iters and dx_max < tol_x and dJ_rel < tol_J) else 0
        x = out["x_next"].clamp(xmin, 1.0).contiguous()
        J_prev = J_val
        t_now = time.time() - t0
        if save_iter_log and log_csv is not None:
            with open(log_csv, "a", newline="") as f:
                csv.writer(f).writerow([it_run, J_val, J_raw_val, P_print_val, P_cavity_val, x_mean, rho_mean, dx_max,
                                        dx_mean, t_now])
        if verbose:
            print(f"it={it_run:04d}  J_total={J_val:.6e}  J_raw={J_raw_val:.6e}  P_print={P_print_val:.6e}  "
                  f"P_cavity={P_cavity_val:.6e}  mean_x={x_mean:.4f}  mean_rho={rho_mean:.4f}  "
                  f"dx_max={dx_max:.3e}  dx_mean={dx_mean:.3e}  stall={stall}/{patience}")
        if stop_rule == "reference" and stall >= patience:
            converged = True
            break
        if stop_rule == "dx" and dx_max < dx_tol:
            converged = True
            break

    hc.set_symmetry("none")
    rho_final = simp(x)
    J_raw_final = evaluate_J(ihd_module, batch, rho_final, obj=objective)
    P_print_final, P_cavity_final = penalties(rho_final)
    J_total_final = float(J_raw_final) - float(lambda_print) * P_print_final - float(lambda_cavity) * P_cavity_final
    if use_print or use_cavity:
        hc.set_penalties(0.0, float(overhang_deg), 0.0)
    rho_final_grid = rho_final.reshape(res, res, res).detach().cpu().numpy().astype(np.float32)
    np.save(final_rho_npy, rho_final_grid)
    summary = {
        "objective": objective, "init_mode": init_mode, "symmetry": str(symmetry),
        "lambda_print": float(lambda_print), "overhang_deg": float(overhang_deg),
        "lambda_cavity": float(lambda_cavity), "cavity_thresh": float(cavity_thresh),
        "cavity_beta": float(cavity_beta), "min_channel_rad": int(min_channel_rad), "cavity_rad": int(cavity_rad),
        "cavity_seed_faces": str(cavity_seed_faces), "cavity_iters": int(cavity_iters),
        "cavity_tiles": int(cavity_tiles),
        "cavity_tiles_xyz": (None if cavity_tiles_xyz is None else str(cavity_tiles_xyz)),
        "cavity_focus_center": bool(cavity_focus_center), "resolution": res, "iters_requested": iters,
        "iters_run": int(it_run), "converged": bool(converged), "seed": int(seed),
        "volfrac_target": float(volfrac), "penal": float(penal), "rho_min": float(rho_min), "move": float(move),
        "xmin": float(xmin), "mesh_every": int(mesh_every), "mesh_res": int(mesh_res), "mesh_iso": float(mesh_iso),
        "mesh_pad": int(mesh_pad), "J_raw_init": float(J_raw_init), "J_raw_final": float(J_raw_final),
        "J_total_init": float(J_total_init), "J_total_final": float(J_total_final),
        "P_print_init": float(P_print_init), "P_print_final": float(P_print_final),
        "P_cavity_init": float(P_cavity_init), "P_cavity_final": float(P_cavity_final),
        "log_csv": (None if log_csv is None else os.path.abspath(log_csv)),
        "rho_final_npy": os.path.abspath(final_rho_npy), "meshes_dir": os.path.abspath(meshes_dir),
        "time_sec": float(time.time() - t0),
    }
    if save_summary and summary_json is not None:
        with open(summary_json, "w", encoding="utf-8") as f:
            json.dump(summary, f, ensure_ascii=False, indent=2)
    return RunResult(J_raw_init=float(J_raw_init), J_raw_final=float(J_raw_final), J_total_init=float(J_total_init),
                     J_total_final=float(J_total_final), P_print_init=float(P_print_init),
                     P_print_final=float(P_print_final), P_cavity_init=float(P_cavity_init),
                     P_cavity_final=float(P_cavity_final), iters_run=int(it_run), converged=bool(converged), rho_final=rho_final_grid,
                     log_csv=log_csv, summary_json=summary_json, meshes_dir=meshes_dir,
                     rho_final_npy=final_rho_npy, final_obj=final_obj)
