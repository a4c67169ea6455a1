"""Manufacturability penalties with the reference's call surface
(maple.core.utils.printability): differentiable w.r.t. the density grid, as
torch.autograd Functions whose forward pass runs the library's CUDA kernels
and computes the gradient at the same time.

The gradients follow the tie rules of the autograd the reference uses (a
max-pool window passes its gradient to its first maximum in scan order,
torch.minimum splits it in half between equal arguments, relu passes nothing
at 0), so they agree with the reference's to rounding.
"""
from __future__ import annotations

from typing import Optional, Tuple

import torch

from .utils import cached_context


def _as_cells(rho_grid: torch.Tensor) -> Tuple[torch.Tensor, int]:
    if rho_grid.ndim != 3 or rho_grid.shape[0] != rho_grid.shape[1] or rho_grid.shape[0] != rho_grid.shape[2]:
        raise ValueError(f"rho_grid must be cubic (r,r,r), got {tuple(rho_grid.shape)}")
    if not rho_grid.is_cuda:
        raise ValueError("rho_grid must be a CUDA tensor (there is no CPU path)")
    r = int(rho_grid.shape[0])
    return rho_grid.detach().reshape(1, -1).to(torch.float64).contiguous(), r


class _Penalty(torch.autograd.Function):
    @staticmethod
    def forward(ctx, rho_grid, kind, settings):
        rho, r = _as_cells(rho_grid)
        hc = cached_context(r, rho_grid.device)
        overhang = kind == "overhang"
        hc.set_penalties(lambda_print=1.0 if overhang else 0.0, lambda_cavity=0.0 if overhang else 1.0, **settings)
        out = hc.penalties(rho, overhang=overhang, cavity=not overhang, grad=True)
        P, dP = (out["P_print"], out["dP_print"]) if overhang else (out["P_cavity"], out["dP_cavity"])
        ctx.save_for_backward(dP.reshape(rho_grid.shape).to(rho_grid.dtype))
        return P.reshape(()).to(rho_grid.dtype)

    @staticmethod
    def backward(ctx, g):
        (dP,) = ctx.saved_tensors
        return g * dP, None, None


def printability_penalty_overhang(rho_grid: torch.Tensor, *, overhang_deg: float = 45.0,
                                  periodic_xy: bool = True) -> torch.Tensor:
    """Overhang penalty (utils/printability.py:91-134): build direction +z;
    layer z is supported by layer z-1 within the lateral radius of the
    overhang angle; the mean unsupported density per layer, averaged."""
    return _Penalty.apply(rho_grid, "overhang", dict(overhang_deg=float(overhang_deg),
                                                     overhang_periodic=bool(periodic_xy)))


def cavity_penalty_closed_void(rho_grid: torch.Tensor, *, void_thresh: float = 0.5, beta: float = 20.0,
                               min_channel_rad: int = 0, rad: int = 1, iters: int = 0, periodic_xyz: bool = True,
                               seed_faces: str = "all") -> torch.Tensor:
    """Trapped-void penalty of one cell (utils/printability.py:139-220)."""
    return _Penalty.apply(rho_grid, "cavity", dict(void_thresh=float(void_thresh), beta=float(beta),
                                                   min_channel_rad=int(min_channel_rad), rad=int(rad),
                                                   iters=int(iters or 0), tiles=(1, 1, 1),
                                                   seed_faces=str(seed_faces), periodic=bool(periodic_xyz)))


def cavity_penalty_periodic_array(rho_grid: torch.Tensor, *, tiles: int = 3,
                                  tiles_xyz: Optional[Tuple[int, int, int]] = None, focus_center: bool = True,
                                  void_thresh: float = 0.5, beta: float = 20.0, min_channel_rad: int = 0,
                                  rad: int = 1, iters: int = 0, seed_faces: str = "all") -> torch.Tensor:
    """Trapped-void penalty of a finite periodic array of the cell
    (utils/printability.py:226-323)."""
    t = (int(tiles),) * 3 if tiles_xyz is None else tuple(int(v) for v in tiles_xyz)
    t = tuple(max(1, v) for v in t)
    return _Penalty.apply(rho_grid, "cavity", dict(void_thresh=float(void_thresh), beta=float(beta),
                                                   min_channel_rad=int(min_channel_rad), rad=int(rad),
                                                   iters=int(iters or 0), tiles=t, focus_center=bool(focus_center),
                                                   seed_faces=str(seed_faces), periodic=False))
