"""``IHD``: drop-in for the reference's homogenization module
(``maple/core/utils/model.py``).

``TO_homo_3d`` / ``TO_homo_1d`` keep their signatures and return C^H (6x6) /
kappa^H (3x3), differentiable w.r.t. ``batch["rho"]``.  The forward runs the
MG-PCG solve of all load cases at once plus the FP64 energy sums on the GPU;
the backward is the analytic adjoint dC_ij/drho_e = (X0-u_e)_i^T Ke0
(X0-u_e)_j, which is what autograd through a converged solve computes
(main_IHD_v3.py:688).  It accounts for the rho-dependence of both K and F, so
the F argument contributes no separate gradient.
"""
from __future__ import annotations

import torch
import torch.nn as nn

from .core import HomogenizationContext, energy_contract
from .gmg import GMGSolver, GMGSolverScalar
from .utils import hexahedron, hexahedron_scalar, isotropic_elastic_tensor

_R = {"elastic": 6, "thermal": 3}


class _Homogenize(torch.autograd.Function):
    @staticmethod
    def forward(ctx, rho, module, physics):
        hc = module.homog_ctx
        r64 = rho.detach().reshape(1, -1).to(device=hc.device, dtype=torch.float64).contiguous()
        hc.set_density(physics, r64, module.precision)
        info = hc.solve(physics, module.precision, rtol=module.rtol, maxit=module.maxit, warm=module.warm_start)
        module.last_solve_info[physics] = info
        need = rho.requires_grad
        out = hc.homogenize(physics, want_energy=need)
        H, E = out if need else (out, None)
        ctx.meta = (rho.shape, rho.dtype, rho.device, physics)
        if need:
            ctx.save_for_backward(E)
        return H[0].clone()

    @staticmethod
    def backward(ctx, gH):
        shape, dtype, device, physics = ctx.meta
        (E,) = ctx.saved_tensors
        R = _R[physics]
        g = gH.detach().to(device=E.device, dtype=torch.float64).reshape(1, R, R).contiguous()
        d = energy_contract(E, g)
        return d.reshape(shape).to(device=device, dtype=dtype), None, None


class IHD(nn.Module):
    """Inverse-homogenization module (utils/model.py:12-159).

    ``cfg.resolution`` sets r; ``cfg.GMG.smooth_iter`` / ``cfg.GMG.max_cycle``
    are accepted for compatibility.  Unlike the reference's fixed number of
    V-cycles, every solve here runs MG-PCG to ``rtol`` (default 1e-10), so the
    result is the converged homogenized tensor the reference approaches.
    Extra keywords: ``precision`` ("fp64" or "mixed"), ``rtol``, ``maxit``,
    ``levels`` (0 = automatic), ``warm_start`` (start each solve from the
    previous solution of the same physics).
    """

    def __init__(self, cfg, device, *, precision: str = "fp64", rtol: float = 1e-10, maxit: int = 500,
                 levels: int = 0, warm_start: bool = True):
        super().__init__()
        self.cfg = cfg
        self.r = self.resolution = int(cfg.resolution)
        device = torch.device(device)
        if device.type == "cuda" and device.index is None:
            device = torch.device("cuda", torch.cuda.current_device())
        self.device = device
        self.C = isotropic_elastic_tensor(1.0, 0.3).to(device)
        self.Ke_3d, self.Fe_3d, self.X0_3d = hexahedron(self.r, self.C.double())
        self.Ke_1d, self.Fe_1d, self.X0_1d = hexahedron_scalar(
            self.r, kappa=torch.as_tensor(1.0, device=device, dtype=torch.float64))
        self.gmg_solver_3d = GMGSolver()
        self.gmg_solver_1d = GMGSolverScalar()
        self.precision, self.rtol, self.maxit, self.warm_start = precision, float(rtol), int(maxit), bool(warm_start)
        self.homog_ctx = HomogenizationContext(self.r, ncells=1, levels=levels, device=device)
        self.last_solve_info = {}

    def _check(self, batch, batch_size):
        if int(batch_size) != 1:
            raise ValueError("IHD.TO_homo_* handles one cell per call (batch_size=1); use "
                             "maple_b200.batch for many cells")
        rho = batch["rho"]
        if rho.numel() != self.r ** 3:
            raise ValueError(f"batch['rho'] must hold {self.r ** 3} densities, got {rho.numel()}")
        return rho

    def TO_homo_3d(self, batch, Ke, F, X0, batch_size):
        """C^H (6,6) float64 of batch["rho"] (utils/model.py:98-130)."""
        return _Homogenize.apply(self._check(batch, batch_size), self, "elastic")

    def TO_homo_1d(self, batch, Ke, F, X0, batch_size):
        """kappa^H (3,3) float64 of batch["rho"] (utils/model.py:131-159)."""
        return _Homogenize.apply(self._check(batch, batch_size), self, "thermal")
