"""``GMGSolver`` / ``GMGSolverScalar``: drop-ins for the reference's element-by-
element multigrid solvers (``maple/core/utils/EBE_GMG.py:466-984`` and
``EBE_GMG_scalar.py:343-832``).

``solve(fine_ke, global_f, node_coords_L0, fine_elem_coords,
fine_topo_indices, ...)`` keeps its signature and returns ``(u, r)``.  The
operator must be the periodic structured cell the reference builds with
``build_unitcell_batch`` and ``Ke_e = rho_e * Ke0`` (utils/model.py:108); the
densities are recovered from ``fine_ke`` and checked.  The solve runs MG-PCG
on the GPU to ``rtol`` (keyword, default 1e-10) instead of a fixed number of
V-cycles; ``max_iter`` is honoured as a lower bound of the PCG iteration cap.
The converged u may differ from the reference's by a rigid translation (the
periodic operator's null space), which leaves C^H unchanged.
``init_list`` is the reference's hook for network-predicted fields
(EBE_GMG.py:648-757, 851-858, 943-952): a dense tensor shaped like
``global_f``, or a list of per-level fields ordered coarse to fine as the
reference's (its last entry is the fine level), each None, a dense
(n_l^3, D) tensor or a sparse tensor with ``.indices`` ([b,]x,y,z) and
``.features`` (``init_feat_slice`` selects the D components, ``init_batch``
the batch entry), aligned to the level's nodes by coordinates as
``_spconv_to_dense_u`` does.  The reference starts level 0 from its field and
injects the coarse ones as the starting corrections of every V-cycle
(``init_is_solution``: minus the restricted iterate).  A preconditioner for
CG must be linear, so here the finest given field is the initial iterate
(prolonged trilinearly to the fine grid when it is a coarse level's), with or
without ``init_is_solution``; the converged answer is the same.

The context solves all load cases of a physics at once (6 elastic, 3
thermal).  The reference's homogenization calls ``solve`` once per load case
with the right-hand sides of ``assemble_F_fast`` (utils/model.py:111-124,
140-152).  When ``global_f`` is one of those load cases of the same density,
the first call solves all of them together and the following calls return
the stored columns, so the R calls cost one R-column solve.  Any other
right-hand side is solved on its own (as one column of an R-column solve).
"""
from __future__ import annotations

import torch
import torch.nn as nn

from .core import element_matrices
from .utils import cached_context, cube_root


class GMGSolver(nn.Module):
    D, R, PHYSICS = 3, 6, "elastic"

    def _reference_ke(self, r):
        Ke3, _, _, Ke1, _, _ = element_matrices(r)
        return Ke3 if self.D == 3 else Ke1

    def solve(self, fine_ke, global_f, node_coords_L0, fine_elem_coords, fine_topo_indices, max_iter: int = 50,
              smooth_iter=1, init_list=None, init_batch=None, init_feat_slice=slice(0, 3),
              init_is_solution: bool = False, max_levels: int = 5, fixed_mask=None, dtype=torch.float, *,
              rtol: float = 1e-10, precision: str = "fp64"):
        if fixed_mask is not None:
            raise NotImplementedError("fixed_mask: periodic unit cells have no Dirichlet DOFs")
        D = self.D
        f = global_f.reshape(-1, D)
        n = f.shape[0]
        r = cube_root(n)
        if r < 0:
            raise ValueError(f"{n} nodes do not form a periodic r^3 cell")
        k = 8 * D
        if fine_ke.shape != (n, k, k):
            raise ValueError(f"fine_ke must be ({n},{k},{k}), got {tuple(fine_ke.shape)}")
        dev = fine_ke.device
        Kref = torch.tensor(self._reference_ke(r), dtype=torch.float64, device=dev)
        ke64 = fine_ke.detach().to(torch.float64)
        rho = (ke64 * Kref).sum(dim=(1, 2)) / (Kref * Kref).sum()
        err = (ke64 - rho[:, None, None] * Kref).abs().max()
        tol = 1e-5 * ke64.abs().max() if fine_ke.dtype == torch.float32 else 1e-10 * ke64.abs().max()
        if float(err) > float(tol):
            raise ValueError("fine_ke is not rho_e * Ke0 of this resolution: only SIMP-scaled copies of the "
                             "voxel element matrix are supported")
        ctx = cached_context(r, dev)
        rho1 = rho.reshape(1, n).contiguous()
        fd = f.to(device=ctx.device, dtype=torch.float64)
        u_init = None
        if init_list is not None:
            u_init = self._initial_iterate(init_list, r, init_batch, init_feat_slice, ctx.device)
        col = None
        if init_list is None:
            col = self._load_case_column(ctx, rho1, fd, precision, rtol, fine_ke.dtype)
        if col is not None:
            u, res = self._cache["u"], self._cache["r"]
            out_u = u[0, col].T.contiguous().to(device=dev, dtype=dtype)
            out_r = res[0, col].T.contiguous().to(device=dev, dtype=dtype)
        else:
            ctx.set_density(self.PHYSICS, rho1, precision)
            F = torch.zeros((1, self.R, D, n), dtype=torch.float64, device=ctx.device)
            F[0, 0] = fd.T
            x0 = None
            if u_init is not None:
                x0 = torch.zeros_like(F)
                x0[0, 0] = u_init.T
            u, res, _ = ctx.solve_rhs(self.PHYSICS, F, x0, precision=precision, rtol=rtol,
                                      maxit=max(int(max_iter), 500))
            out_u = u[0, 0].T.contiguous().to(device=dev, dtype=dtype)
            out_r = res[0, 0].T.contiguous().to(device=dev, dtype=dtype)
        if D == 1:
            return out_u.reshape(n, 1), out_r.reshape(n, 1)
        return out_u, out_r


    def _level_field(self, item, nl, batch, feat_slice, device):
        """One level's field as a dense (nl^3, D) FP64 tensor, or None."""
        D, N = self.D, nl ** 3
        if item is None:
            return None
        if isinstance(item, torch.Tensor):
            if item.numel() != N * D:
                raise ValueError(f"init_list field of {item.numel()} values does not fit {N} nodes x {D}")
            return item.reshape(N, D).to(device=device, dtype=torch.float64)
        idx, feat = getattr(item, "indices", None), getattr(item, "features", None)
        if idx is None or feat is None:
            raise TypeError("init_list entries must be tensors or carry .indices and .features")
        idx = idx.to(device=device, dtype=torch.long)
        vals = feat.to(device=device, dtype=torch.float64)[:, feat_slice]
        if vals.shape[1] < D:
            raise ValueError(f"init_list features hold {vals.shape[1]} components, {D} needed")
        vals = vals[:, :D]
        if idx.shape[1] == 4:
            if batch is not None:
                keep = idx[:, 0] == int(batch)
                idx, vals = idx[keep], vals[keep]
            idx = idx[:, 1:]
        idx = idx % nl
        lin = (idx[:, 0] * nl + idx[:, 1]) * nl + idx[:, 2]
        out = torch.zeros((N, D), dtype=torch.float64, device=device)
        out.index_add_(0, lin, vals)
        return out

    def _initial_iterate(self, init_list, r, batch, feat_slice, device):
        """The fine-level initial iterate (n, D) from the reference's
        ``init_list``: the finest given level, prolonged to the fine grid."""
        from .core import transfer
        D, n = self.D, r ** 3
        if isinstance(init_list, torch.Tensor):
            if init_list.numel() != n * D:
                raise ValueError("a dense init_list must have the shape of global_f")
            return init_list.reshape(n, D).to(device=device, dtype=torch.float64)
        if not isinstance(init_list, (list, tuple)):
            raise TypeError("init_list must be a tensor or a list of per-level fields (coarse to fine)")
        for level, item in enumerate(reversed(init_list)):  # level 0 = the fine grid
            if item is None:
                continue
            if r % (1 << level):
                raise ValueError(f"level {level} does not exist for a {r}^3 cell")
            nl = r >> level
            u = self._level_field(item, nl, batch, feat_slice, device)
            for _ in range(level):  # trilinear prolongation, one level at a time
                f3 = torch.zeros((1, 3, nl ** 3), dtype=torch.float64, device=device)
                f3[0, :D] = u.T
                u = transfer("prolong_add", f3.contiguous())[0, :D].T.contiguous()
                nl *= 2
            return u
        return None

    def _load_case_column(self, ctx, rho1, fd, precision, rtol, in_dtype):
        """Index of the load case of ``assemble_F_fast`` that ``fd`` (n, D) is,
        for this density, with every load case solved (once per density,
        precision and tolerance); None when ``fd`` is not one of them."""
        F_all = ctx.assemble_rhs(self.PHYSICS, rho1)  # (1, R, D, n)
        ft = fd.T
        scale = float(ft.abs().max())
        tol = (1e-5 if in_dtype == torch.float32 else 1e-10) * max(scale, 1e-300)
        col = None
        for i in range(self.R):
            if float((F_all[0, i] - ft).abs().max()) <= tol:
                col = i
                break
        if col is None:
            return None
        key = (precision, float(rtol))
        c = getattr(self, "_cache", None)
        if c is None or c["key"] != key or c["rho"].shape != rho1.shape or not torch.equal(c["rho"], rho1):
            ctx.set_density(self.PHYSICS, rho1, precision)
            u, res, _ = ctx.solve_rhs(self.PHYSICS, F_all, None, precision=precision, rtol=rtol, maxit=500)
            self._cache = dict(key=key, rho=rho1.clone(), u=u, r=res)
        return col


class GMGSolverScalar(GMGSolver):
    D, R, PHYSICS = 1, 3, "thermal"
