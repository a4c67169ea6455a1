"""Element tables and RHS assembly with the call surface of the reference's
``maple/core/utils/_utils.py``.

Element matrices come from the library's host code (``maple_element_matrices``),
the RHS assembly runs as a CUDA kernel.  Contexts are cached per
(resolution, device).
"""
from __future__ import annotations

import math
from typing import Dict, Tuple

import torch

from .core import HomogenizationContext, element_matrices

_CTX: Dict[Tuple[int, int, str], HomogenizationContext] = {}


def cached_context(r: int, device, ncells: int = 1) -> HomogenizationContext:
    dev = torch.device(device)
    if dev.type != "cuda":
        raise ValueError(f"maple_b200 runs on CUDA devices only, got {dev}")
    if dev.index is None:
        dev = torch.device("cuda", torch.cuda.current_device())
    key = (int(r), int(ncells), str(dev))
    if key not in _CTX:
        _CTX[key] = HomogenizationContext(int(r), ncells=int(ncells), device=dev)
    return _CTX[key]


def isotropic_elastic_tensor(E, v) -> torch.Tensor:
    """6x6 isotropic stiffness (Voigt), float32 like utils/_utils.py:39-48."""
    lam = v / (1.0 + v) / (1.0 - 2.0 * v) * E
    mu = 1.0 / (2.0 * (1.0 + v)) * E
    C = torch.zeros(6, 6, dtype=torch.float32)
    C[:3, :3] = lam
    for i in range(3):
        C[i, i] = lam + 2 * mu
        C[i + 3, i + 3] = mu
    return C


def _material_from_C(C: torch.Tensor) -> Tuple[float, float]:
    lam, mu = float(C[0, 1]), float(C[3, 3])
    E = mu * (3 * lam + 2 * mu) / (lam + mu)
    nu = lam / (2 * (lam + mu))
    return E, nu


def hexahedron(r: int, C: torch.Tensor):
    """Ke (24,24), Fe (24,6), X0 (24,6) of an isotropic voxel of edge 1/r
    (utils/_utils.py:49-109), in C's dtype and on C's device."""
    E, nu = _material_from_C(C)
    Ke3, Fe3, X03, *_ = element_matrices(r, E, nu, 1.0)
    f = lambda a: torch.tensor(a, dtype=C.dtype, device=C.device)  # noqa: E731
    return f(Ke3), f(Fe3), f(X03)


def hexahedron_scalar(r: int, kappa=1.0):
    """Ke (8,8), Fe (8,3), X0 (8,3) for conduction (utils/_utils.py:116-196)."""
    dev, dtype = torch.device("cpu"), torch.float32
    if isinstance(kappa, torch.Tensor):
        dev, dtype, k = kappa.device, kappa.dtype, float(kappa.item())
    else:
        k = float(kappa)
    *_, Ke1, Fe1, X01 = element_matrices(r, 1.0, 0.3, k)
    f = lambda a: torch.tensor(a, dtype=dtype, device=dev)  # noqa: E731
    return f(Ke1), f(Fe1), f(X01)


def _resolution(n_nodes: int) -> int:
    r = int(round(n_nodes ** (1.0 / 3.0)))
    if r ** 3 != n_nodes:
        raise ValueError(f"n_nodes={n_nodes} is not a cube: a periodic r^3 cell is required")
    return r


def _check_topology(node_index: torch.Tensor, r: int):
    if node_index.dim() != 2 or node_index.shape != (r ** 3, 8):
        raise ValueError(f"Expected node_index shape ({r ** 3},8), got {tuple(node_index.shape)}")


def _rho_vector(rho, n: int, device) -> torch.Tensor:
    return torch.as_tensor(rho).detach().reshape(1, n).to(device=device, dtype=torch.float64).contiguous()


def assemble_F_fast(node_index: torch.Tensor, Fe: torch.Tensor, n_nodes: int, rho) -> torch.Tensor:
    """F = sum_e rho_e Fe0 -> (n_nodes, 3, 6) (utils/_utils.py:480-507), computed
    by the RHS kernel on the structured periodic cell.  The result carries no
    autograd graph: IHD.TO_homo_3d already differentiates through F(rho)."""
    r = _resolution(n_nodes)
    _check_topology(node_index, r)
    if Fe.shape != (24, 6):
        raise ValueError(f"Expected Fe shape (24,6), got {tuple(Fe.shape)}")
    ctx = cached_context(r, node_index.device)
    F = ctx.assemble_rhs("elastic", _rho_vector(rho, n_nodes, ctx.device))  # (1,6,3,N)
    return F[0].permute(2, 1, 0).contiguous().to(Fe.dtype)


def assemble_F_fast_scalar(node_index: torch.Tensor, Fe: torch.Tensor, n_nodes: int, rho) -> torch.Tensor:
    """Scalar RHS (n_nodes, 3) (utils/_utils.py:453-478)."""
    if Fe.dim() != 2 or Fe.shape[0] != 8:
        raise ValueError(f"Expected Fe shape (8,3), got {tuple(Fe.shape)}")
    r = _resolution(n_nodes)
    if node_index.dim() != 2 or node_index.shape[1] != 8:
        raise ValueError(f"Expected node_index shape (E,8), got {tuple(node_index.shape)}")
    _check_topology(node_index, r)
    ctx = cached_context(r, node_index.device)
    F = ctx.assemble_rhs("thermal", _rho_vector(rho, n_nodes, ctx.device))  # (1,3,1,N)
    return F[0, :, 0, :].T.contiguous().to(Fe.dtype)


def cube_root(n: int) -> int:
    r = int(round(math.pow(n, 1.0 / 3.0)))
    return r if r ** 3 == n else -1
