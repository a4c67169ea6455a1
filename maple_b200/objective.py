"""Scalar objectives from C^H / kappa^H and the weighted-spec parser.

Same call surface and semantics as the reference's
``maple/core/utils/objective.py`` (xing-yuu/MAPLE): a 6x6 / 3x3 host-side
computation on whatever device the tensors live on, differentiable with
torch autograd so that ``IHD.TO_homo_3d/1d`` gradients flow through it.
"""
from __future__ import annotations

import re
from typing import Dict, Mapping, Optional, Tuple

import torch


def _compliance(CH: torch.Tensor) -> torch.Tensor:
    C = 0.5 * (CH + CH.T)
    return torch.linalg.inv(C + 1e-9 * torch.eye(6, device=C.device, dtype=C.dtype))


def stiffness_objective(CH: torch.Tensor) -> torch.Tensor:
    """mean(Ex, Ey, Ez) with E_i = 1 / S_ii, S = inv(sym(C) + 1e-9 I)
    (utils/objective.py:11-19)."""
    S = _compliance(CH)
    return (1.0 / S[0, 0] + 1.0 / S[1, 1] + 1.0 / S[2, 2]) / 3.0


def shear_objective(CH: torch.Tensor) -> torch.Tensor:
    """mean(Gyz, Gxz, Gxy) with G = 1 / S_shear (utils/objective.py:22-30)."""
    S = _compliance(CH)
    return (1.0 / S[3, 3] + 1.0 / S[4, 4] + 1.0 / S[5, 5]) / 3.0


def thermal_objective(kappa: torch.Tensor) -> torch.Tensor:
    """trace(kappa) (utils/objective.py:33-41)."""
    if kappa.dim() < 2 or kappa.shape[-1] != kappa.shape[-2]:
        raise ValueError(f"kappa must be square, got {tuple(kappa.shape)}")
    return torch.diagonal(kappa, dim1=-2, dim2=-1).sum()


_ALIASES: Dict[str, str] = {
    "stiff": "stiffness", "stiffness": "stiffness", "e": "stiffness", "young": "stiffness", "youngs": "stiffness",
    "shear": "shear", "g": "shear",
    "thermal": "thermal", "kappa": "thermal", "conductivity": "thermal", "heat": "thermal",
}
_CANONICAL = ("stiffness", "shear", "thermal")


def _canonical(name: str) -> str:
    n = _ALIASES.get(str(name).strip().lower(), str(name).strip().lower())
    if n not in _CANONICAL:
        raise ValueError(f"Unknown objective term: {name!r}. Supported: {list(_CANONICAL)}")
    return n


def _number(s: str) -> bool:
    try:
        float(s)
        return True
    except ValueError:
        return False


def parse_objective_spec(spec: str) -> Dict[str, float]:
    """Spec string -> {term: weight}.  Accepts "stiffness", "stiffness,thermal",
    "stiffness:0.4,thermal:0.6", "0.4*stiffness+0.6*thermal",
    "shear=0.3+thermal=0.7"; None or "" mean {"shear": 1}
    (utils/objective.py:93-157)."""
    if spec is None or not str(spec).strip():
        return {"shear": 1.0}
    s = str(spec).strip()
    try:
        return {_canonical(s): 1.0}
    except ValueError:
        pass
    parts = [p for p in re.split(r"[,+]", s.replace(" ", "")) if p]
    if not parts:
        raise ValueError(f"Invalid objective spec: {spec!r}")
    out: Dict[str, float] = {}
    for part in parts:
        if ":" in part or "=" in part:
            name, w = re.split(r"[:=]", part, maxsplit=1)
            weight = float(w)
        elif "*" in part:
            a, b = part.split("*", 1)
            if _number(a) and not _number(b):
                weight, name = float(a), b
            elif _number(b) and not _number(a):
                weight, name = float(b), a
            else:
                raise ValueError(f"Invalid term {part!r} in objective spec {spec!r}. "
                                 f"Expected something like '0.4*stiffness' or 'stiffness:0.4'.")
        else:
            name, weight = part, 1.0
        term = _canonical(name)
        out[term] = out.get(term, 0.0) + float(weight)
    if not out:
        raise ValueError(f"Invalid objective spec: {spec!r}")
    return out


def objective_requires(obj_spec: str) -> Tuple[bool, bool]:
    """(need_CH, need_kappa) (utils/objective.py:160-165)."""
    terms = parse_objective_spec(obj_spec)
    return any(k in ("stiffness", "shear") for k in terms), "thermal" in terms


def objective_weights(obj_spec: str) -> Tuple[float, float, float]:
    """(w_stiffness, w_shear, w_thermal) of a spec, the per-cell weight row
    consumed by the fused OC kernels."""
    t = parse_objective_spec(obj_spec)
    return (t.get("stiffness", 0.0), t.get("shear", 0.0), t.get("thermal", 0.0))


def objective_from_tensor(T: torch.Tensor, obj: str) -> torch.Tensor:
    o = _canonical(obj)
    if o == "stiffness":
        return stiffness_objective(T)
    if o == "shear":
        return shear_objective(T)
    return thermal_objective(T)


def objective_from_spec(*, obj: str, CH: Optional[torch.Tensor] = None, kappa: Optional[torch.Tensor] = None,
                        normalize_by: Optional[Mapping[str, float]] = None, return_parts: bool = False):
    """Weighted multi-objective J (utils/objective.py:180-251)."""
    terms = parse_objective_spec(obj)
    raw_parts: Dict[str, torch.Tensor] = {}
    used_parts: Dict[str, torch.Tensor] = {}
    J = None
    for term, w in terms.items():
        if term in ("stiffness", "shear"):
            if CH is None:
                raise ValueError(f"Objective '{obj}' requires CH (mechanical), but CH=None")
            raw = stiffness_objective(CH) if term == "stiffness" else shear_objective(CH)
        else:
            if kappa is None:
                raise ValueError(f"Objective '{obj}' requires kappa (thermal), but kappa=None")
            raw = thermal_objective(kappa)
        raw_parts[term] = raw
        used = raw
        if normalize_by is not None and term in normalize_by:
            used = raw / max(abs(float(normalize_by[term])), 1e-12)
        used_parts[term] = used
        J = float(w) * used if J is None else J + float(w) * used
    if J is None:
        raise ValueError(f"Empty objective spec: {obj!r}")
    return (J, raw_parts, used_parts) if return_parts else J


objective_from_CH = objective_from_tensor
