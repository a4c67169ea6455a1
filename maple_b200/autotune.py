"""Autotuner for the solver's launch shapes and smoother settings.

The fastest setting of a multigrid-preconditioned solve depends on the cell
size, the batch size and the precision: which coarse-level kernel (the tile
shape a level is swept with) is fastest changes with the level's size and the
number of cells, and so do the Chebyshev degrees that balance PCG iterations
against the cost of a sweep.  ``autotune`` measures them on the caller's own
workload and applies the fastest to the context.

Knobs (runtime settings of a ``HomogenizationContext``):

* ``fine_degree``: Chebyshev degree on the fine level and level 1;
* ``coarse_degree``: degree on levels 2 and deeper (0: the library's rule);
* ``nine_max_n``: coarse levels with at most this many nodes per axis use the
  nine-thread kernel (one thread per node and (x, y) offset pair, 32 nodes
  per CTA); ``split_min_n``: larger levels from this size use the split
  kernel (8x4x4-node tiles, three threads per node); the others the 4^3-node
  tile kernel;
* ``tail_fused``: the 8^3 level and the coarsest solve as one cluster launch;
* ``pdl``: programmatic dependent launch of the small coarse-level launches;
* ``device_loop``: the PCG iterations looped on the device (one host wait
  per solve) or one graph replay per iteration;
* ``check_every``: PCG iterations between host convergence checks (without
  the device loop);
* ``mixed_mode`` (mixed precision only): FP32 PCG with FP64 residual
  replacement (reliable updates), flexible FP64 PCG, or FP32 PCG in FP64
  refinement.

Search: coordinate descent from the library defaults, two passes over the
knobs.  Every candidate runs the same short OC trajectory from the caller's
designs: one step from zero initial iterates, then ``steps`` warm-started
steps timed with CUDA events (their sum is the score).  Every candidate
solves to the same tolerance, so the setting changes the time and not the
answer beyond that tolerance.  Results are cached per (GPU, resolution,
cells, precision, tolerance) in a JSON file.

The reference has no counterpart: its solver settings are fixed
(utils/EBE_GMG.py:758-774 defaults, smooth_iter from the CLI).
"""
from __future__ import annotations

import json
import os
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import torch

from .core import HomogenizationContext

DEFAULTS = dict(fine_degree=1, coarse_degree=0, nine_max_n=64, split_min_n=32, tail_fused=True, pdl=True,
                device_loop=True, check_every=1, mixed_mode="flexible")

SPACE = dict(fine_degree=[1, 2], coarse_degree=[0, 2, 3, 4], nine_max_n=[0, 16, 32, 64], split_min_n=[0, 16, 32],
             tail_fused=[True, False], pdl=[True, False], device_loop=[True, False], check_every=[1, 2],
             mixed_mode=["flexible", "reliable", "refine"])

CACHE = os.path.join(os.path.expanduser("~"), ".cache", "maple_b200", "autotune.json")


@dataclass
class TuneResult:
    settings: Dict[str, object]
    ms_per_step: float
    default_ms_per_step: float
    trials: List[dict] = field(default_factory=list)
    cached: bool = False


def apply(ctx: HomogenizationContext, settings: Dict[str, object]) -> None:
    """Apply a setting dict (missing keys: the defaults) to a context."""
    s = dict(DEFAULTS, **settings)
    ctx.set_options(cheb_degree=int(s["fine_degree"]), check_every=int(s["check_every"]),
                    coarse_degree=int(s["coarse_degree"]))
    ctx.set_stencil_nine(int(s["nine_max_n"]))
    ctx.set_stencil_split(int(s["split_min_n"]))
    ctx.set_tail_fused(bool(s["tail_fused"]))
    ctx.set_pdl(bool(s["pdl"]))
    ctx.set_device_loop(bool(s["device_loop"]))
    ctx.set_mixed_mode(str(s["mixed_mode"]))


def _key(ctx, precision, rtol):
    name = torch.cuda.get_device_name(ctx.device).replace(" ", "_")
    return f"{name}|r{ctx.r}|B{ctx.B}|{precision}|{rtol:g}"


def _time(ctx, x0, w, vf, kw, steps) -> float:
    x = x0
    out = ctx.oc_step(x, w, vf, **dict(kw, warm=False))
    x = out["x_next"].clone()
    ms = 0.0
    for _ in range(steps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        out = ctx.oc_step(x, w, vf, **dict(kw, warm=True))
        e1.record()
        torch.cuda.synchronize(ctx.device)
        ms += e0.elapsed_time(e1)
        x = out["x_next"].clone()
    return ms / steps


def autotune(ctx: HomogenizationContext, x: torch.Tensor, weights: torch.Tensor, volfrac: torch.Tensor, *,
             precision: str = "mixed", rtol: float = 1e-8, maxit: int = 500, steps: int = 3, passes: int = 2,
             penal: float = 3.0, rho_min: float = 1e-9, move: float = 0.2, xmin: float = 1e-3, filter_k: int = 3,
             cache: Optional[str] = CACHE, use_cache: bool = True, space: Optional[dict] = None) -> TuneResult:
    """Find and apply the fastest setting for OC steps of these cells.
    x (B, r^3), weights (B, 3), volfrac (B,) as for ``oc_step``; the context
    keeps its warm-start state from the last trial, so callers start their
    own run with warm=False or from fresh solutions."""
    key = _key(ctx, precision, rtol)
    if cache and use_cache and os.path.exists(cache):
        try:
            with open(cache) as f:
                hit = json.load(f).get(key)
        except (OSError, ValueError):
            hit = None
        if hit:
            apply(ctx, hit["settings"])
            return TuneResult(dict(hit["settings"]), hit["ms_per_step"], hit["default_ms_per_step"], cached=True)
    space = dict(space or SPACE)
    if precision != "mixed":
        space.pop("mixed_mode", None)
    kw = dict(penal=penal, rho_min=rho_min, move=move, xmin=xmin, filter_k=filter_k, precision=precision,
              rtol=rtol, maxit=maxit)
    x0 = x.contiguous()
    best = dict(DEFAULTS)
    apply(ctx, best)
    _time(ctx, x0, weights, volfrac, kw, 1)  # warm-up: first-use set-up, graph capture
    best_ms = default_ms = _time(ctx, x0, weights, volfrac, kw, steps)
    trials = [dict(settings=dict(best), ms=best_ms)]
    for _ in range(passes):
        improved = False
        for knob, values in space.items():
            start = best[knob]  # already timed with the other knobs as they are
            for v in values:
                if v == start or v == best[knob]:
                    continue
                cand = dict(best, **{knob: v})
                apply(ctx, cand)
                ms = _time(ctx, x0, weights, volfrac, kw, steps)
                trials.append(dict(settings=cand, ms=ms))
                if ms < best_ms * 0.99:  # 1% margin against timing noise
                    best, best_ms, improved = cand, ms, True
        if not improved:
            break
    apply(ctx, best)
    res = TuneResult(best, best_ms, default_ms, trials)
    if cache:
        try:
            os.makedirs(os.path.dirname(cache), exist_ok=True)
            data = {}
            if os.path.exists(cache):
                with open(cache) as f:
                    data = json.load(f)
            data[key] = dict(settings=best, ms_per_step=best_ms, default_ms_per_step=default_ms)
            with open(cache + ".tmp", "w") as f:
                json.dump(data, f, indent=1)
            os.replace(cache + ".tmp", cache)
        except (OSError, ValueError):
            pass
    return res
