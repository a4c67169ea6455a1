"""Many independent unit cells advanced together.

Every kernel of the library takes a cell index, so B cells with their own
volume fractions, objective weights and stopping points advance in the same
launches: one ``maple_oc_step`` per OC iteration for all still-active cells.
A cell stops when max|dx| < dx_tol or after max_iters iterations; stopped
cells are masked out and cost nothing in later launches.

This replaces the reference's task-level parallelism (one optimizer run per
process / GPU in ``maple/pareto/densify_pareto_property_network_32.py:
1055-1256``) for the inner loop.
"""
from __future__ import annotations

import os
import time
from dataclasses import dataclass, field
from typing import Optional

import numpy as np
import torch

from ._lib import MapleError
from .core import HomogenizationContext


@dataclass
class BatchResult:
    x: torch.Tensor             # (B, r^3) final designs
    J: np.ndarray               # (B,) objective of the last iteration
    terms: np.ndarray           # (B, 3): E, G, trace(kappa)
    iters_run: np.ndarray       # (B,) OC iterations per cell
    converged: np.ndarray       # (B,) stopped by the dx rule
    pcg_iters: np.ndarray       # (B,) PCG iterations summed over the run
    seconds: float
    history: list = field(default_factory=list)
    J_raw: Optional[np.ndarray] = None     # (B,) unpenalised objective of the last iteration
    P_print: Optional[np.ndarray] = None   # (B,) overhang penalty of the last iteration
    P_cavity: Optional[np.ndarray] = None  # (B,) trapped-void penalty of the last iteration
    logs: list = field(default_factory=list)  # per cell: iteration rows (ITER_LOG_COLUMNS)

    @property
    def oc_iterations(self) -> int:
        return int(self.iters_run.sum())


def config2_inputs(B: int = 256, r: int = 32, sigma: float = 2.0, rng_seed: int = 10_000, scale: float = 0.25,
                   xmin: float = 1e-3, seed0: int = 0):
    """Seeded designs of the batched benchmark: cell b uses seed seed0 + b and
    periodic Gaussian smoothing sigma; vf_b ~ U[0.01, 0.40] and weights ~
    Dirichlet(1,1,1), drawn from default_rng(rng_seed) in that order."""
    rng = np.random.default_rng(rng_seed)
    vf = rng.uniform(0.01, 0.40, B)
    w = rng.dirichlet((1.0, 1.0, 1.0), B)
    x = np.stack([seeded_design(seed0 + b, r, sigma, vf[b], scale, xmin).reshape(-1) for b in range(B)])
    return x, w, vf


def seeded_design(seed, r, sigma, vf, scale=0.25, xmin=1e-3):
    """N(0,1) voxels, periodic Gaussian smoothing (FFT), standardised, affine
    map to mean vf, clipped to [xmin, 1], mean-matched."""
    z = np.random.default_rng(seed).standard_normal((r, r, r))
    k = np.fft.fftfreq(r)
    k2 = k[:, None, None] ** 2 + k[None, :, None] ** 2 + k[None, None, :] ** 2
    z = np.real(np.fft.ifftn(np.fft.fftn(z) * np.exp(-2.0 * (np.pi ** 2) * (sigma ** 2) * k2)))
    z = (z - z.mean()) / z.std()
    x = np.clip(vf + scale * z, xmin, 1.0)
    for _ in range(200):
        x = np.clip(x - x.mean() + vf, xmin, 1.0)
        if abs(x.mean() - vf) < 1e-12:
            break
    return x


ITER_LOG_COLUMNS = ["iter", "J_total", "J_raw", "P_print", "P_cavity", "mean_x", "mean_rho", "dx_max", "dx_mean",
                    "time_sec"]
CHECKPOINT_VERSION = 1


def save_checkpoint(path: str, state: dict) -> None:
    """Write a batched OC state (numpy arrays and scalars) to `path` atomically
    (a temporary file renamed over it)."""
    tmp = path + ".tmp.npz"
    np.savez(tmp, version=CHECKPOINT_VERSION, **state)
    os.replace(tmp, path)


def load_checkpoint(path: str) -> dict:
    with np.load(path, allow_pickle=False) as f:
        state = {k: f[k] for k in f.files}
    if int(state.pop("version")) != CHECKPOINT_VERSION:
        raise ValueError(f"{path}: unsupported checkpoint version")
    return state
# stall test of main_IHD_v3.py:611-618, 711-714
STALL_TOL_X, STALL_TOL_J, STALL_PATIENCE, STALL_MIN_ITERS = 1e-3, 1e-4, 10, 10


def oc_run(x0, weights, volfrac, *, r: Optional[int] = None, move: float = 0.2, xmin: float = 1e-3,
           penal: float = 3.0, rho_min: float = 1e-9, filter_k: int = 3, precision: str = "mixed",
           rtol: float = 1e-8, maxit: int = 500, dx_tol: float = 0.01, max_iters: int = 200,
           ctx: Optional[HomogenizationContext] = None, device=None, record: bool = False,
           guess=None, symmetry: str = "none", penalties: Optional[dict] = None, stop_rule: str = "dx",
           log_rows: bool = False, checkpoint: Optional[str] = None, checkpoint_every: int = 0,
           resume: bool = False, checkpoint_fields: bool = False) -> BatchResult:
    """Run B independent OC loops to their own stopping points (with the
    symmetry projection `symmetry`, a spec as in parse_symmetry).  `guess` =
    (elastic (B, 6, 3, N), thermal (B, 3, 1, N)) float64 fields: the initial
    iterates of the first iteration's solves (later iterations start from the
    previous iteration's solutions).

    stop_rule "dx": a cell stops when max|dx| < dx_tol; "reference": the
    optimizer's stall test (main_IHD_v3.py:611-618, 711-714), i.e. after
    STALL_PATIENCE consecutive iterations, from iteration STALL_MIN_ITERS on,
    with max|dx| < STALL_TOL_X and |dJ|/|J_prev| < STALL_TOL_J.  `penalties`:
    keyword arguments of HomogenizationContext.set_penalties, applied to every
    cell (J is then the penalised objective).  log_rows: keep each cell's
    iteration rows (ITER_LOG_COLUMNS, the optimizer's iter_log.csv).

    Checkpoints: with `checkpoint` (a .npz path) and checkpoint_every = k > 0,
    the state of every cell is written after every k-th iteration and at the
    end.  The state is the design, iteration and PCG counts, stop state, last
    objective terms and stall counters.  With checkpoint_fields it also holds
    the solver fields, which are the next warm start.  resume=True continues
    from an existing checkpoint instead of x0 (same cells, shapes and settings),
    up to max_iters iterations in total.  With the fields the continuation
    repeats the uninterrupted run exactly; without them its first solves start
    from zero (same results to the solver tolerance)."""
    if stop_rule not in ("dx", "reference"):
        raise ValueError("stop_rule must be 'dx' or 'reference'")
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    x = torch.as_tensor(x0, dtype=torch.float64).to(dev).reshape(len(volfrac), -1).contiguous()
    B, N = x.shape
    r = r or int(round(N ** (1 / 3)))
    if r ** 3 != N:
        raise ValueError(f"designs must be (B, r^3); got N={N}")
    w = torch.as_tensor(np.asarray(weights), dtype=torch.float64).to(dev).reshape(B, 3).contiguous()
    vf = torch.as_tensor(np.asarray(volfrac), dtype=torch.float64).to(dev).reshape(B).contiguous()
    ctx = ctx or HomogenizationContext(r, ncells=B, device=dev)
    from .optimize import parse_symmetry
    sym_kind, sym_axes = parse_symmetry(symmetry)
    ctx.set_symmetry(sym_kind, sym_axes)
    if sym_kind != "none":
        from .core import symmetrize
        x = symmetrize(x, r, sym_kind, sym_axes).clamp(xmin, 1.0).contiguous()
    if penalties:
        ctx.set_penalties(**penalties)
    if guess is not None:
        ctx.set_solution("elastic", guess[0].contiguous())
        ctx.set_solution("thermal", guess[1].contiguous())
    active = np.ones(B, dtype=np.int32)
    iters = np.zeros(B, dtype=np.int64)
    pcg = np.zeros(B, dtype=np.int64)
    conv = np.zeros(B, dtype=bool)
    J, J_raw, P_print, P_cavity = np.zeros(B), np.zeros(B), np.zeros(B), np.zeros(B)
    J_prev = np.full(B, np.nan)
    stall = np.zeros(B, dtype=np.int64)
    terms = np.zeros((B, 3))
    hist = []
    logs = [[] for _ in range(B)]
    it0 = 0
    if resume:
        if not checkpoint or not os.path.exists(checkpoint):
            raise FileNotFoundError(f"no checkpoint to resume from: {checkpoint}")
        ck = load_checkpoint(checkpoint)
        if tuple(ck["x"].shape) != (B, N) or str(ck["stop_rule"]) != stop_rule:
            raise ValueError("checkpoint does not match this run (cells, resolution or stop rule)")
        x = torch.as_tensor(ck["x"], dtype=torch.float64).to(dev).contiguous()
        active, iters, pcg, conv = (ck["active"].astype(np.int32), ck["iters"].astype(np.int64),
                                    ck["pcg"].astype(np.int64), ck["conv"].astype(bool))
        J, J_raw, P_print, P_cavity = ck["J"], ck["J_raw"], ck["P_print"], ck["P_cavity"]
        J_prev, stall, terms, it0 = ck["J_prev"], ck["stall"].astype(np.int64), ck["terms"], int(ck["it"])
        for phys in ("elastic", "thermal"):
            if f"u_{phys}" in ck:
                ctx.set_solution(phys, torch.as_tensor(ck[f"u_{phys}"]).to(dev).contiguous())

    def write_checkpoint(it_next):
        state = dict(x=x.cpu().numpy(), active=active, iters=iters, pcg=pcg, conv=conv, J=J, J_raw=J_raw,
                     P_print=P_print, P_cavity=P_cavity, J_prev=J_prev, stall=stall, terms=terms, it=it_next,
                     stop_rule=stop_rule)
        if checkpoint_fields:
            for phys in ("elastic", "thermal"):
                try:
                    state[f"u_{phys}"] = ctx.solution(phys).cpu().numpy()
                except MapleError:  # that physics was never solved (no cell weights it)
                    pass
        save_checkpoint(checkpoint, state)

    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    it = it0 - 1
    try:
        for it in range(it0, max_iters):
            if not active.any():
                break
            ctx.set_active(active)
            if log_rows:
                xc = x.clamp(xmin, 1.0)
                means = torch.stack([xc.mean(1), (rho_min + (1.0 - rho_min) * xc ** penal).clamp(rho_min, 1.0)
                                     .mean(1)], 1).cpu().numpy()
            out = ctx.oc_step(x, w, vf, penal=penal, rho_min=rho_min, move=move, xmin=xmin, filter_k=filter_k,
                              precision=precision, rtol=rtol, maxit=maxit, warm=True)
            st = out["stats"].cpu().numpy()
            act = active.astype(bool)
            Jn = out["J"].cpu().numpy()
            J[act] = Jn[act]
            J_raw[act] = out["J_raw"].cpu().numpy()[act]
            P_print[act] = out["P_print"].cpu().numpy()[act]
            P_cavity[act] = out["P_cavity"].cpu().numpy()[act]
            terms[act] = out["terms"].cpu().numpy()[act]
            mask = torch.as_tensor(act, device=dev).reshape(B, 1)
            x = torch.where(mask, out["x_next"].clamp(xmin, 1.0), x).contiguous()
            iters[act] += 1
            pcg[act] += out["iters"][act]
            if stop_rule == "dx":
                done = act & (st[:, 0] < dx_tol)
            else:
                with np.errstate(invalid="ignore", divide="ignore"):
                    dJ = np.where(np.isnan(J_prev), np.inf, np.abs(Jn - J_prev) / np.maximum(np.abs(J_prev), 1e-12))
                ok = (it >= STALL_MIN_ITERS) & (st[:, 0] < STALL_TOL_X) & (dJ < STALL_TOL_J)
                stall = np.where(act, np.where(ok, stall + 1, 0), stall)
                done = act & (stall >= STALL_PATIENCE)
            J_prev = np.where(act, Jn, J_prev)
            if log_rows:
                t_now = time.perf_counter() - t0
                for b in np.nonzero(act)[0]:
                    logs[b].append([int(iters[b]), float(J[b]), float(J_raw[b]), float(P_print[b]),
                                    float(P_cavity[b]), float(means[b, 0]), float(means[b, 1]), float(st[b, 0]),
                                    float(st[b, 1]), t_now])
            conv |= done
            active[done] = 0
            if record:
                hist.append(dict(active=int(act.sum()), J=J.copy(), dx_max=st[:, 0].copy(),
                                 pcg=np.array(out["iters"])))
            if checkpoint and checkpoint_every > 0 and (it + 1) % checkpoint_every == 0:
                write_checkpoint(it + 1)
        if checkpoint and checkpoint_every > 0:
            write_checkpoint(it + 1)
        torch.cuda.synchronize(dev)
    finally:
        ctx.set_active(np.ones(B, dtype=np.int32))
        if sym_kind != "none":
            ctx.set_symmetry("none")
        if penalties:
            ctx.set_penalties(0.0, 45.0, 0.0)
    return BatchResult(x=x, J=J, terms=terms, iters_run=iters, converged=conv, pcg_iters=pcg,
                       seconds=time.perf_counter() - t0, history=hist, J_raw=J_raw, P_print=P_print,
                       P_cavity=P_cavity, logs=logs)
