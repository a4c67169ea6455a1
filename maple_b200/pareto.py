"""Pareto dataset worker, batched: many 32^3 optimizer runs per launch.

Drop-in for ``dataset_worker`` of pareto/densify_pareto_property_network_32.py
(:1055-1256).  The reference's worker takes one task at a time from a queue and
runs, per task: Stage-II generator inference, warm-start post-processing
(noise, periodic binomial smoothing, clamped mean matching), one OC run of
``optimize_inverse_homogenization`` (symmetry and printability penalties on)
and ``evaluate_homogenized_terms`` of the final density.  Here a worker drains
up to ``batch_cells`` tasks and advances them together: one generator pass for
all conditions, the warm-start kernels over all cells, then one batched OC loop
(``batch.oc_run``) in which every kernel launch serves every still-running
cell, each cell stopping on the reference's own stall test, and one batched
evaluation.  Per task it writes the same files (``condition.npy``,
``rho_net_32.npy``, ``rho_warmstart_32.npy``, ``rho_final.npy``, optionally
``iter_log.csv``) and returns the same result record (``FIELDNAMES`` keys plus
``ok`` / ``worker`` / ``gpu_id``).

Not produced: the final marching-cubes mesh (``meshes/final.obj``); the
record's ``final_obj`` is the empty string.
"""
from __future__ import annotations

import csv
import os
import queue as _queue
import traceback
from typing import Dict, List, Optional, Sequence

import numpy as np
import torch

from .batch import ITER_LOG_COLUMNS, oc_run
from .core import HomogenizationContext
from .generator import Stage2DensityGenerator, binomial_smooth_periodic, load_generator, match_mean_clamped
from .objective import objective_weights, shear_objective, stiffness_objective, thermal_objective
from .optimize import _parse_tiles_xyz

RES = 32

# dataset_log.csv columns and the generator's condition vector
# (pareto/densify_pareto_property_network_32.py:25-82)
CONDITION_COLUMNS = ["w_stiffness", "w_shear", "w_thermal", "vf_target", "stiffness", "shear", "thermal"]
FIELDNAMES = [
    "sample_id", "front_objectives", "weight_tag", "weight_idx", "w_stiffness", "w_shear", "w_thermal", "objective",
    "vf_target", "vf_final", "seed", "sampling_mode", "front_gap", "front_interval_rank", "tri_front_edge",
    "condition_npy", "condition_stiffness", "condition_shear", "condition_thermal", "condition_kappa",
    "source_lower_w", "source_upper_w", "source_alpha", "source_lower_seed", "source_upper_seed", "source_lower_vf",
    "source_upper_vf", "source_lower_stiffness", "source_lower_shear", "source_lower_thermal", "source_lower_kappa",
    "source_upper_stiffness", "source_upper_shear", "source_upper_thermal", "source_upper_kappa", "rho_net_32_npy",
    "rho_warmstart_32_npy", "stiffness", "shear", "thermal", "kappa", "sample_dir", "rho_final_npy", "final_obj",
    "checkpoint", "source_csv",
]

# the worker's argparse defaults (densify_pareto_property_network_32.py:100-221) for the fields it reads
WORKER_DEFAULTS = dict(
    resolution=32, iters=2000, penal=3.0, rho_min=1.0e-5, move=0.05, xmin=1.0e-5, filter_k=3, symmetry="iso",
    lambda_print=0.9, overhang_deg=45.0, lambda_cavity=0.9, cavity_thresh=0.5, cavity_beta=20.0, min_channel_rad=3,
    cavity_rad=1, cavity_seed_faces="all", cavity_iters=128, cavity_tiles=2, cavity_tiles_xyz=None,
    cavity_focus_center=True, gmg_smooth_iter=[2, 2, 3, 4, 5], gmg_max_cycle=1, warm_sigma=0.0,
    warm_smooth_passes=0, volume_iters=8, match_volume=True, save_iter_log=False, quiet=True,
    optimizer_verbose=False, checkpoint="", source_csv="",
    # this implementation only: cells per batch, solver precision and tolerance
    batch_cells=64, precision="mixed", rtol=1e-8, maxit=500,
)


def _arg(args, name):
    return getattr(args, name, WORKER_DEFAULTS[name])


def make_cfg(args):
    """The IHD configuration object of the worker (densify...py:974-980)."""
    cfg = type("Cfg", (), {})()
    cfg.resolution = int(_arg(args, "resolution"))
    cfg.GMG = type("GMG", (), {})()
    cfg.GMG.smooth_iter = list(_arg(args, "gmg_smooth_iter"))
    cfg.GMG.max_cycle = int(_arg(args, "gmg_max_cycle"))
    return cfg


def ensure_dataset_log(log_csv: str) -> None:
    if os.path.exists(log_csv):
        return
    os.makedirs(os.path.dirname(os.path.abspath(log_csv)), exist_ok=True)
    with open(log_csv, "w", encoding="utf-8", newline="") as f:
        csv.DictWriter(f, fieldnames=FIELDNAMES).writeheader()


def append_dataset_row(log_csv: str, row: Dict[str, object]) -> None:
    with open(log_csv, "a", encoding="utf-8", newline="") as f:
        csv.DictWriter(f, fieldnames=FIELDNAMES).writerow({k: row.get(k, "") for k in FIELDNAMES})


def _penalty_kwargs(args) -> Optional[dict]:
    lp, lc = float(_arg(args, "lambda_print")), float(_arg(args, "lambda_cavity"))
    if lp <= 0.0 and lc <= 0.0:
        return None
    return dict(lambda_print=lp, overhang_deg=float(_arg(args, "overhang_deg")), lambda_cavity=lc,
                void_thresh=float(_arg(args, "cavity_thresh")), beta=float(_arg(args, "cavity_beta")),
                min_channel_rad=int(_arg(args, "min_channel_rad")), rad=int(_arg(args, "cavity_rad")),
                iters=int(_arg(args, "cavity_iters") or 0),
                tiles=_parse_tiles_xyz(_arg(args, "cavity_tiles_xyz"), int(_arg(args, "cavity_tiles"))),
                focus_center=bool(_arg(args, "cavity_focus_center")), seed_faces=str(_arg(args, "cavity_seed_faces")),
                periodic=True)


def warm_start(generator: Stage2DensityGenerator, tasks: Sequence[dict], args, device):
    """(rho_net, rho_warm), each (B, 32^3) float32 on the device: the
    generator's densities (latent mixtures where a task carries
    latent_conditions / latent_etas) and the warm starts after the optional
    noise, smoothing and mean matching (densify...py:1082-1111)."""
    B = len(tasks)
    cond = np.stack([np.asarray(t["condition"], dtype=np.float32) for t in tasks])
    lat = generator.encode_latent(torch.from_numpy(cond))
    mixed = [i for i, t in enumerate(tasks) if "latent_conditions" in t and "latent_etas" in t]
    if mixed:
        for i in mixed:
            lc = np.asarray(tasks[i]["latent_conditions"], dtype=np.float32)
            eta = torch.as_tensor(np.asarray(tasks[i]["latent_etas"], dtype=np.float32), device=device).reshape(-1, 1)
            lat[i] = (generator.encode_latent(torch.from_numpy(lc)) * eta).sum(0)
    rho_net = generator.decode_latent(lat).reshape(B, -1)
    warm = rho_net.clone()
    sigma = float(_arg(args, "warm_sigma"))
    if sigma > 0.0:
        for i, t in enumerate(tasks):  # setup_seed(seed) then randn_like on the device's default generator
            g = torch.Generator(device=device).manual_seed(int(t["seed"]))
            warm[i] += sigma * torch.randn(warm.shape[1], generator=g, device=device, dtype=torch.float32)
    passes = int(_arg(args, "warm_smooth_passes"))
    if passes > 0:
        warm = binomial_smooth_periodic(warm.reshape(B, RES, RES, RES), passes).reshape(B, -1)
    rho_min = float(_arg(args, "rho_min"))
    if bool(_arg(args, "match_volume")):
        warm = match_mean_clamped(warm, [float(t["vf_target"]) for t in tasks], rho_min, int(_arg(args, "volume_iters")))
    else:
        warm = warm.clamp(rho_min, 1.0)
    return rho_net, warm


def _record(task, worker_name, gpu_id, args, paths, vf_final, metrics) -> dict:
    lower, upper = task["lower"], task["upper"]
    condition = np.asarray(task["condition"], dtype=np.float32)
    L = lambda s, k: getattr(s, k) if not isinstance(s, dict) else s[k]  # noqa: E731
    return {
        "ok": True, "worker": worker_name, "gpu_id": gpu_id,
        "sample_id": task.get("sample_id", ""), "front_objectives": task.get("front_objectives", ""),
        "weight_tag": task["weight_tag"], "weight_idx": task["weight_idx"],
        "w_stiffness": task["w_stiffness"], "w_shear": task["w_shear"], "w_thermal": task["w_thermal"],
        "objective": task["objective"], "vf_target": float(task["vf_target"]), "vf_final": float(vf_final),
        "seed": int(task["seed"]), "sampling_mode": task.get("sampling_mode", ""),
        "front_gap": task.get("front_gap", ""), "front_interval_rank": task.get("front_interval_rank", ""),
        "tri_front_edge": task.get("tri_front_edge", ""),
        "condition_npy": os.path.abspath(paths["condition"]),
        "condition_stiffness": float(condition[4]), "condition_shear": float(condition[5]),
        "condition_thermal": float(condition[6]), "condition_kappa": float(condition[6]),
        "source_lower_w": L(lower, "weight"), "source_upper_w": L(upper, "weight"),
        "source_alpha": float(task["alpha"]),
        "source_lower_seed": L(lower, "seed"), "source_upper_seed": L(upper, "seed"),
        "source_lower_vf": L(lower, "vf"), "source_upper_vf": L(upper, "vf"),
        "source_lower_stiffness": L(lower, "stiffness"), "source_lower_shear": L(lower, "shear"),
        "source_lower_thermal": L(lower, "thermal"), "source_lower_kappa": L(lower, "thermal"),
        "source_upper_stiffness": L(upper, "stiffness"), "source_upper_shear": L(upper, "shear"),
        "source_upper_thermal": L(upper, "thermal"), "source_upper_kappa": L(upper, "thermal"),
        "rho_net_32_npy": os.path.abspath(paths["rho_net"]), "rho_warmstart_32_npy": os.path.abspath(paths["rho_warm"]),
        "stiffness": metrics["stiffness"], "shear": metrics["shear"], "thermal": metrics["thermal"],
        "kappa": metrics["thermal"], "sample_dir": os.path.abspath(paths["dir"]),
        "rho_final_npy": os.path.abspath(paths["rho_final"]), "final_obj": "",
        "checkpoint": os.path.abspath(str(_arg(args, "checkpoint"))) if _arg(args, "checkpoint") else "",
        "source_csv": os.path.abspath(str(_arg(args, "source_csv"))) if _arg(args, "source_csv") else "",
    }


def evaluate_terms(ctx: HomogenizationContext, rho: torch.Tensor, precision: str, rtol: float, maxit: int):
    """(B, 3) stiffness, shear, thermal of fixed densities rho (B, N) float64,
    each as evaluate_homogenized_terms (main_IHD_v3.py:431-466)."""
    out = np.zeros((rho.shape[0], 3))
    ctx.set_density("thermal", rho, precision)
    ctx.solve("thermal", precision=precision, rtol=rtol, maxit=maxit)
    K = ctx.homogenize("thermal").cpu()
    ctx.set_density("elastic", rho, precision)
    ctx.solve("elastic", precision=precision, rtol=rtol, maxit=maxit)
    CH = ctx.homogenize("elastic").cpu()
    for b in range(rho.shape[0]):
        out[b] = (float(stiffness_objective(CH[b])), float(shear_objective(CH[b])), float(thermal_objective(K[b])))
    return out


def dataset_worker_batch(worker_name: str, gpu_id: Optional[int], args, tasks: Sequence[dict], *,
                         generator: Optional[Stage2DensityGenerator] = None,
                         ctx: Optional[HomogenizationContext] = None) -> List[dict]:
    """Run `tasks` together; returns one result message per task, in order
    (``{"ok": False, "traceback": ...}`` for a task whose files could not be
    written; a failure of the batched compute fails every task of the batch)."""
    if not tasks:
        return []
    if int(_arg(args, "resolution")) != RES:
        raise ValueError(f"This worker is fixed to 32-resolution TO, got resolution {_arg(args, 'resolution')}")
    if gpu_id is None:
        raise RuntimeError(f"{worker_name}: this implementation runs on a CUDA device (gpu_id=None)")
    device = torch.device("cuda", int(gpu_id))
    generator = generator or load_generator(str(_arg(args, "checkpoint")), device)
    B = len(tasks)
    results: List[Optional[dict]] = [None] * B
    penal, rho_min, xmin = float(_arg(args, "penal")), float(_arg(args, "rho_min")), float(_arg(args, "xmin"))

    def fail(i, exc_text):
        t = tasks[i]
        results[i] = {"ok": False, "worker": worker_name, "gpu_id": gpu_id, "weight_tag": t.get("weight_tag"),
                      "seed": t.get("seed"), "traceback": exc_text}

    with torch.no_grad(), torch.cuda.device(device):
        rho_net, rho_warm = warm_start(generator, tasks, args, device)
        net_np = rho_net.reshape(B, RES, RES, RES).cpu().numpy().astype(np.float32)
        warm_np = rho_warm.reshape(B, RES, RES, RES).cpu().numpy().astype(np.float32)
        paths = []
        for i, t in enumerate(tasks):
            d = str(t["sample_dir"])
            p = dict(dir=d, condition=os.path.join(d, "condition.npy"), rho_net=os.path.join(d, "rho_net_32.npy"),
                     rho_warm=os.path.join(d, "rho_warmstart_32.npy"), rho_final=os.path.join(d, "rho_final.npy"))
            paths.append(p)
            try:
                os.makedirs(d, exist_ok=True)
                np.save(p["condition"], np.asarray(t["condition"], dtype=np.float32))
                np.save(p["rho_net"], net_np[i])
                np.save(p["rho_warm"], warm_np[i])
            except Exception:
                fail(i, traceback.format_exc())
        # init_mode "voxel" (main_IHD_v3.py:548-551), then the batched OC loop
        rho0 = rho_warm.double().clamp(rho_min, 1.0)
        x0 = ((rho0 - rho_min) / (1.0 - rho_min)).clamp(0.0, 1.0).pow(1.0 / penal).clamp(xmin, 1.0).contiguous()
        w = np.array([objective_weights(str(t["objective"])) for t in tasks], dtype=np.float64)
        vf = np.array([float(t["vf_target"]) for t in tasks], dtype=np.float64)
        own_ctx = ctx is None
        ctx = ctx or HomogenizationContext(RES, ncells=B, device=device)
        try:
            res = oc_run(x0, w, vf, r=RES, move=float(_arg(args, "move")), xmin=xmin, penal=penal, rho_min=rho_min,
                         filter_k=int(_arg(args, "filter_k")), precision=str(_arg(args, "precision")),
                         rtol=float(_arg(args, "rtol")), maxit=int(_arg(args, "maxit")),
                         max_iters=int(_arg(args, "iters")), ctx=ctx, device=device,
                         symmetry=str(_arg(args, "symmetry")), penalties=_penalty_kwargs(args),
                         stop_rule="reference", log_rows=bool(_arg(args, "save_iter_log")))
            rho_final = (rho_min + (1.0 - rho_min) * res.x.clamp(xmin, 1.0) ** penal).clamp(rho_min, 1.0)
            final_np = rho_final.reshape(B, RES, RES, RES).cpu().numpy().astype(np.float32)
            # the reference evaluates the FP32-rounded final density
            rho_eval = torch.from_numpy(final_np.reshape(B, -1)).to(device=device, dtype=torch.float64).contiguous()
            terms = evaluate_terms(ctx, rho_eval, str(_arg(args, "precision")), float(_arg(args, "rtol")),
                                   int(_arg(args, "maxit")))
        finally:
            if own_ctx:
                ctx.close()
    for i, t in enumerate(tasks):
        if results[i] is not None:
            continue
        try:
            np.save(paths[i]["rho_final"], final_np[i])
            if bool(_arg(args, "save_iter_log")):
                with open(os.path.join(paths[i]["dir"], "iter_log.csv"), "w", newline="") as f:
                    wr = csv.writer(f)
                    wr.writerow(ITER_LOG_COLUMNS)
                    wr.writerows(res.logs[i])
            metrics = dict(stiffness=float(terms[i, 0]), shear=float(terms[i, 1]), thermal=float(terms[i, 2]))
            results[i] = _record(t, worker_name, gpu_id, args, paths[i], final_np[i].mean(), metrics)
        except Exception:
            fail(i, traceback.format_exc())
    return results


def dataset_worker(worker_name: str, gpu_id: Optional[int], args, task_queue, result_queue) -> None:
    """The reference worker's signature and protocol: take tasks from
    task_queue until None, put one message per task on result_queue.  Tasks
    are taken in batches of up to ``args.batch_cells`` (the first blocking,
    the rest as available) and run by dataset_worker_batch."""
    try:
        if gpu_id is None:
            raise RuntimeError(f"{worker_name}: this implementation runs on a CUDA device (gpu_id=None)")
        if not torch.cuda.is_available():
            raise RuntimeError(f"{worker_name}: CUDA unavailable for gpu_id={gpu_id}")
        torch.cuda.set_device(gpu_id)
        device = torch.device(f"cuda:{gpu_id}")
        generator = load_generator(str(_arg(args, "checkpoint")), device)
        cap = max(1, int(_arg(args, "batch_cells")))
        done = False
        while not done:
            batch = []
            task = task_queue.get()
            if task is None:
                break
            batch.append(task)
            while len(batch) < cap:
                try:
                    task = task_queue.get_nowait()
                except _queue.Empty:
                    break
                if task is None:
                    done = True
                    break
                batch.append(task)
            try:
                msgs = dataset_worker_batch(worker_name, gpu_id, args, batch, generator=generator)
            except Exception:
                tb = traceback.format_exc()
                msgs = [{"ok": False, "worker": worker_name, "gpu_id": gpu_id, "weight_tag": t.get("weight_tag"),
                         "seed": t.get("seed"), "traceback": tb} for t in batch]
            for m in msgs:
                result_queue.put(m)
            torch.cuda.empty_cache()
    except Exception:
        result_queue.put({"ok": False, "worker": worker_name, "gpu_id": gpu_id, "weight_tag": None, "seed": None,
                          "traceback": traceback.format_exc()})


__all__ = ["CONDITION_COLUMNS", "FIELDNAMES", "WORKER_DEFAULTS", "make_cfg", "ensure_dataset_log",
           "append_dataset_row", "warm_start", "evaluate_terms", "dataset_worker_batch", "dataset_worker"]
