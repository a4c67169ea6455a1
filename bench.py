"""Benchmark: OC iterations per second of the inverse-homogenization inner loop.

Workload (the precision configuration): one periodic 64^3 cell (262,144
elements; 786k elastic DOF x 6 load cases + 262k thermal DOF x 3), seeded
density (seed = rank, N(0,1) voxels, periodic Gaussian sigma 4, affine map to
mean 0.25, clip [0.001, 1]), J = (E + G + trace kappa)/3, vf 0.25, move 0.2,
3^3 sensitivity filter, SIMP p=3, rho_min=1e-9.  Each step is one full OC
iteration (SIMP map, 6+3 MG-PCG solves with FP32 multigrid inside FP64
iterative refinement to rtol 1e-10, FP64 C^H / kappa^H, analytic
sensitivities, filter, OC bisection).  Inputs are synthetic.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl maple|reference]

Multi-GPU: one process per GPU (torchrun), each rank an independent replica
cell (the path shards by cell, no data-path collective); value = all ranks'
steps / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "OC iters/s & C^H solves/s, 32³/64³: mixed+learned vs plain FP64, rel err ≤1e-6"
UNIT = "OC iters/s"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="maple", choices=["maple", "reference"])
    p.add_argument("--res", type=int, default=64)
    p.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    p.add_argument("--rtol", type=float, default=1e-10)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-e2e", action="store_true")
    p.add_argument("--serial", action="store_true",
                   help="run the elastic and thermal solves one after the other on one host thread")
    return p.parse_args()


def seeded_design(seed, r, sigma, vf, scale=0.25, xmin=1e-3):
    """Benchmark input: N(0,1) voxels, periodic Gaussian smoothing (FFT),
    standardised, affine map to mean vf, clipped, mean-matched."""
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


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index, self.proc, self.lines = index, None, []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.index)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


# ---------------------------------------------------------------------------
TRAFFIC_FILE = "profiles/k_apply_fine_64cube_full.md"


def measured_traffic(kernel, res):
    """DRAM bytes (read + write) per launch of `kernel` from the committed ncu
    capture, which was taken on the 64^3 workload; None otherwise."""
    import re
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), TRAFFIC_FILE)
    if res != 64 or not os.path.exists(path):
        return None
    m = re.search(r"traffic_bytes_per_launch\[" + re.escape(kernel) + r"\] = (\d+)", open(path).read())
    return int(m.group(1)) if m else None


def max_over_ranks(value: float, world: int, device) -> float:
    """The largest of every rank's `value` (all ranks take part; world 1:
    the value itself).  Device times of a multi-GPU run are reported as the
    max over ranks."""
    if world <= 1:
        return float(value)
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_maple(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist

    from maple_b200.core import HomogenizationContext, launch_count

    dev = torch.device("cuda", local_rank)
    torch.cuda.set_device(dev)
    r = args.res
    ctx = HomogenizationContext(r, ncells=1, device=dev)
    ctx.set_concurrency(not args.serial)
    w = torch.tensor([[1 / 3, 1 / 3, 1 / 3]], dtype=torch.float64, device=dev)
    vf = torch.tensor([0.25], dtype=torch.float64, device=dev)
    x0 = seeded_design(rank, r, sigma=r / 16.0, vf=0.25)
    x = torch.tensor(x0.reshape(1, -1), dtype=torch.float64, device=dev)
    kw = dict(penal=3.0, rho_min=1e-9, move=0.2, xmin=1e-3, filter_k=3, precision=args.precision, rtol=args.rtol,
              maxit=500, warm=True)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)  # > 126 MB L2

    def barrier():
        if world > 1:
            dist.barrier()

    # warm-up (advances the design)
    out = None
    for _ in range(args.warmup):
        out = ctx.oc_step(x, w, vf, **kw)
        x = out["x_next"].clone()
    torch.cuda.synchronize()

    # timed region: K steps, each bracketed by events; L2 flushed between steps
    sampler = ClockSampler(local_rank)
    sampler.start()
    time.sleep(0.3)
    barrier()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    iters = []
    lc0 = launch_count()
    t_wall = time.perf_counter()
    for k in range(args.steps):
        flush.fill_(float(k))
        ev[k][0].record()
        out = ctx.oc_step(x, w, vf, **kw)
        ev[k][1].record()
        x = out["x_next"]
        iters.append(int(out["iters"][0]))
        x = x.clone()
    torch.cuda.synchronize()
    t_wall = time.perf_counter() - t_wall
    launches = launch_count() - lc0
    barrier()
    clocks = sampler.stop()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    t_dev = max_over_ranks(sum(step_ms) / 1000.0, world, dev)
    value = world * args.steps / t_dev

    # live roofline of the dominant kernel class over K further steps
    ctx.profile(True, max_launches=200000)
    for k in range(args.steps):
        flush.fill_(float(k))
        out = ctx.oc_step(x, w, vf, **kw)
        x = out["x_next"].clone()
    torch.cuda.synchronize()
    prof = ctx.profile_read()
    ctx.profile(False)
    peak, peak_kind = measured_peaks()
    # the kernel class with the most device time among those with known
    # algorithmic bytes (grid transfers and PCG vector updates carry none)
    known = [kv for kv in prof.items() if kv[1]["bytes_per_launch"] > 0]
    top_name, top = max(known, key=lambda kv: kv[1]["total_ms"]) if known else (None, None)
    roofline = None
    if top:
        avg_s = top["total_ms"] / top["launches"] / 1000.0
        achieved = top["bytes_per_launch"] / avg_s / 1e9
        roofline = {"bound": "hbm", "kernel": top_name, "achieved": round(achieved, 1), "peak": peak,
                    "peak_source": peak_kind, "unit": "GB/s", "frac": round(achieved / peak, 4),
                    "traffic": measured_traffic(top_name, args.res), "avg_launch_us": round(avg_s * 1e6, 2),
                    "launches_per_step": top["launches"] / args.steps, "bytes_per_launch": top["bytes_per_launch"],
                    "share_of_step_kernel_time": round(top["total_ms"] / sum(v["total_ms"] for v in prof.values()),
                                                       3)}
        if roofline["traffic"] is not None:
            roofline["traffic_source"] = TRAFFIC_FILE

    # end to end through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        x_host = torch.tensor(x.cpu().numpy(), dtype=torch.float64).pin_memory()
        x_out = torch.empty_like(x_host).pin_memory()
        J_out = torch.empty((1,), dtype=torch.float64).pin_memory()
        barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e_ms = 0.0
        for k in range(args.steps):
            flush.fill_(float(k))
            e0.record()
            xd = x_host.to(dev, non_blocking=True)
            out = ctx.oc_step(xd, w, vf, **kw)
            x_out.copy_(out["x_next"], non_blocking=True)
            J_out.copy_(out["J"], non_blocking=True)
            e1.record()
            torch.cuda.synchronize()
            e_ms += e0.elapsed_time(e1)
            x_host.copy_(x_out)
        t_e2e = max_over_ranks(e_ms / 1000.0, world, dev)
        e2e = {"value": round(world * args.steps / t_e2e, 3), "unit": UNIT,
               "h2d_bytes_per_step": int(x_host.numel() * 8), "d2h_bytes_per_step": int(x_out.numel() * 8 + 8)}

    return dict(value=value, t_dev=t_dev, step_ms=step_ms, wall=t_wall, launches=launches, clocks=clocks,
                roofline=roofline, e2e=e2e, iters=iters, levels=ctx.levels, J=float(out["J"][0]))


# ---------------------------------------------------------------------------
def _oracle_step(r, precision_note=None):
    from oracle import ihd_oracle as O
    x = seeded_design(0, r, sigma=r / 16.0, vf=0.25)
    lv = int(np.log2(r // 4)) + 1
    t = time.perf_counter()
    O.oc_iteration(x, r, {"stiffness": 1 / 3, "shear": 1 / 3, "thermal": 1 / 3}, volfrac=0.25, move=0.2,
                   levels=lv, rtol=1e-10, max_cycles=500)
    return time.perf_counter() - t


def cpu_baseline(res):
    """The FP64 oracle (the reference's V-cycle algorithm restated in numpy/scipy)
    on the host cores: one OC iteration at 32^3, scaled to the bench cell by
    element count."""
    rs = 32
    t = _oracle_step(rs)
    scale = (res / rs) ** 3
    return {"value": round(1.0 / (t * scale), 6), "unit": UNIT, "cores": 1, "kind": "port",
            "sample": f"1 OC iteration at {rs}^3 (tri-objective, FP64 V-cycles to rtol 1e-10) = {t:.2f} s, "
                      f"scaled x{scale:g} to {res}^3 by element count"}


def run_reference(args):
    """Reference arm: the oracle port of the reference's CPU path, one bounded
    sample per step (one OC iteration at 16^3, scaled to the bench cell)."""
    rs = 16
    scale = (args.res / rs) ** 3
    for _ in range(args.warmup):
        _oracle_step(rs)
    ts = [_oracle_step(rs) for _ in range(args.steps)]
    tot = sum(ts) * scale
    value = args.steps / tot
    return {"metric": METRIC, "value": round(value, 6), "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1000 * tot / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": f"OC iteration, {args.res}^3 periodic cell, tri-objective, vf 0.25",
                       "res": args.res},
            "cpu_baseline": {"value": round(value, 6), "unit": UNIT, "cores": 1, "kind": "port",
                             "sample": f"{args.steps} x 1 OC iteration at {rs}^3 (FP64 V-cycles to 1e-10), "
                                       f"scaled x{scale:g} by element count"},
            "e2e": {"value": round(value, 6), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args)), flush=True)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    res = run_maple(args, rank, world, local_rank)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args.res)
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(res["value"], 3), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(1000 * res["t_dev"] / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64+f32" if args.precision == "mixed" else "f64",
            "data": "synthetic",
            "config": {"workload": f"OC iteration, {args.res}^3 periodic cell (config 1: precision)",
                       "res": args.res, "precision": args.precision, "rtol": args.rtol,
                       "solves": "one after the other" if args.serial else "elastic and thermal concurrent",
                       "objective": "(E+G+kappa)/3", "volfrac": 0.25, "move": 0.2, "filter_k": 3,
                       "mg_levels": res["levels"], "l2": "flushed between steps (256 MiB write outside the events)",
                       "parallelism": f"replicas x{world}", "pcg_iters_per_step": res["iters"]},
            "gpu_launches": int(res["launches"]), "clocks": res["clocks"], "roofline": res["roofline"],
            "cpu_baseline": cpu, "e2e": res["e2e"], "wall_s": round(res["wall"], 3),
            "step_ms": [round(v, 3) for v in res["step_ms"]], "J_last": res["J"],
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
