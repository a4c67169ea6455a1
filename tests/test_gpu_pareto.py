"""The batched Pareto dataset worker on the GPU: every task of a batch gives
the same files and record as a single-cell optimizer run of that task
(optimize_inverse_homogenization + evaluate_homogenized_terms, the reference
worker's per-task calls), and the queue protocol of the reference worker."""
import csv
import os
import queue
from types import SimpleNamespace

import numpy as np
import pytest
import torch

from oracle import generator_oracle as G

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
CFG = dict(cond_dim=7, out_res=32, base_res=4, latent_dim=256, base_channels=128)


def _args(**kw):
    from maple_b200.pareto import WORKER_DEFAULTS
    a = dict(WORKER_DEFAULTS)
    a.update(iters=6, cavity_iters=6, save_iter_log=True, precision="fp64", rtol=1e-10)
    a.update(kw)
    return SimpleNamespace(**a)


def _tasks(root, n):
    rng = np.random.default_rng(12)
    out = []
    for i in range(n):
        ws, wsh = float(rng.uniform(0.2, 0.6)), float(rng.uniform(0.0, 0.3))
        wt = 1.0 - ws - wsh
        vf = float(rng.uniform(0.25, 0.4))
        src = dict(weight=ws, seed=100 + i, vf=vf, stiffness=0.1, shear=0.05, thermal=0.3)
        t = dict(sample_dir=os.path.join(root, f"s{i}"), seed=1000 + i, lower=src, upper=dict(src, weight=ws + 0.05),
                 condition=np.array([ws, wsh, wt, vf, 0.1, 0.05, 0.3], dtype=np.float32),
                 objective=f"stiffness:{ws},shear:{wsh},thermal:{wt}", vf_target=vf, weight_tag=f"w{i}",
                 weight_idx=i, w_stiffness=ws, w_shear=wsh, w_thermal=wt, alpha=0.5, sample_id=f"id{i}")
        if i == 1:  # a latent mixture task
            t["latent_conditions"] = np.stack([t["condition"], t["condition"] * 0.5]).astype(np.float32)
            t["latent_etas"] = np.array([0.6, 0.4], dtype=np.float32)
        out.append(t)
    return out


def _generator():
    from maple_b200.generator import Stage2DensityGenerator
    return Stage2DensityGenerator(**CFG, device=DEV).load_state_dict(G.synthetic_state_dict(seed=21, **CFG))


def test_worker_batch_matches_single_cell_runs(lib, tmp_path):
    from maple_b200.model import IHD
    from maple_b200.optimize import build_unitcell_batch, evaluate_homogenized_terms, optimize_inverse_homogenization
    from maple_b200.pareto import FIELDNAMES, dataset_worker_batch, make_cfg
    args = _args(warm_smooth_passes=1, warm_sigma=0.05)
    tasks = _tasks(str(tmp_path), 3)
    gen = _generator()
    msgs = dataset_worker_batch("gpu0-w0", 0, args, tasks, generator=gen)
    assert [m["ok"] for m in msgs] == [True] * 3, [m.get("traceback") for m in msgs]
    for t, m in zip(tasks, msgs):
        assert set(FIELDNAMES) <= set(m) and m["weight_tag"] == t["weight_tag"]
        for key in ("condition_npy", "rho_net_32_npy", "rho_warmstart_32_npy", "rho_final_npy"):
            assert os.path.exists(m[key]), key
        warm = np.load(m["rho_warmstart_32_npy"])
        assert warm.shape == (32, 32, 32) and warm.dtype == np.float32
        assert abs(float(warm.astype(np.float64).mean()) - t["vf_target"]) < 1e-4
        with open(os.path.join(t["sample_dir"], "iter_log.csv")) as f:
            rows = list(csv.reader(f))
        assert rows[0][:3] == ["iter", "J_total", "J_raw"] and len(rows) == 1 + args.iters

        # the reference worker's per-task path, one cell at a time
        ihd = IHD(make_cfg(args), DEV, precision="fp64", rtol=1e-10)
        rho_warm = torch.from_numpy(warm).to(DEV)
        batch = build_unitcell_batch(DEV, 32, rho_warm)
        one = optimize_inverse_homogenization(
            ihd, batch, res=32, objective=t["objective"], init_mode="voxel", volfrac=t["vf_target"],
            penal=args.penal, rho_min=args.rho_min, move=args.move, xmin=args.xmin, iters=args.iters, seed=t["seed"],
            symmetry=args.symmetry, lambda_print=args.lambda_print, overhang_deg=args.overhang_deg,
            lambda_cavity=args.lambda_cavity, cavity_thresh=args.cavity_thresh, cavity_beta=args.cavity_beta,
            min_channel_rad=args.min_channel_rad, cavity_rad=args.cavity_rad, cavity_seed_faces=args.cavity_seed_faces,
            cavity_iters=args.cavity_iters, cavity_tiles=args.cavity_tiles, cavity_tiles_xyz=args.cavity_tiles_xyz,
            cavity_focus_center=args.cavity_focus_center, filter_k=args.filter_k,
            output_dir=os.path.join(str(tmp_path), "single", t["weight_tag"]), mesh_every=0, mesh_res=64, mesh_iso=0.3,
            mesh_pad=2, save_iter_log=False, save_summary=False, save_initial_mesh=False, verbose=False)
        fin = np.load(m["rho_final_npy"])
        np.testing.assert_allclose(fin, one.rho_final, rtol=0, atol=1e-5)
        assert abs(m["vf_final"] - float(one.rho_final.mean())) < 1e-6
        ref = evaluate_homogenized_terms(ihd, batch, torch.from_numpy(one.rho_final).to(DEV).reshape(-1, 1).double())
        for k in ("stiffness", "shear", "thermal"):
            assert abs(m[k] - ref[k]) <= 1e-5 * abs(ref[k]) + 1e-12, (k, m[k], ref[k])
        ihd.homog_ctx.close()


def test_worker_queue_protocol(lib, tmp_path):
    from maple_b200.pareto import dataset_worker
    path = os.path.join(tmp_path, "gen.pt")
    torch.save({"model": G.synthetic_state_dict(seed=21, **CFG), "args": dict(CFG)}, path)
    args = _args(iters=2, cavity_iters=2, save_iter_log=False, batch_cells=2, checkpoint=path,
                 precision="mixed", rtol=1e-8)
    tasks = _tasks(str(tmp_path), 3)
    tq, rq = queue.Queue(), queue.Queue()
    for t in tasks:
        tq.put(t)
    tq.put(None)
    dataset_worker("gpu0-w0", 0, args, tq, rq)
    msgs = [rq.get_nowait() for _ in range(3)]
    assert rq.empty() and tq.empty()
    assert all(m["ok"] for m in msgs), [m.get("traceback") for m in msgs]
    assert sorted(m["weight_tag"] for m in msgs) == ["w0", "w1", "w2"]
    assert all(m["checkpoint"] == os.path.abspath(path) for m in msgs)
    # a worker without a device reports one failure message and returns
    rq2 = queue.Queue()
    dataset_worker("cpu-w0", None, args, queue.Queue(), rq2)
    m = rq2.get_nowait()
    assert m["ok"] is False and "CUDA device" in m["traceback"]
