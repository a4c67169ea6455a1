"""Host logic of the batched Pareto worker (no GPU): the dataset_log.csv
columns and condition vector of the reference worker (from
tests/golden/generator.npz), its configuration object, the CSV writers and
the penalty settings handed to the OC loop."""
import csv
import os
from types import SimpleNamespace

import numpy as np

from maple_b200 import pareto


def test_columns_match_reference(golden):
    g = golden("generator.npz")
    assert pareto.FIELDNAMES == [str(s) for s in g["fieldnames"]]
    assert pareto.CONDITION_COLUMNS == [str(s) for s in g["condition_columns"]]


def test_make_cfg_and_defaults():
    cfg = pareto.make_cfg(SimpleNamespace(resolution=32, gmg_smooth_iter=[1, 2], gmg_max_cycle=3))
    assert cfg.resolution == 32 and cfg.GMG.smooth_iter == [1, 2] and cfg.GMG.max_cycle == 3
    cfg = pareto.make_cfg(SimpleNamespace())
    assert cfg.GMG.smooth_iter == [2, 2, 3, 4, 5] and cfg.GMG.max_cycle == 1


def test_dataset_log_roundtrip(tmp_path):
    path = os.path.join(tmp_path, "out", "dataset_log.csv")
    pareto.ensure_dataset_log(path)
    pareto.ensure_dataset_log(path)  # idempotent
    pareto.append_dataset_row(path, {"sample_id": "a", "stiffness": 0.5, "not_a_column": 1})
    with open(path) as f:
        rows = list(csv.DictReader(f))
    assert len(rows) == 1 and rows[0]["sample_id"] == "a" and rows[0]["stiffness"] == "0.5"
    assert list(rows[0]) == pareto.FIELDNAMES and rows[0]["objective"] == ""


def test_penalty_settings():
    kw = pareto._penalty_kwargs(SimpleNamespace(**pareto.WORKER_DEFAULTS))
    assert kw["lambda_print"] == 0.9 and kw["lambda_cavity"] == 0.9 and kw["tiles"] == (2, 2, 2)
    assert kw["min_channel_rad"] == 3 and kw["iters"] == 128 and kw["seed_faces"] == "all"
    a = dict(pareto.WORKER_DEFAULTS, cavity_tiles_xyz="3,1,2")
    assert pareto._penalty_kwargs(SimpleNamespace(**a))["tiles"] == (3, 1, 2)
    a = dict(pareto.WORKER_DEFAULTS, lambda_print=0.0, lambda_cavity=0.0)
    assert pareto._penalty_kwargs(SimpleNamespace(**a)) is None


def test_record_fields():
    task = dict(condition=np.arange(7, dtype=np.float32), lower=dict(weight=0.1, seed=1, vf=0.2, stiffness=1.0,
                shear=2.0, thermal=3.0), upper=SimpleNamespace(weight=0.2, seed=2, vf=0.3, stiffness=4.0, shear=5.0,
                thermal=6.0), weight_tag="w", weight_idx=0, w_stiffness=0.5, w_shear=0.0, w_thermal=0.5,
                objective="stiffness:0.5,thermal:0.5", vf_target=0.25, seed=7, alpha=0.3)
    paths = dict(dir="d", condition="d/c.npy", rho_net="d/n.npy", rho_warm="d/w.npy", rho_final="d/f.npy")
    rec = pareto._record(task, "gpu0-w0", 0, SimpleNamespace(**pareto.WORKER_DEFAULTS), paths, 0.26,
                         dict(stiffness=1.5, shear=0.5, thermal=0.7))
    assert set(pareto.FIELDNAMES) <= set(rec) and rec["ok"] is True
    assert rec["condition_thermal"] == rec["condition_kappa"] == 6.0 and rec["kappa"] == 0.7
    assert rec["source_upper_shear"] == 5.0 and rec["source_lower_kappa"] == 3.0 and rec["final_obj"] == ""
