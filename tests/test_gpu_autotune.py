"""The autotuner: it times candidate settings on the caller's cells, applies
the fastest, caches it, and whatever it picks solves to the same answer."""
import json

import numpy as np
import pytest
import torch

from oracle import ihd_oracle as O

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


def _cells(r, B):
    x = np.stack([O.seed_density(s, r, 2.0, 0.3).reshape(-1) for s in range(B)])
    w = np.array([[0.5, 0.0, 0.5], [0.2, 0.3, 0.5], [0.0, 1.0, 0.0]])[:B]
    return (torch.tensor(x, device=DEV), torch.tensor(w, device=DEV),
            torch.tensor(np.full(B, 0.3), device=DEV))


def test_autotune_picks_from_its_space_and_keeps_the_answer(lib, tmp_path):
    from maple_b200 import autotune as A
    from maple_b200.core import HomogenizationContext
    r, B = 16, 3
    x, w, vf = _cells(r, B)
    kw = dict(precision="mixed", rtol=1e-10, maxit=500, warm=False)
    ref_ctx = HomogenizationContext(r, ncells=B, device=DEV)
    ref = ref_ctx.oc_step(x, w, vf, **kw)
    ref_J, ref_x = ref["J"].cpu().numpy(), ref["x_next"].cpu().numpy()
    ref_ctx.close()
    ctx = HomogenizationContext(r, ncells=B, device=DEV)
    cache = str(tmp_path / "tune.json")
    space = dict(fine_degree=[1, 2], coarse_degree=[0, 4], nine_max_n=[0, 64], mixed_mode=["flexible", "reliable"])
    res = A.autotune(ctx, x, w, vf, precision="mixed", rtol=1e-10, steps=1, passes=1, cache=cache, space=space)
    for k, vals in space.items():
        assert res.settings[k] in vals
    assert len(res.trials) == 1 + sum(len(v) - 1 for v in space.values())
    assert res.ms_per_step <= res.default_ms_per_step
    out = ctx.oc_step(x, w, vf, **kw)
    assert np.abs(out["J"].cpu().numpy() - ref_J).max() <= 1e-9 * np.abs(ref_J).max()
    assert np.abs(out["x_next"].cpu().numpy() - ref_x).max() <= 1e-7
    with open(cache) as f:
        assert len(json.load(f)) == 1
    again = A.autotune(ctx, x, w, vf, precision="mixed", rtol=1e-10, cache=cache)
    assert again.cached and again.settings == res.settings
    ctx.close()
