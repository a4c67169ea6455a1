"""Stage-II generator inference and warm-start kernels on the GPU against the
CPU FP32 oracle (itself pinned to the reference module by
tests/golden/generator.npz).

Tolerances: the MLP and normalisations are FP32 (1e-4); the 3x3x3
convolutions multiply BF16-rounded operands with FP32 accumulation, so the
densities agree with the FP32 module to 1e-2 absolute (2e-3 on average); the
binomial smoothing is bit-identical; the mean matching agrees to 1e-6."""
import os

import numpy as np
import pytest
import torch
import torch.nn.functional as F

from oracle import generator_oracle as G

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")
CONFIGS = {
    "full": dict(cond_dim=7, out_res=32, base_res=4, latent_dim=256, base_channels=128),
    "small": dict(cond_dim=7, out_res=16, base_res=4, latent_dim=64, base_channels=32),
}


def _p(t):
    return None if t is None else t.data_ptr()


def _s():
    return torch.cuda.current_stream(DEV).cuda_stream


def _gen(cfg, seed=11):
    from maple_b200.generator import Stage2DensityGenerator
    g = Stage2DensityGenerator(**cfg, device=DEV)
    return g.load_state_dict(G.synthetic_state_dict(seed=seed, **cfg))


@pytest.mark.parametrize("tag", sorted(CONFIGS))
def test_generator_matches_oracle(lib, tag):
    cfg = CONFIGS[tag]
    state = G.synthetic_state_dict(seed=11, **cfg)
    gen = _gen(cfg)
    cond = torch.from_numpy(np.random.default_rng(5).uniform(0.0, 1.0, (5, 7)).astype(np.float32))
    with torch.no_grad():
        ref_lat = G.encode_latent(state, cond)
        ref = G.decode_latent(state, ref_lat)
    lat = gen.encode_latent(cond).cpu()
    torch.testing.assert_close(lat, ref_lat, atol=1e-4, rtol=1e-4)
    out = gen(cond).cpu()
    assert out.shape == ref.shape == (5, 1, cfg["out_res"], cfg["out_res"], cfg["out_res"])
    err = (out - ref).abs()
    assert float(err.max()) < 1e-2 and float(err.mean()) < 2e-3, (float(err.max()), float(err.mean()))
    # decode of a latent mixture (the worker's latent_conditions / latent_etas path)
    eta = torch.tensor([[0.25], [0.75]])
    mix = gen.decode_latent((gen.encode_latent(cond[:2]).cpu() * eta).sum(0, keepdim=True)).cpu()
    with torch.no_grad():
        mref = G.decode_latent(state, (ref_lat[:2] * eta).sum(0, keepdim=True))
    assert float((mix - mref).abs().max()) < 1e-2


def test_generator_chunking_is_invariant(lib):
    gen = _gen(CONFIGS["small"])
    cond = torch.from_numpy(np.random.default_rng(7).uniform(0.0, 1.0, (6, 7)).astype(np.float32))
    a = gen(cond).cpu()
    gen.max_cells = 4
    b = gen(cond).cpu()
    torch.testing.assert_close(a, b, atol=0, rtol=0)


def test_conv_zero_padding_matches_torch(lib):
    from maple_b200 import _lib
    rng = np.random.default_rng(3)
    B, n, ci, co = 2, 8, 32, 16
    x = torch.tensor(rng.standard_normal((B, ci, n, n, n)), dtype=torch.float32).to(torch.bfloat16).float()
    w = torch.tensor(rng.standard_normal((co, ci, 3, 3, 3)) * 0.1, dtype=torch.float32).to(torch.bfloat16).float()
    b = torch.tensor(rng.standard_normal(co), dtype=torch.float32)
    ref = F.conv3d(x.double(), w.double(), b.double(), padding=1).float()
    xin = x.permute(0, 2, 3, 4, 1).reshape(B, n ** 3, ci).to(torch.bfloat16).contiguous().to(DEV)
    wt = w.permute(2, 3, 4, 1, 0).reshape(27, ci, co).to(torch.bfloat16).contiguous().to(DEV)
    bd = b.to(DEV)
    out = torch.empty((B, n ** 3, co), dtype=torch.float32, device=DEV)
    _lib.nn_call("maple_nn_conv3d_padded", _p(xin), _p(wt), _p(bd), None, None, _p(out), B, n, ci, co, 3, 0,
                 _lib.NN_PAD_ZEROS, _s())
    got = out.cpu().reshape(B, n, n, n, co).permute(0, 4, 1, 2, 3)
    torch.testing.assert_close(got, ref, atol=1e-4, rtol=1e-4)
    with pytest.raises(_lib.MapleError):
        _lib.nn_call("maple_nn_conv3d_padded", _p(xin), _p(wt), _p(bd), None, None, _p(out), B, n, ci, co, 3, 0, 7,
                     _s())


def test_generator_elementwise_kernels(lib):
    from maple_b200 import _lib
    rng = np.random.default_rng(4)
    g = _lib.gen_call
    d = lambda t: t.contiguous().to(DEV)  # noqa: E731  (device copies are kept alive by the names below)
    # linear (+ SiLU) and layernorm (+ SiLU)
    x = torch.tensor(rng.standard_normal((13, 37)), dtype=torch.float32)
    W = torch.tensor(rng.standard_normal((70, 37)) * 0.2, dtype=torch.float32)
    bb = torch.tensor(rng.standard_normal(70), dtype=torch.float32)
    xd, Wd, bd = d(x), d(W), d(bb)
    y = torch.empty((13, 70), device=DEV)
    g("maple_gen_linear", _p(xd), _p(Wd), _p(bd), _p(y), 13, 37, 70, 1, _s())
    torch.testing.assert_close(y.cpu(), F.silu(F.linear(x, W, bb)), atol=1e-5, rtol=1e-5)
    gam, bet = torch.rand(70) + 0.5, torch.randn(70)
    gd, betd = d(gam), d(bet)
    z = torch.empty_like(y)
    g("maple_gen_layernorm", _p(y), _p(gd), _p(betd), _p(z), 13, 70, 1e-5, 0, _s())
    torch.testing.assert_close(z.cpu(), F.layer_norm(y.cpu(), (70,), gam, bet), atol=1e-5, rtol=1e-5)
    # trilinear x2 from a channels-first source into channels-last BF16
    B, C, n = 2, 24, 5
    v = torch.tensor(rng.standard_normal((B, C, n, n, n)), dtype=torch.float32)
    vd = d(v)
    up = torch.empty((B, (2 * n) ** 3, C), dtype=torch.bfloat16, device=DEV)
    g("maple_gen_upsample2", _p(vd), C * n ** 3, 1, n ** 3, _p(up), B, n, C, _s())
    ref = F.interpolate(v, scale_factor=2, mode="trilinear", align_corners=False)
    ref = ref.permute(0, 2, 3, 4, 1).reshape(B, -1, C)
    torch.testing.assert_close(up.float().cpu(), ref.to(torch.bfloat16).float(), atol=2e-2, rtol=8e-3)
    # group norm + SiLU on channels-last FP32, both outputs
    C, N, Gs = 32, 216, 8
    h = torch.tensor(rng.standard_normal((B, N, C)) * 3 + 1, dtype=torch.float32)
    gam, bet = torch.rand(C) + 0.5, torch.randn(C)
    hd, gd, betd = d(h), d(gam), d(bet)
    ob = torch.empty((B, N, C), dtype=torch.bfloat16, device=DEV)
    of = torch.empty((B, N, C), dtype=torch.float32, device=DEV)
    st = torch.empty(B * Gs * 2, dtype=torch.float64, device=DEV)
    g("maple_gen_groupnorm", _p(hd), _p(gd), _p(betd), Gs, 1e-5, 1, _p(ob), _p(of), _p(st), B, N, C, _s())
    ref = F.silu(F.group_norm(h.permute(0, 2, 1), Gs, gam, bet)).permute(0, 2, 1)
    torch.testing.assert_close(of.cpu(), ref, atol=1e-5, rtol=1e-5)
    torch.testing.assert_close(ob.float().cpu(), ref.to(torch.bfloat16).float(), atol=1e-6, rtol=8e-3)
    # 1x1 head + sigmoid
    hw = torch.randn(C)
    hwd = d(hw)
    out = torch.empty((B, N), device=DEV)
    g("maple_gen_head_sigmoid", _p(hd), _p(hwd), 0.3, _p(out), B, N, C, _s())
    torch.testing.assert_close(out.cpu(), torch.sigmoid(h @ hw + 0.3), atol=1e-5, rtol=1e-5)
    with pytest.raises(_lib.MapleError):
        g("maple_gen_groupnorm", _p(hd), None, None, 5, 1e-5, 1, _p(ob), None, _p(st), B, N, C, _s())


def test_binomial_smoothing_bit_exact(lib, golden):
    from maple_b200.generator import binomial_smooth_periodic
    gd = golden("generator.npz")
    vol = torch.from_numpy(gd["warm_in"]).to(DEV)
    for passes in (0, 1, 3):
        got = binomial_smooth_periodic(vol, passes).cpu().numpy()
        np.testing.assert_array_equal(got, gd[f"smooth_{passes}"])
    vb = np.random.default_rng(8).uniform(-0.2, 1.2, (3, 16, 16, 16)).astype(np.float32)
    got = binomial_smooth_periodic(torch.from_numpy(vb).to(DEV), 2).cpu().numpy()
    for b in range(3):
        np.testing.assert_array_equal(got[b], G.binomial_smooth_periodic(vb[b], 2))


def test_match_mean_clamped(lib, golden):
    from maple_b200.generator import match_mean_clamped
    gd = golden("generator.npz")
    vol = torch.from_numpy(gd["warm_in"]).to(DEV)
    for i in range(4):
        t, iters = gd[f"match_{i}_args"]
        got = match_mean_clamped(vol, float(t), 1e-5, int(iters)).cpu().numpy()
        np.testing.assert_allclose(got, gd[f"match_{i}"], rtol=0, atol=1e-6)
    vb = np.random.default_rng(2).uniform(0.0, 1.0, (4, 8, 8, 8)).astype(np.float32)
    tg = [0.1, 0.3, 0.6, 0.02]
    got = match_mean_clamped(torch.from_numpy(vb).to(DEV), tg, 1e-5, 8).cpu().numpy()
    for b in range(4):
        np.testing.assert_allclose(got[b], G.match_mean_clamped(vb[b], tg[b], 1e-5, 8), rtol=0, atol=1e-6)


def test_load_generator_checkpoint(lib, tmp_path):
    from maple_b200.generator import load_generator
    cfg = CONFIGS["full"]
    state = G.synthetic_state_dict(seed=3, **cfg)
    path = os.path.join(tmp_path, "g.pt")
    torch.save({"model": state, "args": dict(cfg)}, path)
    gen = load_generator(path, DEV)
    cond = torch.rand(2, 7)
    with torch.no_grad():
        ref = G.generate(state, cond)
    assert float((gen(cond).cpu() - ref).abs().max()) < 1e-2
    bad = dict(state)
    bad["noise_encoder.fc.weight"] = torch.zeros(1)
    torch.save({"model": bad, "args": dict(cfg)}, path)
    with pytest.raises(ValueError):
        load_generator(path, DEV)
    small = CONFIGS["small"]
    torch.save({"model": G.synthetic_state_dict(seed=3, **small), "args": dict(small)}, path)
    with pytest.raises(ValueError):
        load_generator(path, DEV)
    missing = dict(state)
    missing.pop("out.bias")
    with pytest.raises(RuntimeError):
        _gen(cfg).load_state_dict(missing)
