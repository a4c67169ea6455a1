"""Learned initial guess: the BF16 tensor-core network kernels against the
torch FP32 CPU oracle, the field conversions, the warm-start entry point and
what a trained network gains over the zero initial guess."""
import ctypes as C

import numpy as np
import pytest
import torch

from oracle import convnet_oracle as ora

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _s():
    return C.c_void_p(torch.cuda.current_stream(DEV).cuda_stream)


def _bf(a):
    """BF16-representable FP32 CPU tensor and its BF16 device copy."""
    t = torch.as_tensor(a, dtype=torch.float32).to(torch.bfloat16)
    return t.float(), t.to(DEV).contiguous()


def _rel(a, b):
    a, b = torch.as_tensor(a).double().cpu(), torch.as_tensor(b).double().cpu()
    return float((a - b).norm() / b.norm().clamp_min(1e-300))


@pytest.mark.parametrize("n,cin,cout,k,relu,B", [(8, 8, 32, 3, 1, 2), (4, 96, 128, 3, 0, 3), (8, 21, 32, 3, 0, 1),
                                                  (16, 32, 21, 1, 0, 2), (2, 128, 64, 3, 1, 2), (8, 64, 96, 1, 1, 1)])
def test_conv3d_forward_matches_torch(lib, n, cin, cout, k, relu, B):
    from maple_b200 import _lib
    g = torch.Generator().manual_seed(n * 1000 + cin + cout)
    taps = 27 if k == 3 else 1
    N = n ** 3
    x, xd = _bf(torch.randn(B, N, cin, generator=g))
    W, Wd = _bf(torch.randn(taps, cin, cout, generator=g) / np.sqrt(taps * cin))
    bias = torch.randn(cout, generator=g)
    res, resd = _bf(torch.randn(B, N, cout, generator=g))
    out = torch.empty(B, N, cout, dtype=torch.bfloat16, device=DEV)
    out32 = torch.empty(B, N, cout, dtype=torch.float32, device=DEV)
    _lib.nn_call("maple_nn_conv3d", _p(xd), _p(Wd), _p(bias.to(DEV)), _p(resd), _p(out), _p(out32), B, n, cin, cout,
                 k, relu, _s())
    ref = ora._to_nvc(ora.conv3d_periodic(ora._to_ncdhw(x, n), W, bias)) + res
    if relu:
        ref = torch.relu(ref)
    torch.cuda.synchronize()
    assert (out32.cpu() - ref).abs().max() < 2e-4 * max(1.0, float(ref.abs().max()))
    assert (out.float().cpu() - ref).abs().max() <= 2 ** -7 * float(ref.abs().max())


@pytest.mark.parametrize("n,cin,cout,k,B", [(8, 8, 32, 3, 2), (4, 96, 128, 3, 3), (8, 32, 21, 1, 2),
                                             (4, 21, 32, 3, 2), (16, 64, 64, 3, 1)])
def test_conv3d_gradients_match_autograd(lib, n, cin, cout, k, B):
    """Weight, bias and data gradients (the data gradient is the forward
    kernel with flipped, transposed weights)."""
    from maple_b200 import _lib
    g = torch.Generator().manual_seed(7 * n + cin)
    taps = 27 if k == 3 else 1
    N = n ** 3
    x, xd = _bf(torch.randn(B, N, cin, generator=g))
    W, Wd = _bf(torch.randn(taps, cin, cout, generator=g) / np.sqrt(taps * cin))
    dz, dzd = _bf(torch.randn(B, N, cout, generator=g))
    xr = x.clone().requires_grad_(True)
    Wr = W.clone().requires_grad_(True)
    br = torch.zeros(cout, requires_grad=True)
    y = ora._to_nvc(ora.conv3d_periodic(ora._to_ncdhw(xr, n), Wr, br))
    (y * dz).sum().backward()
    dW = torch.zeros(taps, cin, cout, device=DEV)
    db = torch.zeros(cout, device=DEV)
    _lib.nn_call("maple_nn_conv3d_wgrad", _p(xd), _p(dzd), _p(dW), _p(db), B, n, cin, cout, k, _s())
    Wt = torch.empty(taps, cout, cin, dtype=torch.bfloat16, device=DEV)
    _lib.nn_call("maple_nn_flip_weights", _p(Wd), _p(Wt), cin, cout, k, _s())
    gx = torch.empty(B, N, cin, dtype=torch.float32, device=DEV)
    _lib.nn_call("maple_nn_conv3d", _p(dzd), _p(Wt), None, None, None, _p(gx), B, n, cout, cin, k, 0, _s())
    torch.cuda.synchronize()
    assert _rel(dW, Wr.grad) < 1e-5
    assert _rel(db, br.grad) < 1e-5
    assert _rel(gx, xr.grad) < 1e-5


def test_resampling_and_adjoints(lib):
    from maple_b200 import _lib
    g = torch.Generator().manual_seed(3)
    B, nc, Cc = 2, 4, 16
    f, fd = _bf(torch.randn(B, (2 * nc) ** 3, Cc, generator=g))
    c, cd = _bf(torch.randn(B, nc ** 3, Cc, generator=g))
    base, based = _bf(torch.randn(B, (2 * nc) ** 3, Cc, generator=g))
    out_c = torch.empty(B, nc ** 3, Cc, dtype=torch.bfloat16, device=DEV)
    out_f = torch.empty(B, (2 * nc) ** 3, Cc, dtype=torch.bfloat16, device=DEV)
    tol = 2 ** -7
    up = lambda t: ora._to_nvc(torch.nn.functional.interpolate(ora._to_ncdhw(t, nc), scale_factor=2, mode="nearest"))
    pool = lambda t: ora._to_nvc(torch.nn.functional.avg_pool3d(ora._to_ncdhw(t, 2 * nc), 2))
    _lib.nn_call("maple_nn_resample", _lib.NN_POOL, _p(fd), None, _p(out_c), B, nc, Cc, 0, _s())
    ref = pool(f)
    torch.cuda.synchronize()
    assert (out_c.float().cpu() - ref).abs().max() <= tol * ref.abs().max()
    _lib.nn_call("maple_nn_resample", _lib.NN_UPSAMPLE, _p(cd), _p(based), _p(out_f), B, nc, Cc, 0, _s())
    ref = up(c) + base
    torch.cuda.synchronize()
    assert (out_f.float().cpu() - ref).abs().max() <= tol * ref.abs().max()
    # adjoints: pooling^T = upsampling / 8, upsampling^T = 8 x pooling
    _lib.nn_call("maple_nn_resample", _lib.NN_POOL_ADJ, _p(cd), None, _p(out_f), B, nc, Cc, 0, _s())
    ref = up(c) / 8
    torch.cuda.synchronize()
    assert (out_f.float().cpu() - ref).abs().max() <= tol * ref.abs().max()
    _lib.nn_call("maple_nn_resample", _lib.NN_UPSAMPLE_ADJ, _p(fd), None, _p(out_c), B, nc, Cc, 0, _s())
    ref = pool(f) * 8
    torch.cuda.synchronize()
    assert (out_c.float().cpu() - ref).abs().max() <= tol * ref.abs().max()
    before = out_c.float().cpu()
    _lib.nn_call("maple_nn_resample", _lib.NN_UPSAMPLE_ADJ, _p(fd), None, _p(out_c), B, nc, Cc, 1, _s())
    torch.cuda.synchronize()
    assert (out_c.float().cpu() - 2 * before).abs().max() <= 2 * tol * before.abs().max()
    acc = torch.zeros_like(out_c)
    _lib.nn_call("maple_nn_accumulate", _p(acc), _p(out_c), out_c.numel(), 0, _s())
    _lib.nn_call("maple_nn_accumulate", _p(acc), _p(out_c), out_c.numel(), 1, _s())
    torch.cuda.synchronize()
    assert (acc.float() - 2 * out_c.float()).abs().max() <= tol * out_c.float().abs().max()


def test_mse_and_adam_match_torch(lib):
    from maple_b200 import _lib
    g = torch.Generator().manual_seed(5)
    n = 1000
    pred = torch.randn(n, generator=g)
    tgt, tgtd = _bf(torch.randn(n, generator=g))
    loss = torch.zeros(1, device=DEV)
    grad = torch.empty(n, dtype=torch.bfloat16, device=DEV)
    _lib.nn_call("maple_nn_mse", _p(pred.to(DEV)), _p(tgtd), _p(grad), _p(loss), n, 4.0, _s())
    torch.cuda.synchronize()
    assert abs(float(loss) - float((pred - tgt).pow(2).mean())) < 1e-5
    want = 4.0 * 2 * (pred - tgt) / n
    assert (grad.float().cpu() - want).abs().max() <= 2 ** -8 * float(want.abs().max())
    # Adam: three steps against torch.optim.Adam
    w0 = torch.randn(n, generator=g)
    grads = [torch.randn(n, generator=g) for _ in range(3)]
    wt = w0.clone().requires_grad_(True)
    opt = torch.optim.Adam([wt], lr=1e-2, betas=(0.9, 0.999), eps=1e-8)
    w, m, v = w0.to(DEV), torch.zeros(n, device=DEV), torch.zeros(n, device=DEV)
    wb = torch.empty(n, dtype=torch.bfloat16, device=DEV)
    for k, gr in enumerate(grads):
        wt.grad = gr.clone()
        opt.step()
        gs = (gr * 64.0).to(DEV)
        _lib.nn_call("maple_nn_adam", _p(w), _p(gs), _p(m), _p(v), _p(wb), n, 1e-2, 0.9, 0.999, 1e-8, 0.0, 64.0, k + 1,
                     _s())
    torch.cuda.synchronize()
    assert (w.cpu() - wt.detach()).abs().max() < 1e-5
    assert (wb.float().cpu() - w.cpu()).abs().max() <= 2 ** -8 * float(w.abs().max())


def test_network_forward_and_gradients_match_cpu_oracle(lib):
    """Whole network: output and every layer's weight / bias gradient of an
    MSE loss against torch CPU autograd on the same (BF16-valued) weights."""
    from maple_b200.learned import OUT, WarmStartNet, design_densities
    r, B = 16, 2
    net = WarmStartNet(r, device=DEV, seed=3)
    g = torch.Generator().manual_seed(9)
    for L in net.layers:  # nonzero biases exercise the bias path and its gradient
        net.w32[L.b_off:L.b_off + L.cout] = (0.05 * torch.randn(L.cout, generator=g)).to(DEV)
    net._refresh()
    rho = torch.tensor(design_densities(B, r, 123), device=DEV)
    target, targetd = _bf(torch.randn(B, r ** 3, OUT, generator=g))
    params = {}
    for L in net.layers:
        W, b = net.layer_weights(L.name)
        params[L.name] = (W.to(torch.bfloat16).float().cpu(), b.cpu())
    x = ora.features(rho.cpu()).to(torch.bfloat16).float()
    loss_ref, out_ref, grads_ref = ora.mse_and_grads(params, x, target, r, net.widths, round_bf16=True)
    net.grad.zero_()
    out = net.forward(net.features(rho))
    gout = net.mse(out, targetd, gscale=1.0)
    net.backward(gout)
    torch.cuda.synchronize()
    assert _rel(out, out_ref) < 1e-2
    assert abs(float(net.loss) - loss_ref) < 1e-2 * loss_ref
    for L in net.layers:
        gW, gb = net.layer_grads(L.name)
        rW, rb = grads_ref[L.name]
        if L.name == "enc0a":
            gW, rW = gW[:, :2], rW[:, :2]
        assert _rel(gW, rW) < 3e-2, L.name
        assert _rel(gb, rb) < 3e-2, L.name


def test_feature_and_field_conversions(lib):
    from maple_b200 import _lib
    g = torch.Generator().manual_seed(1)
    B, n, F, Cn = 2, 8, 18, 21
    N = n ** 3
    rho = torch.rand(B, N, generator=g, dtype=torch.float64)
    feat = torch.empty(B, N, 8, dtype=torch.bfloat16, device=DEV)
    _lib.nn_call("maple_nn_features", _p(rho.to(DEV)), _p(feat), B, N, 8, _s())
    ref = ora.features(rho)
    torch.cuda.synchronize()
    assert (feat.float().cpu() - ref).abs().max() <= 2 ** -8
    u = torch.randn(B, F, N, generator=g, dtype=torch.float64) + 3.0
    scale = torch.linspace(0.5, 2.0, F, dtype=torch.float64)
    ch = torch.zeros(B, N, Cn, dtype=torch.bfloat16, device=DEV)
    mw = torch.empty(B * F, dtype=torch.float64, device=DEV)
    _lib.nn_call("maple_nn_fields_to_channels", _p(u.to(DEV)), _p(mw), _p(ch), B, N, F, Cn, 0, _p(scale.to(DEV)),
                 _s())
    want = ((u - u.mean(2, keepdim=True)) * scale[None, :, None]).permute(0, 2, 1)
    torch.cuda.synchronize()
    assert (ch[..., :F].float().cpu().double() - want).abs().max() <= 2 ** -7 * want.abs().max()
    back = torch.empty(B, F, N, dtype=torch.float64, device=DEV)
    inv = (1.0 / scale).to(DEV)
    chf = ch.float().contiguous()
    _lib.nn_call("maple_nn_channels_to_fields", _p(chf), _p(back), B, N, F, Cn, 0, _p(inv), _s())
    torch.cuda.synchronize()
    assert (back.cpu() - (u - u.mean(2, keepdim=True))).abs().max() <= 2 ** -7 * u.abs().max()
    # trilinear prolongation (factor 4) and density restriction against numpy
    nc, s = 4, 4
    uc = torch.randn(3, nc ** 3, generator=g, dtype=torch.float64)
    uf = torch.empty(3, (nc * s) ** 3, dtype=torch.float64, device=DEV)
    _lib.nn_call("maple_nn_prolong_fields", _p(uc.to(DEV)), _p(uf), 3, nc, s, _s())
    a = uc.numpy().reshape(3, nc, nc, nc)
    t = np.arange(nc * s) / s
    i0 = np.floor(t).astype(int)
    fr = t - i0
    i1 = (i0 + 1) % nc
    want = np.zeros((3, nc * s, nc * s, nc * s))
    for wx, ix in ((1 - fr, i0), (fr, i1)):
        for wy, iy in ((1 - fr, i0), (fr, i1)):
            for wz, iz in ((1 - fr, i0), (fr, i1)):
                w3 = wx[:, None, None] * wy[None, :, None] * wz[None, None, :]
                want += w3[None] * a[:, ix][:, :, iy][:, :, :, iz]
    torch.cuda.synchronize()
    assert np.abs(uf.cpu().numpy().reshape(want.shape) - want).max() < 1e-12
    rf = torch.rand(2, (nc * s) ** 3, generator=g, dtype=torch.float64)
    rc = torch.empty(2, nc ** 3, dtype=torch.float64, device=DEV)
    _lib.nn_call("maple_nn_restrict_density", _p(rf.to(DEV)), _p(rc), 2, nc, s, _s())
    want = rf.numpy().reshape(2, nc, s, nc, s, nc, s).mean(axis=(2, 4, 6)).reshape(2, -1)
    torch.cuda.synchronize()
    assert np.abs(rc.cpu().numpy() - want).max() < 1e-14


def test_warm_start_from_given_solution(lib):
    """maple_set_solution: a converged field as initial iterate needs (almost)
    no iterations; a rebuilt hierarchy keeps the previous solution as the
    warm start but refuses to homogenize it."""
    from maple_b200.core import HomogenizationContext
    from maple_b200.learned import design_densities
    r, B = 16, 2
    rho = torch.tensor(design_densities(B, r, 77), device=DEV)
    ctx = HomogenizationContext(r, ncells=B, device=DEV)
    ctx.set_density("elastic", rho, "fp64")
    cold = ctx.solve("elastic", "fp64", rtol=1e-10, warm=False)
    u = ctx.solution("elastic")
    H1 = ctx.homogenize("elastic").cpu().numpy()
    ctx.set_density("elastic", rho, "fp64")
    with pytest.raises(Exception):
        ctx.homogenize("elastic")  # the solution belongs to the previous density build
    ctx.set_solution("elastic", torch.zeros_like(u))
    ctx.set_solution("elastic", u)
    hot = ctx.solve("elastic", "fp64", rtol=1e-10, warm=True)
    assert hot.iters.max() <= 1 < cold.iters.min()
    H2 = ctx.homogenize("elastic").cpu().numpy()
    assert np.abs(H1 - H2).max() < 1e-9 * np.abs(H1).max()
    ctx.close()


def test_trained_network_reduces_pcg_iterations(lib):
    """Train the network on solves generated by the library (16^3 cells,
    seeds 100,000+) and compare PCG iterations on held-out cells (seeds
    200,000+) from its guess and from the zero guess."""
    from maple_b200.learned import WarmStartNet, design_densities, evaluate, generate_solves, train
    r = 16
    data = generate_solves(192, r, seed0=100_000, batch=96, precision="mixed", rtol=1e-8, device=DEV)
    net = WarmStartNet(r, device=DEV, seed=0)
    hist = train(net, data, steps=300, batch=16, lr=2e-3, log_every=50)
    assert hist[-1][1] < 0.5 * hist[0][1], hist
    held = torch.tensor(design_densities(32, r, 200_000), device=DEV)
    rep = evaluate(net, held, precision="mixed", rtol=1e-8)
    s = rep.summary()
    assert rep.iters_learned.sum() < 0.9 * rep.iters_zero.sum(), s
    assert (rep.iters_learned[:, 0] <= rep.iters_zero[:, 0]).mean() > 0.8, s
