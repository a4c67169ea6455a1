"""CPU checks of the network oracle and of the host-side layer plan (no GPU)."""
import numpy as np
import torch

from oracle import convnet_oracle as ora


def test_periodic_conv_tap_convention():
    """conv3d_periodic computes out[v] = sum_tap in[v + off(tap)] @ W[tap]
    with tap = 9(dx+1) + 3(dy+1) + (dz+1) and periodic wrap-around."""
    rng = np.random.default_rng(0)
    n, cin, cout = 4, 3, 2
    x = rng.standard_normal((1, n ** 3, cin))
    W = rng.standard_normal((27, cin, cout))
    want = np.zeros((n, n, n, cout))
    xv = x.reshape(n, n, n, cin)
    for tap in range(27):
        dx, dy, dz = tap // 9 - 1, (tap // 3) % 3 - 1, tap % 3 - 1
        shifted = np.roll(xv, shift=(-dx, -dy, -dz), axis=(0, 1, 2))  # shifted[v] = x[v + d]
        want += shifted @ W[tap]
    got = ora._to_nvc(ora.conv3d_periodic(ora._to_ncdhw(torch.tensor(x), n), torch.tensor(W)))
    assert np.abs(got.numpy().reshape(n, n, n, cout) - want).max() < 1e-12


def test_layer_plan_and_oracle_forward():
    from maple_b200.learned import OUT, WIDTHS, unet_layers
    layers = unet_layers(WIDTHS)
    n_params = sum(L.wsize + L.cout for L in layers)
    assert 2.0e6 < n_params < 2.4e6
    g = torch.Generator().manual_seed(0)
    params = {L.name: (torch.randn(L.taps, L.cin, L.cout, generator=g) / np.sqrt(L.fan_in),
                       torch.zeros(L.cout)) for L in layers}
    r = 16
    rho = torch.rand(2, r ** 3, generator=g, dtype=torch.float64)
    out = ora.unet_forward(params, ora.features(rho), r, WIDTHS)
    assert out.shape == (2, r ** 3, OUT) and torch.isfinite(out).all()
    # translation by a multiple of 2^(levels-1) commutes with the network
    shift = 8
    rho_s = torch.roll(rho.reshape(2, r, r, r), shifts=shift, dims=1).reshape(2, -1)
    out_s = ora.unet_forward(params, ora.features(rho_s), r, WIDTHS)
    want = torch.roll(out.reshape(2, r, r, r, OUT), shifts=shift, dims=1).reshape(2, -1, OUT)
    assert (out_s - want).abs().max() < 1e-4 * out.abs().max()


def test_forward_flops_of_a_32_cube():
    from maple_b200.learned import WIDTHS, layer_level, unet_layers
    r = 32
    total = sum(2 * (r >> layer_level(L.name, len(WIDTHS))) ** 3 * L.taps * L.cin * L.cout
                for L in unet_layers(WIDTHS))
    assert 5e9 < total < 2e10  # about 10 GFLOP per 32^3 cell
