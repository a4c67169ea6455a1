"""The generator / warm-start oracle against fixtures made by the reference's
own Stage2DensityGenerator and Pareto worker helpers (CPU only)."""
import os

import numpy as np
import pytest
import torch

from oracle import generator_oracle as G

GOLD = np.load(os.path.join(os.path.dirname(__file__), "golden", "generator.npz"))
CONFIGS = {
    "full": dict(cond_dim=7, out_res=32, base_res=4, latent_dim=256, base_channels=128),
    "small": dict(cond_dim=7, out_res=16, base_res=4, latent_dim=64, base_channels=32),
}


@pytest.mark.parametrize("tag", sorted(CONFIGS))
def test_generator_oracle_matches_reference(tag):
    cfg = CONFIGS[tag]
    state = G.synthetic_state_dict(seed=11, **cfg)
    assert G.config_from_state(state) == dict(cfg, hidden_dim=256)
    cond = torch.from_numpy(GOLD[f"{tag}_cond"])
    with torch.no_grad():
        lat = G.encode_latent(state, cond)
        rho = G.decode_latent(state, lat).numpy().reshape(3, -1)
        eta = torch.from_numpy(GOLD[f"{tag}_eta"]).reshape(-1, 1)
        mix = G.decode_latent(state, (lat[:2] * eta).sum(0, keepdim=True)).numpy().reshape(1, -1)
    np.testing.assert_allclose(lat.numpy(), GOLD[f"{tag}_latent"], rtol=0, atol=2e-6)
    for name, a in (("rho", rho), ("mix", mix)):
        np.testing.assert_allclose(a[:, ::7], GOLD[f"{tag}_{name}_sub"], rtol=0, atol=2e-6)
        np.testing.assert_allclose(a.astype(np.float64).sum(1), GOLD[f"{tag}_{name}_sum"], rtol=1e-6)
        np.testing.assert_allclose((a.astype(np.float64) ** 2).sum(1), GOLD[f"{tag}_{name}_sumsq"], rtol=1e-6)


def test_param_shapes_cover_the_reference_state_dict():
    names = list(G.param_shapes(**CONFIGS["full"]))
    assert names[0] == "condition_encoder.net.0.weight" and names[-1] == "out.bias"
    assert "decoder.5.net.4.bias" in names and "decoder.7.net.0.weight" not in names
    assert G.decoder_channels(128, 3) == [(128, 64), (64, 32), (32, 16)]
    assert [G.group_count(c) for c in (64, 32, 16, 12, 6)] == [8, 8, 8, 6, 6]
    with pytest.raises(ValueError):
        G.upsample_levels(24, 5)


@pytest.mark.parametrize("passes", [0, 1, 3])
def test_binomial_smoothing_bit_exact(passes):
    got = G.binomial_smooth_periodic(GOLD["warm_in"], passes)
    assert got.dtype == np.float32
    np.testing.assert_array_equal(got, GOLD[f"smooth_{passes}"])


@pytest.mark.parametrize("i", range(4))
def test_match_mean_clamped(i):
    t, iters = GOLD[f"match_{i}_args"]
    got = G.match_mean_clamped(GOLD["warm_in"], float(t), 1e-5, int(iters))
    np.testing.assert_allclose(got, GOLD[f"match_{i}"], rtol=0, atol=1e-6)
