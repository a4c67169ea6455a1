"""CPU FP32 oracle of the Stage-II density generator and of the Pareto
worker's warm-start post-processing.

TEST INFRASTRUCTURE ONLY: the parity tests, ``__graft_entry__.smoke()`` and
the fixture script use it as the checker; nothing in the product imports it.

Restates, functionally on torch CPU primitives in FP32:
  * ``Stage2DensityGenerator`` (core/stage2/density_generator.py:123-197) with
    ``ConvBlock3d`` (:65-81) and ``ConditionEncoder`` (:84-99), condition-only
    (``use_noise_encoder=False``, the only form the worker loads,
    pareto/densify_pareto_property_network_32.py:995-1015);
  * ``match_mean_clamped_torch`` (densify_pareto_property_network_32.py:1031-1037);
  * ``binomial_smooth_periodic_torch`` (:1040-1052).

``synthetic_state_dict`` makes seeded weights under the reference's parameter
names, so the reference module, this oracle and the CUDA path can all be
loaded with the same numbers (no trained checkpoint ships with the reference).
"""
from __future__ import annotations

import math
from typing import Dict

import numpy as np
import torch
import torch.nn.functional as F


def decoder_channels(base_channels: int, levels: int):
    """(cin, cout) of each decoder ConvBlock3d (density_generator.py:166-172)."""
    out, c = [], int(base_channels)
    for _ in range(levels):
        o = max(16, c // 2)
        out.append((c, o))
        c = o
    return out


def upsample_levels(out_res: int, base_res: int) -> int:
    if out_res % base_res != 0:
        raise ValueError(f"out_res must be divisible by base_res, got {out_res} and {base_res}")
    lv = int(round(np.log2(out_res // base_res)))
    if base_res * (2 ** lv) != out_res:
        raise ValueError(f"out_res/base_res must be a power of two, got {out_res}/{base_res}")
    return lv


def group_count(channels: int) -> int:
    """GroupNorm groups of ConvBlock3d (density_generator.py:68-70)."""
    g = min(8, channels)
    while channels % g != 0:
        g -= 1
    return g


def param_shapes(cond_dim=7, out_res=32, base_res=4, latent_dim=256, base_channels=128, hidden_dim=256):
    """Parameter name -> shape, in the reference module's state_dict order."""
    s = {}
    enc = "condition_encoder.net."
    s[enc + "0.weight"], s[enc + "0.bias"] = (hidden_dim, cond_dim), (hidden_dim,)
    s[enc + "1.weight"], s[enc + "1.bias"] = (hidden_dim,), (hidden_dim,)
    s[enc + "3.weight"], s[enc + "3.bias"] = (hidden_dim, hidden_dim), (hidden_dim,)
    s[enc + "4.weight"], s[enc + "4.bias"] = (hidden_dim,), (hidden_dim,)
    s[enc + "6.weight"], s[enc + "6.bias"] = (latent_dim, hidden_dim), (latent_dim,)
    nfc = base_channels * base_res ** 3
    s["fc.0.weight"], s["fc.0.bias"] = (nfc, latent_dim), (nfc,)
    for i, (ci, co) in enumerate(decoder_channels(base_channels, upsample_levels(out_res, base_res))):
        p = f"decoder.{2 * i + 1}.net."
        s[p + "0.weight"], s[p + "0.bias"] = (co, ci, 3, 3, 3), (co,)
        s[p + "1.weight"], s[p + "1.bias"] = (co,), (co,)
        s[p + "3.weight"], s[p + "3.bias"] = (co, co, 3, 3, 3), (co,)
        s[p + "4.weight"], s[p + "4.bias"] = (co,), (co,)
    cl = decoder_channels(base_channels, upsample_levels(out_res, base_res))
    c_last = cl[-1][1] if cl else base_channels
    s["out.weight"], s["out.bias"] = (1, c_last, 1, 1, 1), (1,)
    return s


def synthetic_state_dict(seed: int = 0, **cfg) -> Dict[str, torch.Tensor]:
    """Seeded FP32 weights: linear / conv weights and biases U(+-1/sqrt(fan_in))
    (the scale of torch's default initialisation), norm weights 1 + 0.1 N(0,1),
    norm biases 0.1 N(0,1)."""
    rng = np.random.default_rng(seed)
    out = {}
    shapes = param_shapes(**cfg)
    for name, shp in shapes.items():
        is_norm = (".net.1." in name or ".net.4." in name) and "decoder" in name or \
                  name.startswith("condition_encoder.net.1.") or name.startswith("condition_encoder.net.4.")
        if is_norm:
            v = (1.0 if name.endswith("weight") else 0.0) + 0.1 * rng.standard_normal(shp)
        else:
            wname = name[:-len("bias")] + "weight" if name.endswith("bias") else name
            fan_in = int(np.prod(shapes[wname][1:]))
            b = 1.0 / math.sqrt(fan_in)
            v = rng.uniform(-b, b, shp)
        out[name] = torch.tensor(v, dtype=torch.float32)
    return out


def config_from_state(state) -> dict:
    """Constructor arguments implied by a state dict's shapes."""
    hidden, cond_dim = state["condition_encoder.net.0.weight"].shape
    latent = state["condition_encoder.net.6.weight"].shape[0]
    nfc = state["fc.0.weight"].shape[0]
    base_channels = state["decoder.1.net.0.weight"].shape[1] if "decoder.1.net.0.weight" in state else \
        state["out.weight"].shape[1]
    base_res = round((nfc // base_channels) ** (1 / 3))
    levels = sum(1 for k in state if k.startswith("decoder.") and k.endswith("net.0.weight"))
    return dict(cond_dim=int(cond_dim), out_res=int(base_res * 2 ** levels), base_res=int(base_res),
                latent_dim=int(latent), base_channels=int(base_channels), hidden_dim=int(hidden))


def encode_latent(state, condition: torch.Tensor) -> torch.Tensor:
    """ConditionEncoder: Linear, LayerNorm, SiLU, Linear, LayerNorm, SiLU, Linear."""
    e = "condition_encoder.net."
    x = condition.float()
    x = F.linear(x, state[e + "0.weight"], state[e + "0.bias"])
    x = F.silu(F.layer_norm(x, x.shape[-1:], state[e + "1.weight"], state[e + "1.bias"]))
    x = F.linear(x, state[e + "3.weight"], state[e + "3.bias"])
    x = F.silu(F.layer_norm(x, x.shape[-1:], state[e + "4.weight"], state[e + "4.bias"]))
    return F.linear(x, state[e + "6.weight"], state[e + "6.bias"])


def decode_latent(state, latent: torch.Tensor) -> torch.Tensor:
    """fc + SiLU -> (B, C, br, br, br) -> [Upsample x2, ConvBlock3d]* -> 1x1 conv -> sigmoid."""
    cfg = config_from_state(state)
    C, br = cfg["base_channels"], cfg["base_res"]
    x = F.silu(F.linear(latent.float(), state["fc.0.weight"], state["fc.0.bias"]))
    x = x.reshape(latent.shape[0], C, br, br, br)
    for i, (_, co) in enumerate(decoder_channels(C, upsample_levels(cfg["out_res"], br))):
        p = f"decoder.{2 * i + 1}.net."
        x = F.interpolate(x, scale_factor=2, mode="trilinear", align_corners=False)
        g = group_count(co)
        x = F.conv3d(x, state[p + "0.weight"], state[p + "0.bias"], padding=1)
        x = F.silu(F.group_norm(x, g, state[p + "1.weight"], state[p + "1.bias"]))
        x = F.conv3d(x, state[p + "3.weight"], state[p + "3.bias"], padding=1)
        x = F.silu(F.group_norm(x, g, state[p + "4.weight"], state[p + "4.bias"]))
    return torch.sigmoid(F.conv3d(x, state["out.weight"], state["out.bias"]))


def generate(state, condition: torch.Tensor) -> torch.Tensor:
    """(B, 1, r, r, r) densities in [0, 1]."""
    with torch.no_grad():
        return decode_latent(state, encode_latent(state, condition))


def match_mean_clamped(vol: np.ndarray, target_mean: float, rho_min: float, iters: int) -> np.ndarray:
    """FP32 x <- clamp(x - mean(x) + clip(target, rho_min, 1), rho_min, 1),
    max(1, iters) times (the mean summed in FP64)."""
    out = np.asarray(vol, dtype=np.float32).copy()
    t = np.float32(np.clip(target_mean, rho_min, 1.0))
    lo, hi = np.float32(rho_min), np.float32(1.0)
    for _ in range(int(max(1, iters))):
        m = np.float32(out.astype(np.float64).mean())
        out = np.minimum(np.maximum((out - m) + t, lo), hi).astype(np.float32)
    return out


def binomial_smooth_periodic(vol: np.ndarray, passes: int) -> np.ndarray:
    """`passes` times along axes 0, 1, 2: acc = 0; acc += w_k * roll(x, s_k)
    for s = -2..2, w = [1 4 6 4 1] / 16, each product and sum rounded to FP32."""
    out = np.asarray(vol, dtype=np.float32).copy()
    w = [np.float32(v / 16.0) for v in (1.0, 4.0, 6.0, 4.0, 1.0)]
    for _ in range(int(max(0, passes))):
        for axis in range(3):
            acc = np.zeros_like(out)
            for wk, s in zip(w, (-2, -1, 0, 1, 2)):
                acc = (acc + (wk * np.roll(out, s, axis=axis)).astype(np.float32)).astype(np.float32)
            out = acc
    return out
