"""Stage-II conditional density generator, inference on this library's kernels.

Drop-in for ``Stage2DensityGenerator`` (core/stage2/density_generator.py:
123-197) as the Pareto dataset worker uses it (condition-only, ``eval()``,
``no_grad``), and for the worker's ``load_generator`` (pareto/
densify_pareto_property_network_32.py:995-1015): same constructor arguments,
same parameter names in ``load_state_dict``, same ``encode_latent`` /
``decode_latent`` / call signature, same output (B, 1, r, r, r) in [0, 1].

Compute path: the condition MLP, fc, upsampling, GroupNorm + SiLU and the
sigmoid head run on the FP32 kernels of ``csrc/generator.cu``; the 3x3x3
convolutions on the BF16 tensor-core implicit GEMM of ``csrc/convnet.cu``
(zero padding, FP32 accumulation).  Activations are channels-last
[cell][voxel][channel].  Results agree with the FP32 module to BF16 accuracy
(the parity test bounds the density error at 1e-2 absolute).
"""
from __future__ import annotations

from typing import Mapping, Optional

import numpy as np
import torch

from . import _lib

EPS = 1e-5  # nn.LayerNorm / nn.GroupNorm default


def _p(t: Optional[torch.Tensor]):
    return None if t is None else t.data_ptr()


def _stream(device):
    return torch.cuda.current_stream(device).cuda_stream


def _groups(channels: int) -> int:
    g = min(8, channels)
    while channels % g != 0:
        g -= 1
    return g


class Stage2DensityGenerator:
    """Condition-only Stage-II generator (inference)."""

    def __init__(self, cond_dim: int = 7, out_res: int = 32, base_res: int = 4, latent_dim: int = 256,
                 base_channels: int = 128, use_noise_encoder: bool = False, device=None, hidden_dim: int = 256,
                 max_cells: int = 64):
        if out_res % base_res != 0:
            raise ValueError(f"out_res must be divisible by base_res, got {out_res} and {base_res}")
        levels = int(round(np.log2(out_res // base_res)))
        if base_res * (2 ** levels) != out_res:
            raise ValueError(f"out_res/base_res must be a power of two, got {out_res}/{base_res}")
        if use_noise_encoder:
            raise ValueError("only the condition-only generator is supported (use_noise_encoder=False), "
                             "as in the Pareto worker")
        self.cond_dim, self.out_res, self.base_res = int(cond_dim), int(out_res), int(base_res)
        self.latent_dim, self.base_channels, self.hidden_dim = int(latent_dim), int(base_channels), int(hidden_dim)
        self.use_noise_encoder = False
        self.levels = levels
        self.max_cells = int(max_cells)
        chans, c = [], self.base_channels
        for _ in range(levels):
            o = max(16, c // 2)
            chans.append((c, o))
            c = o
        self.channels = chans
        self.out_channels = c
        dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        if dev.type == "cuda" and dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        if dev.type != "cuda":
            raise ValueError("the generator runs on a CUDA device")
        self.device = dev
        self._lib = _lib.load()
        self._w = None

    # ------------------------------------------------------------------ weights
    def parameter_shapes(self):
        s, e, H = {}, "condition_encoder.net.", self.hidden_dim
        s[e + "0.weight"], s[e + "0.bias"] = (H, self.cond_dim), (H,)
        s[e + "1.weight"], s[e + "1.bias"] = (H,), (H,)
        s[e + "3.weight"], s[e + "3.bias"] = (H, H), (H,)
        s[e + "4.weight"], s[e + "4.bias"] = (H,), (H,)
        s[e + "6.weight"], s[e + "6.bias"] = (self.latent_dim, H), (self.latent_dim,)
        nfc = self.base_channels * self.base_res ** 3
        s["fc.0.weight"], s["fc.0.bias"] = (nfc, self.latent_dim), (nfc,)
        for i, (ci, co) in enumerate(self.channels):
            p = f"decoder.{2 * i + 1}.net."
            s[p + "0.weight"], s[p + "0.bias"] = (co, ci, 3, 3, 3), (co,)
            s[p + "1.weight"], s[p + "1.bias"] = (co,), (co,)
            s[p + "3.weight"], s[p + "3.bias"] = (co, co, 3, 3, 3), (co,)
            s[p + "4.weight"], s[p + "4.bias"] = (co,), (co,)
        s["out.weight"], s["out.bias"] = (1, self.out_channels, 1, 1, 1), (1,)
        return s

    def load_state_dict(self, state: Mapping, strict: bool = True):
        """Reference parameter names and shapes; convolution weights are
        re-laid out to [tap][cin][cout] BF16 (tap = 9 dx + 3 dy + dz over the
        3x3x3 offsets), everything else stays FP32."""
        shapes = self.parameter_shapes()
        missing = [k for k in shapes if k not in state]
        unexpected = [k for k in state if k not in shapes]
        if strict and (missing or unexpected):
            raise RuntimeError(f"Error(s) in loading state_dict: missing keys {missing}, unexpected keys {unexpected}")
        dev = self.device
        w = {}
        for k, shp in shapes.items():
            t = torch.as_tensor(np.asarray(state[k].detach().cpu() if torch.is_tensor(state[k]) else state[k]),
                                dtype=torch.float32)
            if tuple(t.shape) != tuple(shp):
                raise RuntimeError(f"size mismatch for {k}: got {tuple(t.shape)}, expected {tuple(shp)}")
            if t.dim() == 5 and k != "out.weight":
                co, ci = t.shape[:2]
                t = t.permute(2, 3, 4, 1, 0).reshape(27, ci, co).to(torch.bfloat16)
            elif k == "out.weight":
                t = t.reshape(-1)
            w[k] = t.contiguous().to(dev)
        w["out.bias"] = float(w["out.bias"].item())
        self._w = w
        return self

    def eval(self):
        return self

    def to(self, device):
        if torch.device(device) != self.device:
            raise ValueError("the generator stays on the device it was built for")
        return self

    def _need(self):
        if self._w is None:
            raise RuntimeError("generator weights not loaded (load_state_dict)")
        return self._w

    # ------------------------------------------------------------------ forward
    def encode_latent(self, condition: torch.Tensor, rho_init: Optional[torch.Tensor] = None) -> torch.Tensor:
        """(B, cond_dim) -> (B, latent_dim): Linear, LayerNorm, SiLU, Linear, LayerNorm, SiLU, Linear."""
        if rho_init is not None:
            raise ValueError("condition-only generator: rho_init must be None")
        w = self._need()
        x = torch.as_tensor(condition, dtype=torch.float32).to(self.device).reshape(-1, self.cond_dim).contiguous()
        B, H, e, s = x.shape[0], self.hidden_dim, "condition_encoder.net.", _stream(self.device)
        h1 = torch.empty((B, H), dtype=torch.float32, device=self.device)
        h2 = torch.empty_like(h1)
        lat = torch.empty((B, self.latent_dim), dtype=torch.float32, device=self.device)
        g = _lib.gen_call
        with torch.cuda.device(self.device):
            g("maple_gen_linear", _p(x), _p(w[e + "0.weight"]), _p(w[e + "0.bias"]), _p(h1), B, self.cond_dim, H, 0, s)
            g("maple_gen_layernorm", _p(h1), _p(w[e + "1.weight"]), _p(w[e + "1.bias"]), _p(h2), B, H, EPS, 1, s)
            g("maple_gen_linear", _p(h2), _p(w[e + "3.weight"]), _p(w[e + "3.bias"]), _p(h1), B, H, H, 0, s)
            g("maple_gen_layernorm", _p(h1), _p(w[e + "4.weight"]), _p(w[e + "4.bias"]), _p(h2), B, H, EPS, 1, s)
            g("maple_gen_linear", _p(h2), _p(w[e + "6.weight"]), _p(w[e + "6.bias"]), _p(lat), B, H, self.latent_dim,
              0, s)
        return lat

    def decode_latent(self, latent: torch.Tensor) -> torch.Tensor:
        """(B, latent_dim) -> (B, 1, out_res, out_res, out_res) densities in [0, 1]."""
        self._need()
        z = torch.as_tensor(latent, dtype=torch.float32).to(self.device).reshape(-1, self.latent_dim).contiguous()
        B, r = z.shape[0], self.out_res
        out = torch.empty((B, r ** 3), dtype=torch.float32, device=self.device)
        for b0 in range(0, B, self.max_cells):
            b1 = min(B, b0 + self.max_cells)
            self._decode_chunk(z[b0:b1], out[b0:b1])
        return out.reshape(B, 1, r, r, r)

    def _decode_chunk(self, z: torch.Tensor, out: torch.Tensor):
        w, dev, s, g = self._w, self.device, _stream(self.device), _lib.gen_call
        B, C, n = z.shape[0], self.base_channels, self.base_res
        nfc = C * n ** 3
        x = torch.empty((B, nfc), dtype=torch.float32, device=dev)
        stats = torch.empty((B * 8 * 2,), dtype=torch.float64, device=dev)
        with torch.cuda.device(dev):
            g("maple_gen_linear", _p(z), _p(w["fc.0.weight"]), _p(w["fc.0.bias"]), _p(x), B, self.latent_dim, nfc, 1,
              s)
            src, strides = x, (nfc, 1, n ** 3)  # (B, C, n, n, n): channels-first
            for i, (ci, co) in enumerate(self.channels):
                p, m = f"decoder.{2 * i + 1}.net.", 2 * n
                M = m ** 3
                up = torch.empty((B, M, ci), dtype=torch.bfloat16, device=dev)
                g("maple_gen_upsample2", _p(src), strides[0], strides[1], strides[2], _p(up), B, n, ci, s)
                y = torch.empty((B, M, co), dtype=torch.float32, device=dev)
                h = torch.empty((B, M, co), dtype=torch.bfloat16, device=dev)
                o = torch.empty((B, M, co), dtype=torch.float32, device=dev)
                G = _groups(co)
                _lib.nn_call("maple_nn_conv3d_padded", _p(up), _p(w[p + "0.weight"]), _p(w[p + "0.bias"]), None, None,
                             _p(y), B, m, ci, co, 3, 0, _lib.NN_PAD_ZEROS, s)
                g("maple_gen_groupnorm", _p(y), _p(w[p + "1.weight"]), _p(w[p + "1.bias"]), G, EPS, 1, _p(h), None,
                  _p(stats), B, M, co, s)
                _lib.nn_call("maple_nn_conv3d_padded", _p(h), _p(w[p + "3.weight"]), _p(w[p + "3.bias"]), None, None,
                             _p(y), B, m, co, co, 3, 0, _lib.NN_PAD_ZEROS, s)
                g("maple_gen_groupnorm", _p(y), _p(w[p + "4.weight"]), _p(w[p + "4.bias"]), G, EPS, 1, None, _p(o),
                  _p(stats), B, M, co, s)
                src, strides, n = o, (M * co, co, 1), m
                del up, y, h
            if self.levels == 0:  # the seed volume itself feeds the head: bring it to channels-last
                src = src.reshape(B, C, n ** 3).transpose(1, 2).contiguous()
            g("maple_gen_head_sigmoid", _p(src), _p(w["out.weight"]), float(w["out.bias"]), _p(out), B, n ** 3,
              self.out_channels, s)

    def forward(self, condition: torch.Tensor, rho_init: Optional[torch.Tensor] = None) -> torch.Tensor:
        return self.decode_latent(self.encode_latent(condition, rho_init))

    __call__ = forward

    def flops_per_cell(self) -> float:
        """Multiply-adds x 2 of one cell's convolutions (the dominant work)."""
        f, n = 0.0, self.base_res
        for ci, co in self.channels:
            n *= 2
            f += 2.0 * n ** 3 * 27 * (ci * co + co * co)
        return f


def load_generator(checkpoint: str, device) -> Stage2DensityGenerator:
    """pareto/densify_pareto_property_network_32.py:995-1015: a checkpoint
    {"model": state_dict, "args": {...}} of a condition-only 32^3 generator."""
    ckpt = torch.load(checkpoint, map_location="cpu")
    state = ckpt["model"]
    if any(key.startswith("noise_encoder.") for key in state):
        raise ValueError("This script requires a condition-only checkpoint. Retrain without --use_rho_init.")
    a = dict(ckpt.get("args", {}))
    model = Stage2DensityGenerator(cond_dim=int(a.get("cond_dim", 7)), out_res=int(a.get("out_res", 32)),
                                   base_res=int(a.get("base_res", 4)), latent_dim=int(a.get("latent_dim", 256)),
                                   base_channels=int(a.get("base_channels", 128)), use_noise_encoder=False,
                                   device=device)
    if int(model.out_res) != 32:
        raise ValueError(f"This script requires a 32-resolution generator, got out_res={model.out_res}")
    model.load_state_dict(state)
    return model.eval()


def binomial_smooth_periodic(vol: torch.Tensor, passes: int) -> torch.Tensor:
    """binomial_smooth_periodic_torch (pareto/densify_pareto_property_network_32.py:
    1040-1052) of (n, n, n) or (B, n, n, n) volumes on the GPU, bit-identical
    to the reference's FP32 result."""
    v = torch.as_tensor(vol).float()
    if v.device.type != "cuda":
        raise ValueError("binomial_smooth_periodic runs on a CUDA tensor")
    shp = v.shape
    n = shp[-1]
    if v.dim() not in (3, 4) or shp[-3:] != (n, n, n):
        raise ValueError("expected (n, n, n) or (B, n, n, n) volumes")
    src = v.reshape(-1, n ** 3).contiguous()
    B = src.shape[0]
    out = torch.empty_like(src)
    work = torch.empty_like(src) if int(passes) > 0 else None
    if src.data_ptr() == out.data_ptr():
        src = src.clone()
    with torch.cuda.device(v.device):
        _lib.gen_call("maple_gen_binomial_smooth", _p(src), _p(out), _p(work), B, n, int(max(0, passes)),
                      _stream(v.device))
    return out.reshape(shp)


def match_mean_clamped(vol: torch.Tensor, target_mean, rho_min: float, iters: int) -> torch.Tensor:
    """match_mean_clamped_torch (same file, 1031-1037) of one volume or a batch
    (leading dim B with one target per volume) on the GPU."""
    v = torch.as_tensor(vol).float()
    if v.device.type != "cuda":
        raise ValueError("match_mean_clamped runs on a CUDA tensor")
    tgt = np.atleast_1d(np.asarray(target_mean, dtype=np.float64))
    B = tgt.size
    out = v.reshape(B, -1).clone().contiguous()
    t = torch.as_tensor(tgt, dtype=torch.float64, device=v.device)
    with torch.cuda.device(v.device):
        _lib.gen_call("maple_gen_match_mean", _p(out), _p(t), B, out.shape[1], float(rho_min), 1.0, int(iters),
                      _stream(v.device))
    return out.reshape(v.shape)


def gen_launch_count() -> int:
    return int(_lib.load().maple_gen_launch_count())


__all__ = ["Stage2DensityGenerator", "load_generator", "binomial_smooth_periodic", "match_mean_clamped",
           "gen_launch_count", "EPS"]
