"""Learned initial guess for the periodic homogenization solves.

A periodic 3-D U-Net maps a cell's element densities (r^3 voxels) to the 21
fluctuation fields of its solves: 6 elastic load cases x 3 components and 3
thermal load cases.  Its prediction is handed to the MG-PCG as the initial
iterate; the solver still runs to the requested tolerance, so the network only
changes how many iterations that takes (plain MG-PCG is its fallback and what
measures its error).  The reference has the hook for this in
``GMGSolver.solve(init_list=...)`` (utils/EBE_GMG.py:648-757, 851-858), which
its live path never feeds.

Everything that computes runs in ``libmaple_b200.so``: BF16 tensor-core
convolutions with FP32 accumulation (forward, data gradient, weight gradient),
pooling / upsampling and their adjoints, ReLU masks, the MSE loss and Adam on
FP32 master weights.  Training data are generated by the library's own solver.
torch allocates buffers, shuffles indices and computes the data set's
per-field normalisation once.

The training loss is the energy norm of the prediction error relative to the
energy of the solution, per cell and load case: e_r^T K(rho) e_r / u_r^T K u_r,
with K applied by the library's FP64 fine-level operator (maple_matvec).  That
is the quantity that decides how many PCG iterations remain; it ignores what
the solver ignores (a constant field, i.e. the periodic rigid translation, and
errors in near-void regions) and weighs the strain of the error, not its
long-range drift.  The per-field normalisation of the outputs is the RMS of the
solutions weighted by the local stiffness (maple_nn_node_weights).

Network (widths (32, 64, 96, 128), about 2.2M parameters):
  level l < 3: two 3x3x3 conv + ReLU, 2x2x2 average pool to level l+1
  level 3:     two 3x3x3 conv + ReLU
  decoder:     1x1 conv at the coarse level, nearest upsampling, add the
               encoder's output of that level, two 3x3x3 conv + ReLU
  head:        1x1 conv to 21 channels (FP32), scaled per field.
All convolutions use circular padding: the cell is periodic.
"""
from __future__ import annotations

import ctypes as C
import math
import time
from dataclasses import dataclass, field
from typing import Optional

import numpy as np
import torch

from . import _lib
from ._lib import NN_POOL, NN_POOL_ADJ, NN_UPSAMPLE, NN_UPSAMPLE_ADJ
from .core import HomogenizationContext, _ptr, _stream

FEATURES = 8          # input channels: rho^(1/3), rho, six zero channels
USED_FEATURES = 2
OUT_ELASTIC = 18      # 6 load cases x 3 components
OUT_THERMAL = 3
OUT = OUT_ELASTIC + OUT_THERMAL
WIDTHS = (32, 64, 96, 128)


@dataclass
class ConvSpec:
    name: str
    cin: int
    cout: int
    k: int          # 1 or 3
    relu: bool
    fan_in: int
    w_off: int = 0
    b_off: int = 0

    @property
    def taps(self) -> int:
        return 27 if self.k == 3 else 1

    @property
    def wsize(self) -> int:
        return self.taps * self.cin * self.cout


def unet_layers(widths=WIDTHS, cin=FEATURES, cout=OUT):
    """Layer list in forward order (names enc{l}a/b, mid_a/b, up{l}, dec{l}a/b, head)."""
    L = []
    c = cin
    for lv, w in enumerate(widths[:-1]):
        L.append(ConvSpec(f"enc{lv}a", c, w, 3, True, 27 * (USED_FEATURES if lv == 0 else c)))
        L.append(ConvSpec(f"enc{lv}b", w, w, 3, True, 27 * w))
        c = w
    wb = widths[-1]
    L.append(ConvSpec("mid_a", c, wb, 3, True, 27 * c))
    L.append(ConvSpec("mid_b", wb, wb, 3, True, 27 * wb))
    c = wb
    for lv in reversed(range(len(widths) - 1)):
        w = widths[lv]
        L.append(ConvSpec(f"up{lv}", c, w, 1, False, c))
        L.append(ConvSpec(f"dec{lv}a", w, w, 3, True, 27 * w))
        L.append(ConvSpec(f"dec{lv}b", w, w, 3, True, 27 * w))
        c = w
    L.append(ConvSpec("head", c, cout, 1, False, c))
    return L


def layer_level(name: str, levels: int) -> int:
    """Grid level (0 = finest) a layer runs on."""
    if name.startswith(("enc", "dec")):
        return int(name[3])
    if name.startswith("up"):
        return int(name[2]) + 1
    if name.startswith("mid"):
        return levels - 1
    return 0


def _align(n: int, a: int = 64) -> int:
    return (n + a - 1) // a * a


class WarmStartNet:
    """The network, its FP32 master weights, BF16 copies and Adam state."""

    def __init__(self, r: int, widths=WIDTHS, device=None, seed: int = 0):
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.widths = tuple(widths)
        self.levels = len(self.widths)
        if r % (1 << (self.levels - 1)) != 0:
            raise ValueError(f"r={r} must be divisible by {1 << (self.levels - 1)}")
        self.r = int(r)
        self.layers = unet_layers(self.widths)
        self.by_name = {L.name: L for L in self.layers}
        off = 0
        for L in self.layers:
            L.w_off = off
            off += _align(L.wsize)
            L.b_off = off
            off += _align(L.cout)
        self.size = off
        self.n_params = sum(L.wsize + L.cout for L in self.layers)
        dev = self.device
        self.w32 = torch.zeros(off, dtype=torch.float32, device=dev)
        self.wbf = torch.zeros(off, dtype=torch.bfloat16, device=dev)
        self.wflip = torch.zeros(off, dtype=torch.bfloat16, device=dev)
        self.grad = torch.zeros(off, dtype=torch.float32, device=dev)
        self.m = torch.zeros(off, dtype=torch.float32, device=dev)
        self.v = torch.zeros(off, dtype=torch.float32, device=dev)
        self.step = 0
        # per-field scale: network output * scale = fluctuation field
        self.scale = torch.ones(OUT, dtype=torch.float64, device=dev)
        self.loss = torch.zeros(1, dtype=torch.float32, device=dev)  # written by the MSE kernels
        self.last_loss = self.loss
        self._buf = {}
        self._fe = {}  # batch size -> context applying K(rho) for the energy loss
        self._act = {}
        self.init_weights(seed)

    # ------------------------------------------------------------------ weights
    def init_weights(self, seed: int = 0, head_std: float = 0.1):
        """He-normal weights (std sqrt(2/fan_in) before a ReLU, sqrt(1/fan_in)
        otherwise; the head head_std of that), zero biases; deterministic in
        seed."""
        g = torch.Generator().manual_seed(seed)
        w = torch.zeros(self.size, dtype=torch.float32)
        for L in self.layers:
            std = math.sqrt((2.0 if L.relu else 1.0) / L.fan_in) * (head_std if L.name == "head" else 1.0)
            vals = torch.randn(L.taps, L.cin, L.cout, generator=g) * std
            if L.name == "enc0a":
                vals[:, USED_FEATURES:, :] = 0.0
            w[L.w_off:L.w_off + L.wsize] = vals.reshape(-1)
        self.w32.copy_(w.to(self.device))
        self.m.zero_()
        self.v.zero_()
        self.step = 0
        self._refresh()

    def _refresh(self):
        """BF16 copies and flipped (data-gradient) weights from the FP32 masters."""
        s = _stream(self.device)
        _lib.nn_call("maple_nn_to_bf16", _ptr(self.w32), _ptr(self.wbf), self.size, s)
        for L in self.layers:
            _lib.nn_call("maple_nn_flip_weights", self._wp(self.wbf, L), self._wp(self.wflip, L), L.cin, L.cout, L.k,
                         s)

    @staticmethod
    def _wp(flat, L):
        return C.c_void_p(flat.data_ptr() + L.w_off * flat.element_size())

    @staticmethod
    def _bp(flat, L):
        return C.c_void_p(flat.data_ptr() + L.b_off * flat.element_size())

    def state_dict(self) -> dict:
        return {"r": self.r, "widths": list(self.widths), "w32": self.w32.cpu().numpy(),
                "scale": self.scale.cpu().numpy(), "step": self.step}

    def load_state_dict(self, sd: dict):
        if tuple(int(w) for w in sd["widths"]) != self.widths:
            raise ValueError("width mismatch")
        self.w32.copy_(torch.as_tensor(np.asarray(sd["w32"]), dtype=torch.float32).to(self.device))
        self.scale.copy_(torch.as_tensor(np.asarray(sd["scale"]), dtype=torch.float64).to(self.device))
        self.step = int(sd.get("step", 0))
        self._refresh()

    def save(self, path: str):
        np.savez(path, **{k: np.asarray(v) for k, v in self.state_dict().items()})

    @classmethod
    def load(cls, path: str, r: Optional[int] = None, device=None) -> "WarmStartNet":
        """Weights saved by save(); r may differ from the training resolution
        (the network is fully convolutional)."""
        z = np.load(path)
        net = cls(int(r if r is not None else z["r"]), tuple(int(w) for w in z["widths"]), device=device)
        net.load_state_dict({k: z[k] for k in z.files})
        return net

    def layer_weights(self, name: str):
        """(W [taps][cin][cout], b [cout]) FP32 views of one layer's masters."""
        L = self.by_name[name]
        return (self.w32[L.w_off:L.w_off + L.wsize].view(L.taps, L.cin, L.cout), self.w32[L.b_off:L.b_off + L.cout])

    def layer_grads(self, name: str):
        L = self.by_name[name]
        return (self.grad[L.w_off:L.w_off + L.wsize].view(L.taps, L.cin, L.cout), self.grad[L.b_off:L.b_off + L.cout])

    # ------------------------------------------------------------------ buffers
    def _t(self, tag: str, B: int, n: int, Cn: int, dtype=torch.bfloat16):
        key = (tag, B)
        t = self._buf.get(key)
        shape = (B, n ** 3, Cn)
        if t is None or tuple(t.shape) != shape or t.dtype != dtype:
            t = torch.empty(shape, dtype=dtype, device=self.device)
            self._buf[key] = t
        return t

    def free_buffers(self):
        self._buf.clear()
        self._act = {}
        for ctx in self._fe.values():
            ctx.close()
        self._fe.clear()

    def _t64(self, tag: str, shape):
        key = (tag, shape)
        t = self._buf.get(key)
        if t is None:
            t = torch.empty(shape, dtype=torch.float64, device=self.device)
            self._buf[key] = t
        return t

    def _fe_ctx(self, B: int) -> HomogenizationContext:
        ctx = self._fe.get(B)
        if ctx is None:
            ctx = HomogenizationContext(self.r, ncells=B, device=self.device)
            self._fe[B] = ctx
        return ctx

    # ------------------------------------------------------------------ primitives
    def _conv(self, L: ConvSpec, x, out, B, n, out_f32=None):
        _lib.nn_call("maple_nn_conv3d", _ptr(x), self._wp(self.wbf, L), self._bp(self.w32, L), None, _ptr(out),
                     _ptr(out_f32), B, n, L.cin, L.cout, L.k, int(L.relu), _stream(self.device))

    def _conv_back(self, L: ConvSpec, x, gz, gx, B, n):
        """Weight/bias gradients of layer L (input x, pre-activation gradient
        gz) and, if gx is given, the data gradient into gx."""
        s = _stream(self.device)
        _lib.nn_call("maple_nn_conv3d_wgrad", _ptr(x), _ptr(gz), self._wp(self.grad, L), self._bp(self.grad, L), B, n,
                     L.cin, L.cout, L.k, s)
        if gx is not None:
            _lib.nn_call("maple_nn_conv3d", _ptr(gz), self._wp(self.wflip, L), None, None, _ptr(gx), None, B, n,
                         L.cout, L.cin, L.k, 0, s)

    def _relu_mask(self, y, g):
        _lib.nn_call("maple_nn_relu_mask", _ptr(y), _ptr(g), y.numel(), _stream(self.device))

    def _resample(self, op, src, base, dst, B, nc, Cn, add=0):
        _lib.nn_call("maple_nn_resample", op, _ptr(src), _ptr(base), _ptr(dst), B, nc, Cn, int(add),
                     _stream(self.device))

    # ------------------------------------------------------------------ forward / backward
    def features(self, rho: torch.Tensor) -> torch.Tensor:
        """(B, N) float64 densities -> (B, N, 8) BF16 network input."""
        B = rho.shape[0]
        x = self._t("in", B, self.r, FEATURES)
        _lib.nn_call("maple_nn_features", _ptr(rho), _ptr(x), B, self.r ** 3, FEATURES, _stream(self.device))
        return x

    def forward(self, x: torch.Tensor) -> torch.Tensor:
        """x (B, N, 8) BF16 -> (B, N, 21) FP32 normalised fields; keeps the
        activations for backward."""
        B = x.shape[0]
        n = self.r
        self._act = act = {"in": x}
        h = x
        for lv in range(self.levels - 1):
            w = self.widths[lv]
            a = self._t(f"enc{lv}a", B, n, w)
            self._conv(self.by_name[f"enc{lv}a"], h, a, B, n)
            b = self._t(f"enc{lv}b", B, n, w)
            self._conv(self.by_name[f"enc{lv}b"], a, b, B, n)
            act[f"enc{lv}a"], act[f"enc{lv}b"] = a, b
            p = self._t(f"pool{lv + 1}", B, n // 2, w)
            self._resample(NN_POOL, b, None, p, B, n // 2, w)
            act[f"pool{lv + 1}"] = p
            h, n = p, n // 2
        wb = self.widths[-1]
        ma = self._t("mid_a", B, n, wb)
        self._conv(self.by_name["mid_a"], h, ma, B, n)
        mb = self._t("mid_b", B, n, wb)
        self._conv(self.by_name["mid_b"], ma, mb, B, n)
        act["mid_a"], act["mid_b"] = ma, mb
        h = mb
        for lv in reversed(range(self.levels - 1)):
            w = self.widths[lv]
            c = self._t(f"up{lv}", B, n, w)
            self._conv(self.by_name[f"up{lv}"], h, c, B, n)
            n *= 2
            d = self._t(f"skip{lv}", B, n, w)
            self._resample(NN_UPSAMPLE, c, act[f"enc{lv}b"], d, B, n // 2, w)
            a = self._t(f"dec{lv}a", B, n, w)
            self._conv(self.by_name[f"dec{lv}a"], d, a, B, n)
            b = self._t(f"dec{lv}b", B, n, w)
            self._conv(self.by_name[f"dec{lv}b"], a, b, B, n)
            act[f"up{lv}"], act[f"skip{lv}"], act[f"dec{lv}a"], act[f"dec{lv}b"] = c, d, a, b
            h = b
        out = self._t("out", B, n, OUT, torch.float32)
        self._conv(self.by_name["head"], h, None, B, n, out_f32=out)
        return out

    def backward(self, gout: torch.Tensor):
        """Accumulates weight gradients (into self.grad) for the output
        gradient gout (B, N, 21) BF16 of the last forward."""
        act = self._act
        B = gout.shape[0]
        n = self.r
        g = self._t("g_head_in", B, n, self.widths[0])
        self._conv_back(self.by_name["head"], act["dec0b"], gout, g, B, n)
        gskip = {}
        for lv in range(self.levels - 1):
            w = self.widths[lv]
            self._relu_mask(act[f"dec{lv}b"], g)
            ga = self._t(f"g_dec{lv}a", B, n, w)
            self._conv_back(self.by_name[f"dec{lv}b"], act[f"dec{lv}a"], g, ga, B, n)
            self._relu_mask(act[f"dec{lv}a"], ga)
            gd = self._t(f"g_skip{lv}", B, n, w)
            self._conv_back(self.by_name[f"dec{lv}a"], act[f"skip{lv}"], ga, gd, B, n)
            gskip[lv] = gd  # d = up(c) + enc_b: the encoder output receives gd itself
            gc = self._t(f"g_up{lv}", B, n // 2, w)
            self._resample(NN_UPSAMPLE_ADJ, gd, None, gc, B, n // 2, w)
            n //= 2
            cin = self.widths[lv + 1]
            src = act["mid_b"] if lv == self.levels - 2 else act[f"dec{lv + 1}b"]
            g = self._t(f"g_up{lv}_in", B, n, cin)
            self._conv_back(self.by_name[f"up{lv}"], src, gc, g, B, n)
        wb = self.widths[-1]
        self._relu_mask(act["mid_b"], g)
        gma = self._t("g_mid_a", B, n, wb)
        self._conv_back(self.by_name["mid_b"], act["mid_a"], g, gma, B, n)
        self._relu_mask(act["mid_a"], gma)
        gp = self._t(f"g_pool{self.levels - 1}", B, n, self.widths[-2])
        self._conv_back(self.by_name["mid_a"], act[f"pool{self.levels - 1}"], gma, gp, B, n)
        for lv in reversed(range(self.levels - 1)):
            w = self.widths[lv]
            gb = gskip[lv]
            self._resample(NN_POOL_ADJ, gp, None, gb, B, n, w, add=1)
            n *= 2
            self._relu_mask(act[f"enc{lv}b"], gb)
            ga = self._t(f"g_enc{lv}a", B, n, w)
            self._conv_back(self.by_name[f"enc{lv}b"], act[f"enc{lv}a"], gb, ga, B, n)
            self._relu_mask(act[f"enc{lv}a"], ga)
            if lv == 0:
                self._conv_back(self.by_name["enc0a"], act["in"], ga, None, B, n)
            else:
                gp = self._t(f"g_pool{lv}", B, n, self.widths[lv - 1])
                self._conv_back(self.by_name[f"enc{lv}a"], act[f"pool{lv}"], ga, gp, B, n)

    def mse(self, out: torch.Tensor, target: torch.Tensor, gscale: float = 1024.0):
        """Plain mean squared error into self.loss (device scalar) and its BF16
        gradient x gscale."""
        B = out.shape[0]
        gout = self._t("g_out", B, self.r, OUT)
        self.loss.zero_()
        _lib.nn_call("maple_nn_mse", _ptr(out), _ptr(target), _ptr(gout), _ptr(self.loss), out.numel(),
                     float(gscale), _stream(self.device))
        return gout

    def weighted_loss(self, out: torch.Tensor, target: torch.Tensor, w: torch.Tensor, gscale: float = 1024.0,
                      grad: bool = True):
        """Node-weighted, offset-free squared error (see the module docstring)
        into self.loss and, if grad, its BF16 gradient x gscale."""
        B = out.shape[0]
        gout = self._t("g_out", B, self.r, OUT) if grad else None
        ebar = self._t("ebar", B, 1, OUT, torch.float32)
        self.loss.zero_()
        _lib.nn_call("maple_nn_mse_weighted", _ptr(out), _ptr(target), _ptr(w), _ptr(ebar), _ptr(gout),
                     _ptr(self.loss), B, self.r ** 3, OUT, float(gscale), _stream(self.device))
        return gout

    def grad_norm(self, gscale: float = 1.0) -> float:
        """Euclidean norm of the accumulated gradient (divided by gscale)."""
        out = self._t64("sumsq", (1,))
        _lib.nn_call("maple_nn_sumsq", _ptr(self.grad), self.size, _ptr(out), _stream(self.device))
        return math.sqrt(float(out.item())) / gscale

    def adam(self, lr: float, beta1=0.9, beta2=0.999, eps=1e-8, weight_decay=0.0, gscale: float = 1024.0):
        self.step += 1
        _lib.nn_call("maple_nn_adam", _ptr(self.w32), _ptr(self.grad), _ptr(self.m), _ptr(self.v), None, self.size,
                     float(lr), float(beta1), float(beta2), float(eps), float(weight_decay), float(gscale), self.step,
                     _stream(self.device))
        self._refresh()

    def energy_loss(self, out: torch.Tensor, target: torch.Tensor, rho: torch.Tensor, energy: torch.Tensor,
                    gscale: float = 1024.0, grad: bool = True, per_cell: bool = False,
                    floor: Optional[torch.Tensor] = None):
        """Relative energy error of the predicted fields, e = scale * (out -
        target): the mean over cells and the 9 load cases of e_r^T K(rho) e_r
        divided by the solution energy of that cell (per_cell), or by that
        energy plus `floor` (9,) -- default the batch mean of each load case --
        so that every term stays bounded and nearly void cells of tiny energy
        cannot dominate the gradient.  Returns (per-(cell, load case) values
        (B, 9), BF16 gradient x gscale w.r.t. out or None); self.last_loss
        holds the mean."""
        B, N = rho.shape
        if not per_cell:
            energy = energy + (energy.mean(dim=0, keepdim=True) if floor is None else floor.reshape(1, 9))
        s = _stream(self.device)
        ctx = self._fe_ctx(B)
        sc_th = C.c_void_p(self.scale.data_ptr() + OUT_ELASTIC * 8)
        e_el = self._t64("e_el", (B, 6, 3, N))
        e_th = self._t64("e_th", (B, 3, 1, N))
        _lib.nn_call("maple_nn_error_fields", _ptr(out), _ptr(target), _ptr(self.scale), _ptr(e_el), B, N,
                     OUT_ELASTIC, OUT, 0, s)
        _lib.nn_call("maple_nn_error_fields", _ptr(out), _ptr(target), sc_th, _ptr(e_th), B, N, OUT_THERMAL, OUT,
                     OUT_ELASTIC, s)
        y_el = ctx.matvec("elastic", rho, e_el)
        y_th = ctx.matvec("thermal", rho, e_th)
        d = self._t64("edot", (B, 9))
        d_el, d_th = self._t64("edot_el", (B, 6)), self._t64("edot_th", (B, 3))
        _lib.nn_call("maple_nn_block_dot", _ptr(e_el), _ptr(y_el), _ptr(d_el), B * 6, 3 * N, s)
        _lib.nn_call("maple_nn_block_dot", _ptr(e_th), _ptr(y_th), _ptr(d_th), B * 3, N, s)
        E_el, E_th = energy[:, :6].contiguous(), energy[:, 6:].contiguous()
        gout = None
        if grad:
            gout = self._t("g_out", B, self.r, OUT)
            coef = 2.0 * gscale / (9.0 * B)
            _lib.nn_call("maple_nn_energy_grad", _ptr(y_el), _ptr(E_el), _ptr(self.scale), _ptr(gout), B, N, 6, 3,
                         OUT, 0, coef, s)
            _lib.nn_call("maple_nn_energy_grad", _ptr(y_th), _ptr(E_th), sc_th, _ptr(gout), B, N, 3, 1, OUT,
                         OUT_ELASTIC, coef, s)
        torch.cat([d_el / E_el, d_th / E_th], dim=1, out=d)
        self.last_loss = d.mean()
        return d, gout

    def train_step(self, rho: torch.Tensor, target: torch.Tensor, energy: torch.Tensor, lr: float,
                   gscale: float = 1024.0, clip: Optional[float] = None, floor: Optional[torch.Tensor] = None):
        """One Adam step on a batch: rho (B, N) float64, target (B, N, 21) BF16,
        solution energies (B, 9) float64.  The gradient is rescaled to norm
        `clip` when it is larger (None: no clipping)."""
        self.grad.zero_()
        out = self.forward(self.features(rho))
        _, gout = self.energy_loss(out, target, rho, energy, gscale, floor=floor)
        self.backward(gout)
        scale = gscale
        if clip is not None:
            gn = self.grad_norm(gscale)
            if gn > clip:
                scale = gscale * gn / clip
        self.adam(lr, gscale=scale)
        return self.last_loss

    # ------------------------------------------------------------------ inference
    def predict(self, rho: torch.Tensor):
        """Initial iterates for densities rho (B, N): elastic (B, 6, 3, N) and
        thermal (B, 3, 1, N) float64 fields."""
        B, N = rho.shape
        out = self.forward(self.features(rho))
        ue = torch.empty((B, 6, 3, N), dtype=torch.float64, device=self.device)
        ut = torch.empty((B, 3, 1, N), dtype=torch.float64, device=self.device)
        s = _stream(self.device)
        _lib.nn_call("maple_nn_channels_to_fields", _ptr(out), _ptr(ue), B, N, OUT_ELASTIC, OUT, 0, _ptr(self.scale), s)
        _lib.nn_call("maple_nn_channels_to_fields", _ptr(out), _ptr(ut), B, N, OUT_THERMAL, OUT, OUT_ELASTIC,
                     C.c_void_p(self.scale.data_ptr() + OUT_ELASTIC * 8), s)
        return ue, ut

    def predict_prolonged(self, rho: torch.Tensor, r: int):
        """Initial iterates for densities rho (B, r^3) on a finer grid than the
        network's (r = factor * self.r): the densities are block-averaged to
        self.r^3, the network predicts there and its fields are trilinearly
        prolonged to the r^3 nodes (periodic).  Returns elastic (B, 6, 3, r^3)
        and thermal (B, 3, 1, r^3) float64 fields."""
        if r % self.r != 0:
            raise ValueError(f"r={r} is not a multiple of the network resolution {self.r}")
        factor = r // self.r
        B = rho.shape[0]
        s = _stream(self.device)
        if factor == 1:
            return self.predict(rho)
        rc = torch.empty((B, self.r ** 3), dtype=torch.float64, device=self.device)
        _lib.nn_call("maple_nn_restrict_density", _ptr(rho), _ptr(rc), B, self.r, factor, s)
        ue_c, ut_c = self.predict(rc)
        ue = torch.empty((B, 6, 3, r ** 3), dtype=torch.float64, device=self.device)
        ut = torch.empty((B, 3, 1, r ** 3), dtype=torch.float64, device=self.device)
        _lib.nn_call("maple_nn_prolong_fields", _ptr(ue_c), _ptr(ue), B * 18, self.r, factor, s)
        _lib.nn_call("maple_nn_prolong_fields", _ptr(ut_c), _ptr(ut), B * 3, self.r, factor, s)
        return ue, ut

    def flops_per_cell(self) -> float:
        """2 x multiply-adds of one forward pass on one r^3 cell."""
        return float(sum(2.0 * (self.r >> layer_level(L.name, self.levels)) ** 3 * L.taps * L.cin * L.cout
                         for L in self.layers))


# ---------------------------------------------------------------------------
# data generated by the solver
@dataclass
class SolveSet:
    rho: torch.Tensor        # (S, N) float64 element densities
    target: torch.Tensor     # (S, N, 21) BF16 normalised, mean-free fields
    energy: torch.Tensor     # (S, 9) float64 u_r^T K u_r per load case (6 elastic, 3 thermal)
    scale: torch.Tensor      # (21,) float64: field = scale * channel
    iters: np.ndarray        # (S, 2) PCG iterations from the zero guess (elastic, thermal)
    seconds: float = 0.0
    generated: int = 0       # cells solved (before dropping unconverged ones)


def simp(x: np.ndarray, penal: float = 3.0, rho_min: float = 1e-9) -> np.ndarray:
    return rho_min + (1.0 - rho_min) * np.power(x, penal)


def design_densities(n: int, r: int, seed0: int, sigma: Optional[float] = None, penal: float = 3.0,
                     rho_min: float = 1e-9) -> np.ndarray:
    """Densities of n seeded designs in the batched benchmark's style: seed
    seed0 + i, periodic Gaussian smoothing sigma (default r/16 voxels), volume
    fractions U[0.01, 0.40] from default_rng(seed0)."""
    from .batch import config2_inputs
    x, _, _ = config2_inputs(n, r, sigma if sigma is not None else r / 16.0, rng_seed=seed0, seed0=seed0)
    return simp(x, penal, rho_min)


def _field_scale(u: torch.Tensor, w: torch.Tensor) -> torch.Tensor:
    """Per-field weighted RMS over cells and nodes of fields (B, F, N) with
    their weighted means removed; w (B, N) averages to 1 per cell."""
    wd = w.double()[:, None, :]
    d = u - (wd * u).mean(dim=2, keepdim=True)
    return (wd * d.pow(2)).mean(dim=(0, 2)).sqrt().clamp_min(1e-30)


def generate_solves(n: int, r: int, seed0: int = 100_000, batch: int = 256, precision: str = "mixed",
                    rtol: float = 1e-8, maxit: int = 500, sigma: Optional[float] = None, device=None,
                    ctx: Optional[HomogenizationContext] = None, scale: Optional[torch.Tensor] = None,
                    verbose: bool = False, keep_unconverged: bool = False) -> SolveSet:
    """Solve n seeded cells with the library's MG-PCG (zero initial guess) and
    keep their normalised, mean-free fields as training targets; cells whose
    solves did not converge within maxit are dropped unless keep_unconverged."""
    dev = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
    batch = min(batch, n)
    ctx = ctx or HomogenizationContext(r, ncells=batch, device=dev)
    N = r ** 3
    rho_all = torch.empty((n, N), dtype=torch.float64, device=dev)
    target = torch.empty((n, N, OUT), dtype=torch.bfloat16, device=dev)
    energy = torch.empty((n, 9), dtype=torch.float64, device=dev)
    ok = np.ones(n, dtype=bool)
    wb = torch.empty((batch, N), dtype=torch.float32, device=dev)
    iters = np.zeros((n, 2), dtype=np.int64)
    mean_work = torch.empty(batch * OUT_ELASTIC, dtype=torch.float64, device=dev)
    inv = None
    t0 = time.perf_counter()
    for start in range(0, n, batch):
        b = min(batch, n - start)
        rho_np = np.ones((batch, N))
        rho_np[:b] = design_densities(b, r, seed0 + start, sigma)
        rho = torch.as_tensor(rho_np, dtype=torch.float64).to(dev).contiguous()
        ctx.set_active(np.arange(batch) < b)
        fields = []
        for k, phys in enumerate(("elastic", "thermal")):
            ctx.set_density(phys, rho, precision)
            info = ctx.solve(phys, precision, rtol=rtol, maxit=maxit, warm=False)
            iters[start:start + b, k] = info.iters[:b]
            ok[start:start + b] &= (info.status[:b] & _lib.CELL_CONVERGED) != 0
            fields.append(ctx.solution(phys))
        ue, ut = fields
        s = _stream(dev)
        en = torch.empty((batch, 9), dtype=torch.float64, device=dev)
        for u, phys, R, D, c0 in ((ue, "elastic", 6, 3, 0), (ut, "thermal", 3, 1, 6)):
            y = ctx.matvec(phys, rho, u)
            dots = torch.empty((batch, R), dtype=torch.float64, device=dev)
            _lib.nn_call("maple_nn_block_dot", _ptr(u), _ptr(y), _ptr(dots), batch * R, D * N, s)
            en[:, c0:c0 + R] = dots
        energy[start:start + b] = en[:b]
        if inv is None:
            if scale is None:
                _lib.nn_call("maple_nn_node_weights", _ptr(rho), _ptr(wb), batch, r, s)
                scale = torch.cat([_field_scale(ue[:b].reshape(b, OUT_ELASTIC, N), wb[:b]),
                                   _field_scale(ut[:b].reshape(b, OUT_THERMAL, N), wb[:b])])
            inv = (1.0 / scale).contiguous()
        tgt = target[start:start + b]
        _lib.nn_call("maple_nn_fields_to_channels", _ptr(ue), _ptr(mean_work), _ptr(tgt), b, N, OUT_ELASTIC, OUT, 0,
                     _ptr(inv), s)
        _lib.nn_call("maple_nn_fields_to_channels", _ptr(ut), _ptr(mean_work), _ptr(tgt), b, N, OUT_THERMAL, OUT,
                     OUT_ELASTIC, C.c_void_p(inv.data_ptr() + OUT_ELASTIC * 8), s)
        rho_all[start:start + b] = rho[:b]
        if verbose:
            print(f"  solves {start + b}/{n}  {time.perf_counter() - t0:.1f}s", flush=True)
    ctx.set_active(None)
    if keep_unconverged or ok.all():
        return SolveSet(rho_all, target, energy, scale, iters, time.perf_counter() - t0, n)
    # cells whose solve stopped at maxit carry no usable target
    keep = torch.as_tensor(np.nonzero(ok)[0], device=dev)
    out = SolveSet(rho_all.index_select(0, keep), target.index_select(0, keep), energy.index_select(0, keep), scale,
                   iters[ok], time.perf_counter() - t0, n)
    torch.cuda.synchronize(dev)
    return out


def train(net: WarmStartNet, data: SolveSet, steps: int, batch: int = 16, lr: float = 1e-3, lr_min: float = 2e-5,
          warmup: int = 50, seed: int = 0, log_every: int = 0, time_limit: Optional[float] = None,
          clip: Optional[float] = None, val: Optional[SolveSet] = None, val_every: int = 100):
    """Adam with linear warm-up and cosine decay over `steps` mini-batches
    drawn without replacement (reshuffled every epoch).  With a validation
    set, the weights are evaluated every val_every steps and the best ones
    are kept at the end.  Returns the loss history [(step, loss)] read every
    log_every steps and at the end."""
    net.scale.copy_(data.scale)
    floor = data.energy.mean(dim=0).contiguous()  # per load case, fixed for the whole run
    best = (math.inf, None)
    S = data.rho.shape[0]
    batch = min(batch, S)
    g = torch.Generator().manual_seed(seed)
    perm = torch.randperm(S, generator=g)
    pos = 0
    hist = []
    t0 = time.perf_counter()
    for it in range(steps):
        if pos + batch > S:
            perm = torch.randperm(S, generator=g)
            pos = 0
        idx = perm[pos:pos + batch].to(net.device)
        pos += batch
        rho = data.rho.index_select(0, idx)
        tgt = data.target.index_select(0, idx)
        en = data.energy.index_select(0, idx)
        if it < warmup:
            lr_t = lr * (it + 1) / warmup
        else:
            c = (it - warmup) / max(1, steps - warmup)
            lr_t = lr_min + 0.5 * (lr - lr_min) * (1 + math.cos(math.pi * c))
        loss = net.train_step(rho, tgt, en, lr_t, clip=clip, floor=floor)
        last = it == steps - 1 or (time_limit is not None and time.perf_counter() - t0 > time_limit)
        if (log_every and (it + 1) % log_every == 0) or last:
            hist.append((it + 1, float(loss.item())))
        if val is not None and ((it + 1) % val_every == 0 or last):
            v = validation_loss(net, val)
            if v < best[0]:
                best = (v, net.w32.clone())
        if last:
            break
    if best[1] is not None:
        net.w32.copy_(best[1])
        net._refresh()
    return hist


def validation_loss(net: WarmStartNet, data: SolveSet, chunk: int = 32) -> float:
    """Training loss (relative energy error) of the prediction over a solve set."""
    tot, cnt = 0.0, 0
    for i in range(0, data.rho.shape[0], chunk):
        rho = data.rho[i:i + chunk].contiguous()
        out = net.forward(net.features(rho))
        net.energy_loss(out, data.target[i:i + chunk].contiguous(), rho, data.energy[i:i + chunk].contiguous(),
                        grad=False)
        b = rho.shape[0]
        tot += float(net.last_loss.item()) * b
        cnt += b
    return tot / max(cnt, 1)


@dataclass
class WarmStartReport:
    cells: int
    iters_zero: np.ndarray       # (B, 2) elastic, thermal
    iters_learned: np.ndarray    # (B, 2)
    ms_zero: float               # both solves, all cells
    ms_learned: float            # network inference + both solves
    ms_network: float            # network inference alone
    extra: dict = field(default_factory=dict)

    def summary(self) -> dict:
        return {"cells": self.cells,
                "pcg_iters_zero": [float(v) for v in self.iters_zero.mean(0)],
                "pcg_iters_learned": [float(v) for v in self.iters_learned.mean(0)],
                "iters_saved_frac": float(1 - self.iters_learned.sum() / max(1, self.iters_zero.sum())),
                "ms_zero": self.ms_zero, "ms_learned": self.ms_learned, "ms_network": self.ms_network,
                "time_saved_frac": float(1 - self.ms_learned / self.ms_zero), **self.extra}


def evaluate(net: WarmStartNet, rho: torch.Tensor, precision: str = "mixed", rtol: float = 1e-8, maxit: int = 500,
             ctx: Optional[HomogenizationContext] = None, repeats: int = 1) -> WarmStartReport:
    """PCG iterations and device time of the elastic + thermal solves of the
    cells rho (B, N), from the zero guess and from the network's guess (its
    inference included in the time).  The last of `repeats` rounds counts."""
    B, N = rho.shape
    dev = net.device
    ctx = ctx or HomogenizationContext(net.r, ncells=B, device=dev)
    res = {}
    converged = {}
    guess = {}
    for _ in range(max(1, repeats)):
        for mode in ("zero", "learned"):
            its = np.zeros((B, 2), dtype=np.int64)
            for phys in ("elastic", "thermal"):
                ctx.set_density(phys, rho, precision)
            torch.cuda.synchronize(dev)
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record()
            if mode == "learned":
                ue, ut = net.predict(rho)
                ctx.set_solution("elastic", ue)
                ctx.set_solution("thermal", ut)
                guess = {"elastic": ue, "thermal": ut}
            e1.record()
            for k, phys in enumerate(("elastic", "thermal")):
                info = ctx.solve(phys, precision, rtol=rtol, maxit=maxit, warm=(mode == "learned"))
                its[:, k] = info.iters
                if mode == "zero":
                    converged[phys] = ctx.solution(phys)
            e2.record()
            torch.cuda.synchronize(dev)
            res[mode] = (its, e0.elapsed_time(e2), e0.elapsed_time(e1))
    # energy-norm error of the network's guess relative to the converged solution
    rel = []
    s = _stream(dev)
    for phys, R, D in (("elastic", 6, 3), ("thermal", 3, 1)):
        u = converged[phys]
        e = (guess[phys] - u).contiguous()
        dots = torch.empty((2, B * R), dtype=torch.float64, device=dev)
        for k, v in enumerate((e, u)):
            y = ctx.matvec(phys, rho, v)
            _lib.nn_call("maple_nn_block_dot", _ptr(v), _ptr(y), _ptr(dots[k]), B * R, D * N, s)
        rel.append(float((dots[0] / dots[1]).mean()))
    return WarmStartReport(B, res["zero"][0], res["learned"][0], res["zero"][1], res["learned"][1],
                           res["learned"][2], {"guess_energy_error": rel})


def forward_tflops(net: WarmStartNet, rho: torch.Tensor, repeats: int = 10) -> dict:
    """Device time of the network's forward pass on rho (B, N) and the
    achieved BF16 tensor-core rate (2 x multiply-adds / time)."""
    x = net.features(rho)
    for _ in range(2):
        net.forward(x)
    torch.cuda.synchronize(net.device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(repeats):
        net.forward(x)
    e1.record()
    torch.cuda.synchronize(net.device)
    ms = e0.elapsed_time(e1) / repeats
    flops = net.flops_per_cell() * rho.shape[0]
    return {"cells": int(rho.shape[0]), "ms": ms, "tflops": flops / (ms * 1e-3) / 1e12}


def main(argv=None):
    """Learned-guess experiment: solver-generated training set (seeds
    100,000+), training on the GPU, evaluation on held-out cells (seeds
    200,000+) against the zero guess.  Prints one JSON object."""
    import argparse
    import json
    ap = argparse.ArgumentParser(description=main.__doc__)
    ap.add_argument("--res", type=int, default=32)
    ap.add_argument("--samples", type=int, default=20_000)
    ap.add_argument("--heldout", type=int, default=256)
    ap.add_argument("--batch", type=int, default=16)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--train-seconds", type=float, default=None)
    ap.add_argument("--precision", default="mixed")
    ap.add_argument("--rtol", type=float, default=1e-8)
    ap.add_argument("--save", default=None, help="write the trained weights (.npz)")
    ap.add_argument("--load", default=None, help="skip training: use these weights (.npz)")
    ap.add_argument("--fine-res", type=int, default=0,
                    help="then run an OC loop at this resolution with the prolonged guess (e.g. 128)")
    ap.add_argument("--fine-iters", type=int, default=30)
    a = ap.parse_args(argv)
    dev = torch.device("cuda", torch.cuda.current_device())
    t0 = time.perf_counter()
    if a.load:
        net = WarmStartNet.load(a.load, r=a.res, device=dev)
        data = generate_solves(min(a.samples, 256), a.res, seed0=100_000, precision=a.precision, rtol=a.rtol,
                               device=dev, scale=net.scale.clone())
    else:
        data = generate_solves(a.samples, a.res, seed0=100_000, precision=a.precision, rtol=a.rtol, device=dev)
        net = WarmStartNet(a.res, device=dev)
    held = generate_solves(a.heldout, a.res, seed0=200_000, precision=a.precision, rtol=a.rtol, device=dev,
                           scale=data.scale)
    t_gen = time.perf_counter() - t0
    t1 = time.perf_counter()
    hist = [] if a.load else train(net, data, a.steps, batch=a.batch, lr=a.lr, log_every=max(1, a.steps // 20),
                                   time_limit=a.train_seconds)
    torch.cuda.synchronize(dev)
    t_train = time.perf_counter() - t1
    val = validation_loss(net, held)
    ctx = HomogenizationContext(a.res, ncells=held.rho.shape[0], device=dev)
    rep = evaluate(net, held.rho, precision=a.precision, rtol=a.rtol, ctx=ctx, repeats=2)
    speed = forward_tflops(net, held.rho[:min(64, held.rho.shape[0])].contiguous())
    if a.save:
        net.save(a.save)
    if a.fine_res:
        out_fine = fine_oc_comparison(net, a.fine_res, a.fine_iters)
    out = {"res": a.res, "params": net.n_params, "samples": a.samples, "samples_converged": int(data.rho.shape[0]),
           "heldout_converged": int(held.rho.shape[0]), "generation_s": round(t_gen, 1),
           "solve_iters_train_mean": [float(v) for v in data.iters.mean(0)],
           "train_steps": hist[-1][0] if hist else 0,
           "batch": a.batch, "train_s": round(t_train, 1), "loss_history": hist, "heldout_energy_error": val,
           "forward": speed, **rep.summary()}
    if a.fine_res:
        out["fine_oc"] = out_fine
    print(json.dumps(out))
    return out


def fine_oc_comparison(net: WarmStartNet, r: int = 128, iters: int = 30, seed: int = 0, sigma: float = 8.0,
                       volfrac: float = 0.15, weights=(0.7, 0.0, 0.3)) -> dict:
    """One fine cell (seeded design, bi-objective stiffness 0.7 / thermal 0.3
    at vf 0.15) run for `iters` OC iterations in mixed precision twice: from
    the zero initial guess and with the network's guess, evaluated at its own
    resolution and prolonged, for the first iteration (later iterations start
    from the previous iterate's solution in both runs)."""
    from .batch import oc_run, seeded_design
    x0 = seeded_design(seed, r, sigma, volfrac).reshape(1, -1)
    res = {}
    for mode in ("zero", "learned"):
        ctx = HomogenizationContext(r, ncells=1, device=net.device)
        guess = None
        t0 = time.perf_counter()
        if mode == "learned":
            rho0 = torch.as_tensor(simp(x0), dtype=torch.float64).to(net.device)
            guess = net.predict_prolonged(rho0, r)
        out = oc_run(x0, np.asarray([weights]), np.asarray([volfrac]), precision="mixed", rtol=1e-10, maxit=500,
                     dx_tol=0.0, max_iters=iters, ctx=ctx, record=True, guess=guess)
        res[mode] = {"seconds": round(time.perf_counter() - t0, 3), "pcg_iters_total": int(out.pcg_iters.sum()),
                     "pcg_iters_first": int(out.history[0]["pcg"][0]) if out.history else None,
                     "J": float(out.J[0])}
        ctx.close()
    return {"res": r, "iters": iters, **res}


if __name__ == "__main__":
    main()
