"""Timing of single operators on the GPU (CUDA events, L2 flushed between
repetitions), for profiling and for the comparisons recorded with the
design:

    python -m maple_b200.opbench conv --cells 16 --res 32 --cin 128 --cout 128
    python -m maple_b200.opbench wgrad --cells 16 --res 32 --cin 128 --cout 128
    python -m maple_b200.opbench ebe --res 64

``conv``: the periodic 3x3x3 BF16 convolution of the learned guess
(maple_nn_conv3d) on B cells of n^3 voxels; prints TFLOP/s (2 * voxels * 27 *
cin * cout flops per launch).

``wgrad``: its weight gradient (maple_nn_conv3d_wgrad), same flop count.

``ebe``: the fine-level elastic operator (6 load cases) of one seeded cell in
the element-batched tensor-core form (maple_matvec_ebe_tc: gather, tcgen05
GEMM, scatter) beside the stencil form the solver uses (maple_matvec, FP64),
with the relative difference of the two results.
"""
from __future__ import annotations

import argparse
import ctypes as C

import numpy as np
import torch

from . import _lib


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _time_us(fn, device, reps=10):
    flush = torch.empty(64 << 20, dtype=torch.float32, device=device)  # 256 MB > L2
    fn()
    torch.cuda.synchronize(device)
    ts = []
    for _ in range(reps):
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize(device)
        ts.append(e0.elapsed_time(e1) * 1000.0)
    return float(np.median(ts))


def conv(args):
    dev = torch.device("cuda", 0)
    lib = _lib.load()
    B, n, cin, cout = args.cells, args.res, args.cin, args.cout
    N = n ** 3
    g = torch.Generator(device=dev).manual_seed(0)
    x = torch.randn(B, N, cin, device=dev, generator=g).to(torch.bfloat16)
    W = (torch.randn(27, cin, cout, device=dev, generator=g) / np.sqrt(27 * cin)).to(torch.bfloat16)
    out = torch.empty(B, N, cout, dtype=torch.bfloat16, device=dev)
    s = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    us = _time_us(lambda: _lib.nn_call("maple_nn_conv3d", _p(x), _p(W), None, None, _p(out), None, B, n, cin, cout,
                                       3, 0, s), dev, args.reps)
    flag = C.c_int(-1)
    _lib.nn_call("maple_nn_wait_status", C.byref(flag), s)
    flops = 2.0 * B * N * 27 * cin * cout
    print(f"conv3d 3x3x3 B={B} n={n} cin={cin} cout={cout}: {us:.1f} us, {flops / us / 1e6:.1f} TFLOP/s, "
          f"waits timed out: {flag.value}")
    del lib


def wgrad(args):
    dev = torch.device("cuda", 0)
    B, n, cin, cout = args.cells, args.res, args.cin, args.cout
    N = n ** 3
    g = torch.Generator(device=dev).manual_seed(0)
    x = torch.randn(B, N, cin, device=dev, generator=g).to(torch.bfloat16)
    dz = torch.randn(B, N, cout, device=dev, generator=g).to(torch.bfloat16)
    dW = torch.zeros(27, cin, cout, dtype=torch.float32, device=dev)
    s = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    us = _time_us(lambda: _lib.nn_call("maple_nn_conv3d_wgrad", _p(x), _p(dz), _p(dW), None, B, n, cin, cout, 3, s),
                  dev, args.reps)
    flag = C.c_int(-1)
    _lib.nn_call("maple_nn_wait_status", C.byref(flag), s)
    flops = 2.0 * B * N * 27 * cin * cout
    print(f"conv3d weight gradient 3x3x3 B={B} n={n} cin={cin} cout={cout}: {us:.1f} us, "
          f"{flops / us / 1e6:.1f} TFLOP/s, waits timed out: {flag.value}")


def ebe(args):
    from .core import HomogenizationContext
    from .batch import seeded_design
    dev = torch.device("cuda", 0)
    lib = _lib.load()
    r = args.res
    N = r ** 3
    x = seeded_design(0, r, r / 16.0, 0.25).reshape(1, -1)
    rho = torch.tensor(1e-9 + (1 - 1e-9) * np.clip(x, 1e-3, 1.0) ** 3, device=dev)
    c = HomogenizationContext(r, ncells=1, device=dev)
    c.set_density("elastic", rho, "mixed")
    u = torch.randn(1, 6, 3, N, dtype=torch.float64, device=dev, generator=torch.Generator(device=dev).manual_seed(1))
    u32 = u.float().contiguous()
    y32 = torch.empty_like(u32)
    rows = torch.empty(N * 6 * 24, dtype=torch.float32, device=dev)
    outw = torch.empty_like(rows)
    s = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    t_ebe = _time_us(lambda: _lib.check(lib.maple_matvec_ebe_tc(c._h, _p(u32), _p(y32), _p(rows), _p(outw), s)),
                     dev, args.reps)
    t_st = _time_us(lambda: c.matvec("elastic", rho, u), dev, args.reps)
    y64 = c.matvec("elastic", rho, u)
    err = float((y32.double() - y64).abs().max() / y64.abs().max())
    print(f"{r}^3 elastic operator, 6 load cases: element-batched tcgen05 (gather + TF32 GEMM + scatter) "
          f"{t_ebe:.1f} us; stencil FP64 (maple_matvec) {t_st:.1f} us; max relative difference {err:.2e}")
    c.close()


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    sub = ap.add_subparsers(dest="op", required=True)
    a = sub.add_parser("conv")
    a.add_argument("--cells", type=int, default=16)
    a.add_argument("--res", type=int, default=32)
    a.add_argument("--cin", type=int, default=128)
    a.add_argument("--cout", type=int, default=128)
    a.add_argument("--reps", type=int, default=10)
    w = sub.add_parser("wgrad")
    w.add_argument("--cells", type=int, default=16)
    w.add_argument("--res", type=int, default=32)
    w.add_argument("--cin", type=int, default=128)
    w.add_argument("--cout", type=int, default=128)
    w.add_argument("--reps", type=int, default=10)
    b = sub.add_parser("ebe")
    b.add_argument("--res", type=int, default=64)
    b.add_argument("--reps", type=int, default=10)
    args = ap.parse_args(argv)
    {"conv": conv, "wgrad": wgrad, "ebe": ebe}[args.op](args)


if __name__ == "__main__":
    main()
