"""The allocation-free OC update entry point.

Some host applications manage all device memory themselves and cannot let a
library call cudaMalloc; maple_oc_update_noalloc serves them by keeping its
scratch in a fixed device array inside the library.  This file checks, through
the C ABI, that it returns what the context-based maple_oc_update returns, on
two calls in a row (the array keeps the previous call's contents), and that it
rejects batches larger than its array.  It is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
DEV = torch.device("cuda:0")


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _inputs(rng, B, N):
    x = np.clip(0.25 + 0.2 * rng.standard_normal((B, N)), 1e-3, 1.0)
    dJ = np.abs(rng.standard_normal((B, N))) * 1e-2
    dJ[:, :3] = -1.0  # clamped to 1e-12 by the update
    vf = np.linspace(0.2, 0.3, B)
    return [torch.tensor(a, dtype=torch.float64, device=DEV).contiguous() for a in (x, dJ, vf)]


@pytest.mark.parametrize("r,B", [(8, 3), (64, 1)])
def test_noalloc_oc_update_matches_context_path(lib, r, B):
    from maple_b200 import _lib
    from maple_b200.core import HomogenizationContext
    N = r ** 3
    x, dJ, vf = _inputs(np.random.default_rng(11 + r), B, N)
    ctx = HomogenizationContext(r, ncells=B, device=DEV)
    ref, ref_stats = ctx.oc_update(x, dJ, vf, move=0.2, xmin=1e-3)
    torch.cuda.synchronize()
    ref, ref_stats = ref.cpu().numpy(), ref_stats.cpu().numpy()
    stream = C.c_void_p(torch.cuda.current_stream(DEV).cuda_stream)
    for call in range(2):
        out = torch.full_like(x, -1.0)
        stats = torch.full((B, 2), -1.0, dtype=torch.float64, device=DEV) if call == 0 else None
        _lib.check(lib.maple_oc_update_noalloc(N, B, _p(x), _p(dJ), _p(vf), 0.2, 1e-3, _p(out), _p(stats), stream))
        torch.cuda.synchronize()
        assert np.abs(out.cpu().numpy() - ref).max() < 1e-10, call
        if stats is not None:
            assert np.abs(stats.cpu().numpy() - ref_stats).max() < 1e-12
    ctx.close()


def test_noalloc_rejects_batches_beyond_its_array(lib):
    N = 512
    x = torch.zeros((1, N), dtype=torch.float64, device=DEV)
    rc = lib.maple_oc_update_noalloc(N, 100000, _p(x), _p(x), _p(x), 0.2, 1e-3, _p(torch.empty_like(x)), None,
                                     C.c_void_p(torch.cuda.current_stream(DEV).cuda_stream))
    assert rc != 0
    assert "scratch" in lib.maple_last_error_string().decode()


def _ctx_reference(r, B, x, dJ, vf):
    from maple_b200.core import HomogenizationContext
    ctx = HomogenizationContext(r, ncells=B, device=DEV)
    ref, ref_stats = ctx.oc_update(x, dJ, vf, move=0.2, xmin=1e-3)
    torch.cuda.synchronize()
    out = ref.cpu().numpy(), ref_stats.cpu().numpy()
    ctx.close()
    return out


def test_noalloc_cell_limits_and_multi_launch(lib):
    """The documented limits, exactly: 8191 cells per call with a statistics
    buffer, 5460 without.  At 8^3 so many cells need several cooperative
    launches per call (each reuses the array's partial sums and clears the
    barrier words again); every cell must still match maple_oc_update."""
    r = 8
    N = r ** 3
    B = 8191
    x, dJ, vf = _inputs(np.random.default_rng(5), B, N)
    ref, ref_stats = _ctx_reference(r, B, x, dJ, vf)
    stream = C.c_void_p(torch.cuda.current_stream(DEV).cuda_stream)
    out = torch.full_like(x, -1.0)
    stats = torch.full((B, 2), -1.0, dtype=torch.float64, device=DEV)
    assert lib.maple_oc_update_noalloc(N, B, _p(x), _p(dJ), _p(vf), 0.2, 1e-3, _p(out), _p(stats), stream) == 0
    torch.cuda.synchronize()
    assert np.abs(out.cpu().numpy() - ref).max() < 1e-10
    assert np.abs(stats.cpu().numpy() - ref_stats).max() < 1e-12
    big = torch.zeros((B + 1, N), dtype=torch.float64, device=DEV)
    rc = lib.maple_oc_update_noalloc(N, B + 1, _p(big), _p(big), _p(big[:, 0].contiguous()), 0.2, 1e-3,
                                     _p(torch.empty_like(big)), _p(torch.empty((B + 1, 2), dtype=torch.float64,
                                                                             device=DEV)), stream)
    assert rc != 0 and "8191 cells" in lib.maple_last_error_string().decode()
    # without a statistics buffer the array also holds the statistics
    Bn = 5460
    out = torch.full_like(x[:Bn], -1.0)
    assert lib.maple_oc_update_noalloc(N, Bn, _p(x), _p(dJ), _p(vf), 0.2, 1e-3, _p(out), None, stream) == 0
    torch.cuda.synchronize()
    assert np.abs(out.cpu().numpy() - ref[:Bn]).max() < 1e-10
    rc = lib.maple_oc_update_noalloc(N, Bn + 1, _p(x), _p(dJ), _p(vf), 0.2, 1e-3, _p(torch.empty_like(x)), None,
                                     stream)
    assert rc != 0 and "5460 cells" in lib.maple_last_error_string().decode()


def test_noalloc_reports_a_barrier_wait_that_runs_out(lib):
    """With a phantom block that never arrives (maple_test_wait_limit) the
    bounded barrier waits run out: the call returns MAPLE_E_TIMEOUT and the
    next normal call gives the normal result."""
    from maple_b200 import _lib
    r, B = 8, 3
    N = r ** 3
    x, dJ, vf = _inputs(np.random.default_rng(21), B, N)
    ref, _ = _ctx_reference(r, B, x, dJ, vf)
    stream = C.c_void_p(torch.cuda.current_stream(DEV).cuda_stream)
    out = torch.full_like(x, -1.0)
    _lib.check(lib.maple_test_wait_limit(1 << 12, 1))
    try:
        rc = lib.maple_oc_update_noalloc(N, B, _p(x), _p(dJ), _p(vf), 0.2, 1e-3, _p(out), None, stream)
    finally:
        _lib.check(lib.maple_test_wait_limit(0, 0))
    assert rc == _lib.MAPLE_E_TIMEOUT
    assert "grid barrier" in lib.maple_last_error_string().decode()
    assert lib.maple_oc_update_noalloc(N, B, _p(x), _p(dJ), _p(vf), 0.2, 1e-3, _p(out), None, stream) == 0
    torch.cuda.synchronize()
    assert np.abs(out.cpu().numpy() - ref).max() < 1e-10
