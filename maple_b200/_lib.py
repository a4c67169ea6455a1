"""ctypes binding of ``libmaple_b200.so`` (the C ABI of include/maple_b200.h).

The library is mandatory: there is no CPU or PyTorch fallback for any compute
entry point.  Loading fails loudly with the reason when the shared object is
missing or does not load.
"""
from __future__ import annotations

import ctypes as C
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG, "libmaple_b200.so")

MAPLE_OK = 0
MAPLE_E_BADARG, MAPLE_E_CUDA, MAPLE_E_NOT_CONVERGED, MAPLE_E_BREAKDOWN, MAPLE_E_TIMEOUT, MAPLE_E_NOMEM = 1, 2, 3, 4, 5, 6
ELASTIC, THERMAL = 0, 1
FP64, MIXED = 0, 1
CELL_CONVERGED, CELL_BREAKDOWN, CELL_MAXIT, CELL_FALLBACK = 1, 2, 4, 8

_P = C.c_void_p
_I = C.c_int
_D = C.c_double
_F = C.c_float
_Z = C.c_size_t
_L = C.c_longlong
_IP = C.POINTER(C.c_int)
_DP = C.POINTER(C.c_double)

# name -> (restype, argtypes); must match include/maple_b200.h
SIGNATURES = {
    "maple_last_error_string": (C.c_char_p, []),
    "maple_version": (_I, []),
    "maple_element_matrices": (_I, [_I, _D, _D, _D, _DP, _DP, _DP, _DP, _DP, _DP]),
    "maple_ctx_create": (_I, [_I, _I, _I, _D, _D, _D, C.POINTER(_P)]),
    "maple_ctx_destroy": (_I, [_P]),
    "maple_ctx_info": (_I, [_P, _IP, _IP, C.POINTER(C.c_size_t)]),
    "maple_set_solver_options": (_I, [_P, _I, _D, _I, _D, _I]),
    "maple_set_graphs": (_I, [_P, _I]),
    "maple_set_mixed_mode": (_I, [_P, _I]),
    "maple_set_extrapolation": (_I, [_P, _D]),
    "maple_set_concurrency": (_I, [_P, _I]),
    "maple_set_stencil_split": (_I, [_P, _I]),
    "maple_set_coarse_degree": (_I, [_P, _I]),
    "maple_set_stencil_nine": (_I, [_P, _I]),
    "maple_set_tail_fused": (_I, [_P, _I]),
    "maple_set_pdl": (_I, [_P, _I]),
    "maple_set_device_loop": (_I, [_P, _I]),
    "maple_set_reliable_options": (_I, [_P, _D, _I]),
    "maple_get_device_loop": (_I, [_P, _P]),
    "maple_set_symmetry": (_I, [_P, _I, _I]),
    "maple_set_penalties": (_I, [_P, _D, _D, _I, _D, _D, _D, _I, _I, _I, _I, _I, _I, _I, _I, _I]),
    "maple_penalties": (_I, [_P, _P, _P, _P, _P, _P, _P]),
    "maple_get_oc_terms": (_I, [_P, _P, _P, _P, _P]),
    "maple_symmetrize": (_I, [_I, _I, _I, _I, _P, _P, _P]),
    "maple_set_active": (_I, [_P, _IP, _P]),
    "maple_set_density": (_I, [_P, _I, _P, _I, _P]),
    "maple_solve": (_I, [_P, _I, _I, _D, _I, _I, _IP, _IP, _P]),
    "maple_solve_rhs": (_I, [_P, _I, _I, _P, _P, _D, _I, _P, _P, _IP, _IP, _P]),
    "maple_get_solution": (_I, [_P, _I, _P, _P]),
    "maple_homogenize": (_I, [_P, _I, _P, _P, _P]),
    "maple_energy_contract": (_I, [_I, _I, _I, _P, _P, _I, _P, _P]),
    "maple_sensitivity": (_I, [_P, _P, _P, _P, _P]),
    "maple_assemble_rhs": (_I, [_P, _I, _P, _P, _P]),
    "maple_matvec": (_I, [_P, _I, _P, _P, _P, _P]),
    "maple_box_filter": (_I, [_I, _I, _I, _P, _P, _P]),
    "maple_get_level_elements": (_I, [_P, _I, _I, _P, _P]),
    "maple_transfer": (_I, [_I, _I, _I, _I, _P, _P, _P]),
    "maple_matvec_ebe_tc": (_I, [_P, _P, _P, _P, _P, _P]),
    "maple_oc_update": (_I, [_P, _P, _P, _P, _D, _D, _P, _P, _P]),
    "maple_oc_update_noalloc": (_I, [_I, _I, _P, _P, _P, _D, _D, _P, _P, _P]),
    "maple_test_wait_limit": (_I, [_L, _I]),
    "maple_launch_count": (C.c_ulonglong, []),
    "maple_profile_enable": (_I, [_P, _I, _I]),
    "maple_profile_read": (_I, [_P, C.c_char_p, _I]),
    "maple_oc_step": (_I, [_P, _P, _P, _P, _D, _D, _D, _D, _I, _I, _D, _I, _I, _P, _P, _P, _P, _P, _P, _IP, _P]),
    "maple_set_solution": (_I, [_P, _I, _P, _P]),
    # learned initial guess: convolution network kernels
    "maple_nn_last_error_string": (C.c_char_p, []),
    "maple_nn_launch_count": (C.c_ulonglong, []),
    "maple_nn_conv3d": (_I, [_P, _P, _P, _P, _P, _P, _I, _I, _I, _I, _I, _I, _P]),
    "maple_nn_conv3d_wgrad": (_I, [_P, _P, _P, _P, _I, _I, _I, _I, _I, _P]),
    "maple_nn_flip_weights": (_I, [_P, _P, _I, _I, _I, _P]),
    "maple_nn_resample": (_I, [_I, _P, _P, _P, _I, _I, _I, _I, _P]),
    "maple_nn_accumulate": (_I, [_P, _P, _Z, _I, _P]),
    "maple_nn_relu_mask": (_I, [_P, _P, _Z, _P]),
    "maple_nn_mse": (_I, [_P, _P, _P, _P, _Z, _F, _P]),
    "maple_nn_node_weights": (_I, [_P, _P, _I, _I, _P]),
    "maple_nn_mse_weighted": (_I, [_P, _P, _P, _P, _P, _P, _I, _I, _I, _F, _P]),
    "maple_nn_error_fields": (_I, [_P, _P, _P, _P, _I, _I, _I, _I, _I, _P]),
    "maple_nn_block_dot": (_I, [_P, _P, _P, _I, _Z, _P]),
    "maple_nn_energy_grad": (_I, [_P, _P, _P, _P, _I, _I, _I, _I, _I, _I, _D, _P]),
    "maple_nn_sumsq": (_I, [_P, _Z, _P, _P]),
    "maple_nn_adam": (_I, [_P, _P, _P, _P, _P, _Z, _F, _F, _F, _F, _F, _F, _I, _P]),
    "maple_nn_to_bf16": (_I, [_P, _P, _Z, _P]),
    "maple_nn_features": (_I, [_P, _P, _I, _I, _I, _P]),
    "maple_nn_fields_to_channels": (_I, [_P, _P, _P, _I, _I, _I, _I, _I, _P, _P]),
    "maple_nn_channels_to_fields": (_I, [_P, _P, _I, _I, _I, _I, _I, _P, _P]),
    "maple_nn_prolong_fields": (_I, [_P, _P, _I, _I, _I, _P]),
    "maple_nn_restrict_density": (_I, [_P, _P, _I, _I, _I, _P]),
    "maple_nn_conv3d_padded": (_I, [_P, _P, _P, _P, _P, _P, _I, _I, _I, _I, _I, _I, _I, _P]),
    "maple_nn_wait_status": (_I, [_IP, _P]),
    # Stage-II density generator and warm-start post-processing
    "maple_gen_last_error_string": (C.c_char_p, []),
    "maple_gen_launch_count": (C.c_ulonglong, []),
    "maple_gen_linear": (_I, [_P, _P, _P, _P, _I, _I, _I, _I, _P]),
    "maple_gen_layernorm": (_I, [_P, _P, _P, _P, _I, _I, _F, _I, _P]),
    "maple_gen_upsample2": (_I, [_P, _L, _L, _L, _P, _I, _I, _I, _P]),
    "maple_gen_groupnorm": (_I, [_P, _P, _P, _I, _F, _I, _P, _P, _P, _I, _L, _I, _P]),
    "maple_gen_head_sigmoid": (_I, [_P, _P, _F, _P, _I, _L, _I, _P]),
    "maple_gen_binomial_smooth": (_I, [_P, _P, _P, _I, _I, _I, _P]),
    "maple_gen_match_mean": (_I, [_P, _P, _I, _L, _F, _F, _I, _P]),
}

NN_POOL, NN_UPSAMPLE, NN_UPSAMPLE_ADJ, NN_POOL_ADJ = 0, 1, 2, 3
NN_PAD_CIRCULAR, NN_PAD_ZEROS = 0, 1
SYM_NONE, SYM_MIRROR, SYM_CUBIC = 0, 1, 2
SEED_FACES = {"all": 0, "x": 1, "y": 2, "z": 3, "xy": 4}

_lib = None


class MapleError(RuntimeError):
    """Error status returned by the maple_b200 C ABI."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"maple_b200 error {code}: {msg}")
        self.code = code


def load(path: str = LIB_PATH):
    """Load the shared library (once) and declare every exported signature."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ImportError(
            f"maple_b200 CUDA library not found at {path}; build it with "
            "`python -m maple_b200._build` (there is no CPU fallback)")
    lib = C.CDLL(path)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def check(status: int) -> None:
    if status != MAPLE_OK:
        msg = load().maple_last_error_string()
        raise MapleError(status, msg.decode() if msg else "")


def call(name: str, *args) -> None:
    check(getattr(load(), name)(*args))


def nn_call(name: str, *args) -> None:
    """Call a maple_nn_* entry point; raise MapleError with its message."""
    lib = load()
    status = getattr(lib, name)(*args)
    if status != MAPLE_OK:
        msg = lib.maple_nn_last_error_string()
        raise MapleError(status, msg.decode() if msg else "")


def gen_call(name: str, *args) -> None:
    """Call a maple_gen_* entry point; raise MapleError with its message."""
    lib = load()
    status = getattr(lib, name)(*args)
    if status != MAPLE_OK:
        msg = lib.maple_gen_last_error_string()
        raise MapleError(status, msg.decode() if msg else "")
