"""ctypes binding of the multithreaded C restatement of the oracle (port.c).

TEST AND MEASUREMENT INFRASTRUCTURE ONLY: the CPU baseline that ``bench.py``
times beside the GPU path, checked against the numpy oracle by
``tests/test_port_oracle.py``.  The product path never imports it.

``oc_iteration`` has the arguments and results of
``ihd_oracle.oc_iteration`` (symmetry "none", no penalties), computed with the
same algorithm (the reference's V-cycles with 8-colour Gauss-Seidel to a
relative residual, main_IHD_v3.py:620-716) on ``threads`` host cores.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from . import ihd_oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_port", "libmaple_port.so")
_lib = None


def build() -> str:
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(os.path.join(HERE, "port.c")):
        subprocess.run(["make", "-C", HERE], check=True, capture_output=True)
    return LIB


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        lib = C.CDLL(LIB)
        P = C.c_void_p
        lib.port_threads.restype = C.c_int
        lib.port_threads.argtypes = [C.c_int]
        lib.port_oc_iteration.restype = C.c_int
        lib.port_oc_iteration.argtypes = [C.c_int, C.c_int, P, P, P, C.c_double, C.c_double, C.c_double,
                                          C.c_double, C.c_double, C.c_int, C.c_double, C.c_int, C.c_int, P, C.c_int,
                                          P, C.c_int, P, P]
        _lib = lib
    return _lib


def set_threads(n: int = 0) -> int:
    """Use n OpenMP threads (0: keep the default, all cores); returns the count."""
    return int(load().port_threads(int(n)))


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p)


class Cell:
    """State of one cell across OC iterations: element tables and the last
    solutions (the next iteration's initial iterates when ``warm``)."""

    def __init__(self, r: int, levels: int):
        self.r, self.levels = r, levels
        el = O.Elements(r)
        Ke3, Fe3, X03 = el.get(3)
        Ke1, Fe1, X01 = el.get(1)
        self.tabs = np.ascontiguousarray(np.concatenate([a.reshape(-1) for a in (Ke3, Fe3, X03, Ke1, Fe1, X01)]))
        N = r ** 3
        self.u3 = np.zeros((N, 3, 6))
        self.u1 = np.zeros((N, 1, 3))
        self.solved = [False, False]


def oc_iteration(x, cell: Cell, weights: dict, *, volfrac: float, penal: float = 3.0, rho_min: float = 1e-9,
                 move: float = 0.2, xmin: float = 1e-3, filter_k: int = 3, rtol: float = 1e-12,
                 max_cycles: int = 200, warm: bool = False, method: str = "vcycle"):
    """One OC iteration of the cell's design x (N,); returns (x_next, info)
    with J, CH, kappa, cycles_elastic, cycles_thermal, dx_max, dx_mean.
    ``method`` as in ``ihd_oracle.gmg_solve`` ("vcycle" or "pcg")."""
    if method not in ("vcycle", "pcg"):
        raise ValueError(f"unknown method {method!r}")
    lib = load()
    r = cell.r
    x = np.ascontiguousarray(np.asarray(x, dtype=np.float64).reshape(-1))
    w3 = np.array([weights.get("stiffness", 0.0), weights.get("shear", 0.0), weights.get("thermal", 0.0)])
    xn = np.empty_like(x)
    out = np.zeros(50)
    rc = lib.port_oc_iteration(r, cell.levels, _ptr(cell.tabs), _ptr(x), _ptr(w3), float(volfrac), float(penal),
                               float(rho_min), float(move), float(xmin), int(filter_k), float(rtol), int(max_cycles),
                               1 if method == "pcg" else 0, _ptr(cell.u3), int(warm and cell.solved[0]), _ptr(cell.u1),
                               int(warm and cell.solved[1]), _ptr(xn), _ptr(out))
    if rc != 0:
        raise ValueError("port_oc_iteration: bad argument")
    if w3[0] or w3[1]:
        cell.solved[0] = True
    if w3[2]:
        cell.solved[1] = True
    info = dict(J=float(out[0]), CH=out[1:37].reshape(6, 6).copy(), kappa=out[37:46].reshape(3, 3).copy(),
                cycles_elastic=int(out[46]), cycles_thermal=int(out[47]), dx_max=float(out[48]),
                dx_mean=float(out[49]))
    return xn, info
