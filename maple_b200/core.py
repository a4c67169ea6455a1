"""Batched homogenization context: the Python face of the C ABI.

``HomogenizationContext`` owns one ``maple_ctx`` (B periodic cells of r^3
voxels on one CUDA device) and moves torch tensors across the boundary as
raw device pointers.  Every compute call runs a CUDA kernel of
``libmaple_b200.so``; nothing here computes on the CPU.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._lib import ELASTIC, FP64, MIXED, THERMAL

PHYSICS = {"elastic": ELASTIC, "thermal": THERMAL, ELASTIC: ELASTIC, THERMAL: THERMAL}
PRECISION = {"fp64": FP64, "mixed": MIXED, FP64: FP64, MIXED: MIXED}
DR = {ELASTIC: (3, 6), THERMAL: (1, 3)}


def _ptr(t: torch.Tensor | None):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _stream(device: torch.device):
    return C.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def element_matrices(r: int, E: float = 1.0, nu: float = 0.3, kappa: float = 1.0):
    """Element tables at resolution r computed by the library's host code:
    (Ke3 24x24, Fe3 24x6, X03 24x6, Ke1 8x8, Fe1 8x3, X01 8x3) as float64 numpy
    arrays (utils/_utils.py:39-196)."""
    lib = _lib.load()
    bufs = [np.zeros(s) for s in ((24, 24), (24, 6), (24, 6), (8, 8), (8, 3), (8, 3))]
    ptrs = [b.ctypes.data_as(C.POINTER(C.c_double)) for b in bufs]
    _lib.check(lib.maple_element_matrices(int(r), float(E), float(nu), float(kappa), *ptrs))
    return tuple(bufs)


@dataclass
class SolveInfo:
    iters: np.ndarray   # per cell
    status: np.ndarray  # per cell, bit 1 = converged


class HomogenizationContext:
    """B cells of r^3 voxels: operator hierarchies, solvers and OC kernels.

    Parameters mirror the reference's IHD configuration (utils/model.py:12-32):
    E=1, nu=0.3 elasticity and kappa=1 conduction by default.
    """

    def __init__(self, r: int, ncells: int = 1, levels: int = 0, device=None, E: float = 1.0, nu: float = 0.3,
                 kappa: float = 1.0, cheb_degree: int = 1, cheb_ratio: float = 10.0, power_iters: int = 12,
                 inner_rtol: float = 1e-5, check_every: int = 1):
        if not torch.cuda.is_available():
            raise RuntimeError("maple_b200 needs a CUDA device (there is no CPU path)")
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        if self.device.type != "cuda":
            raise ValueError(f"device must be a CUDA device, got {self.device}")
        self.r, self.B, self.N = int(r), int(ncells), int(r) ** 3
        self._lib = _lib.load()
        h = C.c_void_p()
        with torch.cuda.device(self.device):
            _lib.check(self._lib.maple_ctx_create(self.r, self.B, int(levels), float(E), float(nu), float(kappa),
                                                  C.byref(h)))
        self._h = h
        self.set_options(cheb_degree, cheb_ratio, power_iters, inner_rtol, check_every)
        lv, nc, nb = C.c_int(), C.c_int(), C.c_size_t()
        _lib.check(self._lib.maple_ctx_info(self._h, C.byref(lv), C.byref(nc), C.byref(nb)))
        self.levels, self.coarsest = lv.value, nc.value

    # ------------------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None):
            with torch.cuda.device(self.device):
                torch.cuda.synchronize(self.device)
                self._lib.maple_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def bytes(self) -> int:
        nb = C.c_size_t()
        _lib.check(self._lib.maple_ctx_info(self._h, None, None, C.byref(nb)))
        return nb.value

    def set_options(self, cheb_degree=1, cheb_ratio=10.0, power_iters=12, inner_rtol=1e-5, check_every=1,
                    coarse_degree=0):
        """Smoother and solver settings; coarse_degree is the Chebyshev degree
        of multigrid levels 2 and deeper (0: automatic, 3 below level 1 and on
        a level 1 of at most 16^3 nodes)."""
        _lib.check(self._lib.maple_set_solver_options(self._h, int(cheb_degree), float(cheb_ratio), int(power_iters),
                                                      float(inner_rtol), int(check_every)))
        _lib.check(self._lib.maple_set_coarse_degree(self._h, int(coarse_degree)))

    def set_active(self, active):
        arr = None
        if active is not None:
            a = np.ascontiguousarray(np.asarray(active, dtype=np.int32).reshape(-1))
            if a.size != self.B:
                raise ValueError(f"active mask must have {self.B} entries, got {a.size}")
            arr = a.ctypes.data_as(C.POINTER(C.c_int))
        with torch.cuda.device(self.device):
            _lib.check(self._lib.maple_set_active(self._h, arr, _stream(self.device)))

    def set_symmetry(self, kind: str = "none", axes=()):
        """Symmetry projection applied by oc_step ("none", "mirror" with axes,
        "cubic"); see ``symmetrize``."""
        k, mask = _sym_args(kind, axes)
        _lib.check(self._lib.maple_set_symmetry(self._h, k, mask))

    def set_penalties(self, lambda_print: float = 0.0, overhang_deg: float = 45.0, lambda_cavity: float = 0.0, *,
                      overhang_periodic: bool = True, void_thresh: float = 0.5, beta: float = 20.0,
                      min_channel_rad: int = 0, rad: int = 1, iters: int = 0, tiles=(1, 1, 1),
                      focus_center: bool = True, seed_faces: str = "all", periodic: bool = True):
        """Manufacturability penalties of oc_step: J = J_raw - lambda_print *
        P_overhang - lambda_cavity * P_cavity (utils/printability.py); a zero
        weight disables a penalty.  tiles (1,1,1): closed-void penalty of the
        cell (periodic as given); more tiles: periodic-array penalty."""
        sf = str(seed_faces).lower()
        if sf not in _lib.SEED_FACES:
            raise ValueError("seed_faces must be one of: all, x, y, z, xy")
        tx, ty, tz = (int(t) for t in tiles)
        _lib.check(self._lib.maple_set_penalties(
            self._h, float(lambda_print), float(overhang_deg), int(bool(overhang_periodic)), float(lambda_cavity),
            float(void_thresh), float(beta), int(min_channel_rad), int(rad), int(iters), tx, ty, tz,
            int(bool(focus_center)), _lib.SEED_FACES[sf], int(bool(periodic))))

    def penalties(self, rho: torch.Tensor, overhang: bool = True, cavity: bool = True, grad: bool = True):
        """The configured penalties of rho (B, N): dict with P_print / dP_print
        and P_cavity / dP_cavity (B,) and (B, N) float64 for the requested ones."""
        self._check(rho, "rho", (self.B, self.N))
        out = {}
        t = lambda shape: torch.empty(shape, dtype=torch.float64, device=self.device)
        Pp = t((self.B,)) if overhang else None
        Pc = t((self.B,)) if cavity else None
        gp = t((self.B, self.N)) if overhang and grad else None
        gc = t((self.B, self.N)) if cavity and grad else None
        with torch.cuda.device(self.device):
            _lib.check(self._lib.maple_penalties(self._h, _ptr(rho), _ptr(Pp), _ptr(gp), _ptr(Pc), _ptr(gc),
                                                 _stream(self.device)))
        if overhang:
            out.update(P_print=Pp, dP_print=gp)
        if cavity:
            out.update(P_cavity=Pc, dP_cavity=gc)
        return out

    def set_concurrency(self, enable: bool):
        """Run the elastic and thermal solves of oc_step at the same time (default on)."""
        _lib.check(self._lib.maple_set_concurrency(self._h, int(bool(enable))))

    def set_stencil_split(self, min_n: int = 32):
        """Coarse levels with at least min_n nodes per axis use the
        split-offset stencil kernel (0: never)."""
        _lib.check(self._lib.maple_set_stencil_split(self._h, int(min_n)))

    def set_stencil_nine(self, max_n: int = 64):
        """Coarse levels with at most max_n nodes per axis use the nine-thread
        stencil kernel (0: never)."""
        _lib.check(self._lib.maple_set_stencil_nine(self._h, int(max_n)))

    def set_tail_fused(self, enable: bool = True):
        """Run the FP32 8^3-node level and the 4^3-node coarsest solve of each
        V-cycle as one cluster launch (default on; off: separate launches)."""
        _lib.check(self._lib.maple_set_tail_fused(self._h, int(bool(enable))))

    def set_pdl(self, enable: bool = True):
        """Launch the coarse-level sweeps, grid transfers and the fused V-cycle
        tail with programmatic dependent launch (default on)."""
        _lib.check(self._lib.maple_set_pdl(self._h, int(bool(enable))))

    def set_device_loop(self, enable: bool = True):
        """Loop the PCG iterations of a solve on the device (a conditional
        graph node; the host waits once per solve).  Default on; off: one
        graph replay and one host convergence check per iteration."""
        _lib.check(self._lib.maple_set_device_loop(self._h, int(bool(enable))))

    def device_loop_state(self) -> int:
        """1: a device-side loop graph is in use; 0: none built yet; -1: the
        runtime refused it (per-iteration graphs run instead)."""
        v = C.c_int(0)
        _lib.check(self._lib.maple_get_device_loop(self._h, C.byref(v)))
        return int(v.value)

    def set_mixed_mode(self, mode: str = "flexible"):
        """Form of the mixed-precision solve: "flexible" (default: FP64
        flexible PCG preconditioned by the FP32 V-cycle), "reliable" (FP32
        MG-PCG with FP64 residual replacement, the direction kept) or
        "refine" (FP32 MG-PCG inside FP64 iterative refinement)."""
        modes = {"flexible": 0, "refine": 1, "reliable": 2}
        if mode not in modes:
            raise ValueError(f"mixed mode must be one of {sorted(modes)}, got {mode!r}")
        _lib.check(self._lib.maple_set_mixed_mode(self._h, modes[mode]))

    def set_reliable_options(self, delta: float = 1e-3, handover: int = 120):
        """The "reliable" mixed form: residual reduction per FP32 segment, and
        the iterations after which an unconverged cell continues in the
        flexible form."""
        _lib.check(self._lib.maple_set_reliable_options(self._h, float(delta), int(handover)))

    def set_extrapolation(self, theta: float = 0.0):
        """oc_step(warm=True) starts its solves from u_k + theta (u_k - u_{k-1})
        (the last two steps' solutions); 0 starts from u_k."""
        _lib.check(self._lib.maple_set_extrapolation(self._h, float(theta)))

    def set_graphs(self, enable: bool):
        """Replay the PCG iteration body as a captured CUDA graph (default on)."""
        _lib.check(self._lib.maple_set_graphs(self._h, int(bool(enable))))

    def profile(self, enable: bool, max_launches: int = 100000):
        """Bracket every fine-level operator launch with CUDA events."""
        _lib.check(self._lib.maple_profile_enable(self._h, int(bool(enable)), int(max_launches)))

    def profile_read(self) -> dict:
        import json
        buf = C.create_string_buffer(1 << 16)
        _lib.check(self._lib.maple_profile_read(self._h, buf, len(buf)))
        return json.loads(buf.value.decode())

    # ------------------------------------------------------------------
    def _check(self, t: torch.Tensor, name: str, shape=None):
        if not isinstance(t, torch.Tensor):
            raise ValueError(f"{name} must be a torch.Tensor")
        if t.device != self.device:
            raise ValueError(f"{name} must be on {self.device}, got {t.device}")
        if t.dtype != torch.float64:
            raise ValueError(f"{name} must be float64, got {t.dtype}")
        if not t.is_contiguous():
            raise ValueError(f"{name} must be contiguous")
        if shape is not None and tuple(t.shape) != tuple(shape):
            raise ValueError(f"{name} must have shape {tuple(shape)}, got {tuple(t.shape)}")
        return t

    def _vec_shape(self, phys):
        D, R = DR[phys]
        return (self.B, R, D, self.N)

    def set_density(self, physics, rho: torch.Tensor, precision="fp64"):
        """rho: (B, N) float64 element densities; builds that physics' hierarchy."""
        ph, pr = PHYSICS[physics], PRECISION[precision]
        self._check(rho, "rho", (self.B, self.N))
        with torch.cuda.device(self.device):
            _lib.check(self._lib.maple_set_density(self._h, ph, _ptr(rho), pr, _stream(self.device)))

    def solve(self, physics, precision="fp64", rtol=1e-10, maxit=500, warm=False) -> SolveInfo:
        ph, pr = PHYSICS[physics], PRECISION[precision]
        it = np.zeros(self.B, dtype=np.int32)
        st = np.zeros(self.B, dtype=np.int32)
        with torch.cuda.device(self.device):
            _lib.check(self._lib.maple_solve(self._h, ph, pr, float(rtol), int(maxit), int(bool(warm)),
                                             it.ctypes.data_as(C.POINTER(C.c_int)),
                                             st.ctypes.data_as(C.POINTER(C.c_int)), _stream(self.device)))
        return SolveInfo(it, st)

    def solve_rhs(self, physics, F: torch.Tensor, x0: torch.Tensor | None = None, precision="fp64", rtol=1e-10,
                  maxit=500, want_residual=True):
        ph, pr = PHYSICS[physics], PRECISION[precision]
        shp = self._vec_shape(ph)
        self._check(F, "F", shp)
        if x0 is not None:
            self._check(x0, "x0", shp)
        u = torch.empty(shp, dtype=torch.float64, device=self.device)
        r = torch.empty_like(u) if want_residual else None
        it = np.zeros(self.B, dtype=np.int32)
        st = np.zeros(self.B, dtype=np.int32)
        with torch.cuda.device(self.device):
            _lib.check(self._lib.maple_solve_rhs(self._h, ph, pr, _ptr(F), _ptr(x0), float(rtol), int(maxit), _ptr(u),
                                                 _ptr(r), it.ctypes.data_as(C.POINTER(C.c_int)),
                                                 st.ctypes.data_as(C.POINTER(C.c_int)), _stream(self.device)))
        return u, r, SolveInfo(it, st)

    def solution(self, physics) -> torch.Tensor:
        ph = PHYSICS[physics]
        u = torch.empty(self._vec_shape(ph), dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(self._lib.maple_get_solution(self._h, ph, _ptr(u), _stream(self.device)))
        return u

    def set_solution(self, physics, u: torch.Tensor):
        """Initial iterate (B, R, D, N) for the next solve / OC step with warm=True."""
        ph = PHYSICS[physics]
        self._check(u, "u", self._vec_shape(ph))
        with torch.cuda.device(self.device):
            _lib.check(self._lib.maple_set_solution(self._h, ph, _ptr(u), _stream(self.device)))

    def level_elements(self, physics, level: int) -> torch.Tensor:
        """Galerkin element matrices (B, N_l, 8D, 8D) of multigrid level
        ``level`` (>= 1) of the last hierarchy built for ``physics``."""
        ph = PHYSICS[physics]
        D = DR[ph][0]
        if not 1 <= level < self.levels:
            raise ValueError(f"level must be in [1, {self.levels}), got {level}")
        n = self.r >> level
        out = torch.empty((self.B, n ** 3, 8 * D, 8 * D), dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(self._lib.maple_get_level_elements(self._h, ph, int(level), _ptr(out), _stream(self.device)))
        return out

    def homogenize(self, physics, want_energy=False):
        """Returns H (B,R,R) and, if asked, the per-element energies (B,R,R,N)."""
        ph = PHYSICS[physics]
        R = DR[ph][1]
        H = torch.empty((self.B, R, R), dtype=torch.float64, device=self.device)
        E = torch.empty((self.B, R, R, self.N), dtype=torch.float64, device=self.device) if want_energy else None
        with torch.cuda.device(self.device):
            _lib.check(self._lib.maple_homogenize(self._h, ph, _ptr(H), _ptr(E), _stream(self.device)))
        return (H, E) if want_energy else H

    def sensitivity(self, gC: torch.Tensor | None = None, gK: torch.Tensor | None = None) -> torch.Tensor:
        if gC is not None:
            self._check(gC, "gC", (self.B, 6, 6))
        if gK is not None:
            self._check(gK, "gK", (self.B, 3, 3))
        out = torch.empty((self.B, self.N), dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(self._lib.maple_sensitivity(self._h, _ptr(gC), _ptr(gK), _ptr(out), _stream(self.device)))
        return out

    def assemble_rhs(self, physics, rho: torch.Tensor) -> torch.Tensor:
        ph = PHYSICS[physics]
        self._check(rho, "rho", (self.B, self.N))
        F = torch.empty(self._vec_shape(ph), dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(self._lib.maple_assemble_rhs(self._h, ph, _ptr(rho), _ptr(F), _stream(self.device)))
        return F

    def matvec(self, physics, rho: torch.Tensor, u: torch.Tensor) -> torch.Tensor:
        ph = PHYSICS[physics]
        self._check(rho, "rho", (self.B, self.N))
        self._check(u, "u", self._vec_shape(ph))
        y = torch.empty_like(u)
        with torch.cuda.device(self.device):
            _lib.check(self._lib.maple_matvec(self._h, ph, _ptr(rho), _ptr(u), _ptr(y), _stream(self.device)))
        return y

    def oc_update(self, x: torch.Tensor, dJdx: torch.Tensor, volfrac: torch.Tensor, move: float, xmin: float):
        self._check(x, "x", (self.B, self.N))
        self._check(dJdx, "dJdx", (self.B, self.N))
        self._check(volfrac, "volfrac", (self.B,))
        xn = torch.empty_like(x)
        stats = torch.empty((self.B, 2), dtype=torch.float64, device=self.device)
        with torch.cuda.device(self.device):
            _lib.check(self._lib.maple_oc_update(self._h, _ptr(x), _ptr(dJdx), _ptr(volfrac), float(move),
                                                 float(xmin), _ptr(xn), _ptr(stats), _stream(self.device)))
        return xn, stats

    def oc_step(self, x: torch.Tensor, weights: torch.Tensor, volfrac: torch.Tensor, *, penal=3.0, rho_min=1e-9,
                move=0.2, xmin=1e-3, filter_k=3, precision="fp64", rtol=1e-8, maxit=500, warm=True, out=None):
        """One OC iteration for every active cell.  Returns a dict of device
        tensors: x_next (B,N), J (B,) (with the configured penalties), J_raw,
        P_print, P_cavity (B,), terms (B,3), CH (B,6,6), kappa (B,3,3),
        stats (B,2) and host iteration counts."""
        self._check(x, "x", (self.B, self.N))
        self._check(weights, "weights", (self.B, 3))
        self._check(volfrac, "volfrac", (self.B,))
        dev, B = self.device, self.B
        if out is None:
            out = dict(x_next=torch.empty_like(x), J=torch.zeros(B, dtype=torch.float64, device=dev),
                       terms=torch.zeros((B, 3), dtype=torch.float64, device=dev),
                       CH=torch.zeros((B, 6, 6), dtype=torch.float64, device=dev),
                       kappa=torch.zeros((B, 3, 3), dtype=torch.float64, device=dev),
                       stats=torch.zeros((B, 2), dtype=torch.float64, device=dev))
        it = np.zeros(B, dtype=np.int32)
        with torch.cuda.device(dev):
            _lib.check(self._lib.maple_oc_step(
                self._h, _ptr(x), _ptr(weights), _ptr(volfrac), float(penal), float(rho_min), float(move),
                float(xmin), int(filter_k), PRECISION[precision], float(rtol), int(maxit), int(bool(warm)),
                _ptr(out["x_next"]), _ptr(out["J"]), _ptr(out["terms"]), _ptr(out["CH"]), _ptr(out["kappa"]),
                _ptr(out["stats"]), it.ctypes.data_as(C.POINTER(C.c_int)), _stream(dev)))
            for k in ("J_raw", "P_print", "P_cavity"):
                if k not in out:
                    out[k] = torch.zeros(B, dtype=torch.float64, device=dev)
            _lib.check(self._lib.maple_get_oc_terms(self._h, _ptr(out["J_raw"]), _ptr(out["P_print"]),
                                                    _ptr(out["P_cavity"]), _stream(dev)))
        out["iters"] = it
        return out


def transfer(op: str, x: torch.Tensor, out: torch.Tensor | None = None) -> torch.Tensor:
    """Periodic trilinear grid transfer of (B, K, n^3) FP64 fields, K = 3 or
    18: op "restrict" returns P^T x on the (n/2)^3 grid; "prolong_add"
    returns out + P x on the (2n)^3 grid (out: zeros when None)."""
    if x.dtype != torch.float64 or not x.is_cuda or not x.is_contiguous() or x.dim() != 3:
        raise ValueError("x must be a contiguous (B, K, n^3) float64 CUDA tensor")
    B, K, N = x.shape
    n = int(round(N ** (1.0 / 3.0)))
    if n ** 3 != N:
        raise ValueError(f"{N} nodes do not form a periodic n^3 grid")
    if op == "restrict":
        if n % 2:
            raise ValueError("restriction needs an even grid")
        nc, code, shape = n // 2, 0, (B, K, (n // 2) ** 3)
        out = torch.empty(shape, dtype=torch.float64, device=x.device)
    elif op == "prolong_add":
        nc, code, shape = n, 1, (B, K, (2 * n) ** 3)
        out = torch.zeros(shape, dtype=torch.float64, device=x.device) if out is None else out
        if tuple(out.shape) != shape or out.dtype != torch.float64 or not out.is_contiguous():
            raise ValueError(f"out must be a contiguous float64 tensor of shape {shape}")
    else:
        raise ValueError(f"op must be 'restrict' or 'prolong_add', got {op!r}")
    with torch.cuda.device(x.device):
        _lib.check(_lib.load().maple_transfer(code, int(nc), int(K), int(B), _ptr(x), _ptr(out), _stream(x.device)))
    return out


def launch_count() -> int:
    """Kernels launched by libmaple_b200 in this process so far."""
    return int(_lib.load().maple_launch_count())


SYMMETRY_KINDS = {"none": _lib.SYM_NONE, "mirror": _lib.SYM_MIRROR, "cubic": _lib.SYM_CUBIC}


def _sym_args(kind: str, axes) -> tuple:
    if kind not in SYMMETRY_KINDS:
        raise ValueError(f"Unknown symmetry kind: {kind}")
    mask = 0
    for a in axes or []:
        if int(a) not in (0, 1, 2):
            raise ValueError(f"symmetry axes are 0, 1, 2; got {a}")
        mask |= 1 << int(a)
    if kind == "mirror" and mask == 0:
        raise ValueError("mirror symmetry needs at least one axis")
    return SYMMETRY_KINDS[kind], mask


def symmetrize(x: torch.Tensor, r: int, kind: str, axes=()) -> torch.Tensor:
    """Symmetry projection of (B, r^3) float64 CUDA element fields: "mirror"
    about the centre planes of `axes` (0 = x, 1 = y, 2 = z) or the 48-map
    "cubic" group (main_IHD_v3.py:259-337)."""
    if x.dtype != torch.float64 or not x.is_cuda or not x.is_contiguous():
        raise ValueError("symmetrize needs a contiguous float64 CUDA tensor")
    B = x.numel() // (r ** 3)
    if B * r ** 3 != x.numel():
        raise ValueError(f"input size {x.numel()} is not a multiple of r^3={r ** 3}")
    k, mask = _sym_args(kind, axes)
    out = torch.empty_like(x)
    with torch.cuda.device(x.device):
        _lib.check(_lib.load().maple_symmetrize(int(r), int(B), k, mask, _ptr(x), _ptr(out), _stream(x.device)))
    return out


def box_filter(x: torch.Tensor, r: int, k: int = 3) -> torch.Tensor:
    """Periodic k^3 box filter of (B, r^3) float64 CUDA data."""
    if x.dtype != torch.float64 or not x.is_cuda or not x.is_contiguous():
        raise ValueError("box_filter needs a contiguous float64 CUDA tensor")
    B = x.numel() // (r ** 3)
    if B * r ** 3 != x.numel():
        raise ValueError(f"input size {x.numel()} is not a multiple of r^3={r ** 3}")
    out = torch.empty_like(x)
    with torch.cuda.device(x.device):
        _lib.check(_lib.load().maple_box_filter(int(r), int(B), int(k), _ptr(x), _ptr(out), _stream(x.device)))
    return out


def energy_contract(energy: torch.Tensor, g: torch.Tensor, out: torch.Tensor | None = None,
                    accumulate: bool = False) -> torch.Tensor:
    """out[b,e] (+)= sum_rs g[b,r,s] energy[b,r,s,e] on the device."""
    B, R, R2, N = energy.shape
    if R != R2 or g.shape != (B, R, R):
        raise ValueError("energy (B,R,R,N) and g (B,R,R) shapes disagree")
    for name, t in (("energy", energy), ("g", g)):
        if t.dtype != torch.float64 or not t.is_cuda or not t.is_contiguous():
            raise ValueError(f"{name} must be a contiguous float64 CUDA tensor")
    if out is None:
        out = torch.zeros((B, N), dtype=torch.float64, device=energy.device)
    with torch.cuda.device(energy.device):
        _lib.check(_lib.load().maple_energy_contract(B, N, R * R, _ptr(energy), _ptr(g), int(bool(accumulate)),
                                                     _ptr(out), _stream(energy.device)))
    return out
