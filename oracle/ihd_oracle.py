"""FP64 CPU oracle for MAPLE's inverse-homogenization inner loop.

TEST INFRASTRUCTURE ONLY.  This module is the checker: only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py`` may import it.  The product path (``maple_b200``) never
calls it and fails loudly when its CUDA library is missing.

It restates, in numpy/scipy FP64, the algorithm of the reference package
``maple`` (xing-yuu/MAPLE, ``src/maple``).  Each function cites the reference
file:line it follows.  Paths are relative to ``src/maple/core``.

Parity pin: ``tests/golden/make_golden.py`` runs the reference's own code
(imported from its source tree, FP64 element matrices, converged V-cycles,
autograd sensitivities) and stores the results as ``tests/golden/*.npz``;
``tests/test_oracle_golden.py`` checks this module against them.

Conventions (same as the reference):
  * ``r`` voxels per axis, ``N = r**3`` elements = nodes (periodic cell).
  * element / node id ``x*r*r + y*r + z`` (main_IHD_v3.py:175-186).
  * element-local node order ``000,100,110,010,001,101,111,011``
    (main_IHD_v3.py:189-193).
  * DOF id ``3*node + c`` (EBE_GMG.py:796); Voigt order xx,yy,zz,xy,yz,zx
    (utils/_utils.py:91-100).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp

# element-local corner offsets (main_IHD_v3.py:189-193, EBE_GMG.py:480-489)
HEX8 = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0],
                 [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], dtype=np.int64)
_SIGNS = 2 * HEX8 - 1                                   # (8,3) in {-1,+1}
_GP = np.array([-np.sqrt(3.0 / 5.0), 0.0, np.sqrt(3.0 / 5.0)])
_GW = np.array([5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0])
ELASTIC_FIXED_DOFS = (0, 1, 2, 4, 5, 11)                # utils/_utils.py:105-106


# ---------------------------------------------------------------------------
# element matrices
# ---------------------------------------------------------------------------
def isotropic_elastic_tensor(E: float = 1.0, nu: float = 0.3, f32_entries: bool = True) -> np.ndarray:
    """6x6 isotropic stiffness in Voigt form (utils/_utils.py:39-48).

    The reference builds it with ``torch.as_tensor`` of Python floats, i.e. in
    float32 (utils/_utils.py:42), and every FP64 use of it casts those float32
    values up.  ``f32_entries`` reproduces that rounding of lambda+2mu, lambda,
    mu (a 1e-8 relative effect on every element matrix)."""
    lam = nu / (1.0 + nu) / (1.0 - 2.0 * nu) * E
    mu = 1.0 / (2.0 * (1.0 + nu)) * E
    if f32_entries:
        lam2mu = float(np.float32(lam + 2 * mu))
        lam, mu = float(np.float32(lam)), float(np.float32(mu))
    else:
        lam2mu = lam + 2 * mu
    C = np.zeros((6, 6))
    C[:3, :3] = lam
    C[np.arange(3), np.arange(3)] = lam2mu
    C[np.arange(3, 6), np.arange(3, 6)] = mu
    return C


def _shape_grads(xi, eta, zeta):
    """d N_a / d(xi,eta,zeta) for the 8 trilinear corners, shape (3,8)."""
    s = _SIGNS
    g = np.empty((3, 8))
    g[0] = s[:, 0] * (1 + s[:, 1] * eta) * (1 + s[:, 2] * zeta) / 8.0
    g[1] = s[:, 1] * (1 + s[:, 0] * xi) * (1 + s[:, 2] * zeta) / 8.0
    g[2] = s[:, 2] * (1 + s[:, 0] * xi) * (1 + s[:, 1] * eta) / 8.0
    return g


def _gauss_points():
    for i in range(3):
        for j in range(3):
            for k in range(3):
                yield _GP[i], _GP[j], _GP[k], _GW[i] * _GW[j] * _GW[k]


def hexahedron(r: int, C: np.ndarray):
    """Ke0 (24,24), Fe0 (24,6), X0 (24,6) of one voxel of edge 1/r.

    3x3x3 Gauss quadrature of B^T C B and B^T C; X0 solves Ke0 X0 = Fe0 with
    DOFs 0,1,2,4,5,11 pinned to zero (utils/_utils.py:49-109).
    """
    h = 1.0 / r / 2.0
    corners = _SIGNS * h                                  # (8,3) physical coords
    Ke = np.zeros((24, 24))
    Fe = np.zeros((24, 6))
    for xi, eta, zeta, w in _gauss_points():
        dN = _shape_grads(xi, eta, zeta)                  # (3,8)
        J = dN @ corners
        dNx = np.linalg.solve(J, dN)                      # (3,8)
        B = np.zeros((6, 24))
        for a in range(8):
            gx, gy, gz = dNx[:, a]
            c = 3 * a
            B[0, c] = gx
            B[1, c + 1] = gy
            B[2, c + 2] = gz
            B[3, c], B[3, c + 1] = gy, gx
            B[4, c + 1], B[4, c + 2] = gz, gy
            B[5, c], B[5, c + 2] = gz, gx
        wd = np.linalg.det(J) * w
        Ke += wd * B.T @ C @ B
        Fe += wd * B.T @ C
    free = np.ones(24, dtype=bool)
    free[list(ELASTIC_FIXED_DOFS)] = False
    X0 = np.zeros((24, 6))
    X0[free] = np.linalg.solve(Ke[np.ix_(free, free)], Fe[free])
    return Ke, Fe, X0


def hexahedron_scalar(r: int, kappa: float = 1.0):
    """Ke0 (8,8), Fe0 (8,3), X0 (8,3) for scalar conduction, node 0 anchored
    (utils/_utils.py:116-196)."""
    h = 1.0 / r / 2.0
    corners = _SIGNS * h
    Ke = np.zeros((8, 8))
    Fe = np.zeros((8, 3))
    for xi, eta, zeta, w in _gauss_points():
        dN = _shape_grads(xi, eta, zeta)
        J = dN @ corners
        G = np.linalg.solve(J, dN)                        # (3,8)
        wd = np.linalg.det(J) * w * kappa
        Ke += wd * G.T @ G
        Fe += wd * G.T
    X0 = np.zeros((8, 3))
    X0[1:] = np.linalg.solve(Ke[1:, 1:], Fe[1:])
    return Ke, Fe, X0


class Elements:
    """Element matrices of both physics at resolution r (model.py:18-28)."""

    def __init__(self, r: int, E: float = 1.0, nu: float = 0.3, kappa: float = 1.0):
        self.r = r
        self.C = isotropic_elastic_tensor(E, nu)
        self.Ke3, self.Fe3, self.X03 = hexahedron(r, self.C)
        self.Ke1, self.Fe1, self.X01 = hexahedron_scalar(r, kappa)

    def get(self, d: int):
        return (self.Ke3, self.Fe3, self.X03) if d == 3 else (self.Ke1, self.Fe1, self.X01)


# ---------------------------------------------------------------------------
# structured periodic grid
# ---------------------------------------------------------------------------
def grid_coords(n: int) -> np.ndarray:
    g = np.stack(np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing="ij"), -1)
    return g.reshape(-1, 3)


def node_index(n: int) -> np.ndarray:
    """Periodic element->node table (N,8) (main_IHD_v3.py:174-197)."""
    g = grid_coords(n)
    c = (g[:, None, :] + HEX8[None]) % n
    return (c[..., 0] * n + c[..., 1]) * n + c[..., 2]


def dof_index(n: int, d: int) -> np.ndarray:
    ni = node_index(n)
    return (ni[:, :, None] * d + np.arange(d)[None, None]).reshape(ni.shape[0], 8 * d)


def assemble_F(rho: np.ndarray, Fe: np.ndarray, n: int, d: int) -> np.ndarray:
    """F = sum_e rho_e Fe0 scattered to nodes -> (N*d, R)
    (utils/_utils.py:453-507, assemble_F_fast / assemble_F_fast_scalar)."""
    di = dof_index(n, d)
    R = Fe.shape[1]
    F = np.zeros((n ** 3 * d, R))
    vals = rho.reshape(-1, 1, 1) * Fe[None]
    np.add.at(F, di.reshape(-1), vals.reshape(-1, R))
    return F


def assemble_K(ke: np.ndarray, n: int, d: int) -> sp.csr_matrix:
    """Assembled operator of per-element matrices ke (M,8d,8d) on an n^3
    periodic grid: the EBE matvec of EBE_GMG.py:412-430 as a sparse matrix."""
    di = dof_index(n, d)
    k = 8 * d
    rows = np.repeat(di, k, axis=1).reshape(-1)
    cols = np.tile(di, (1, k)).reshape(-1)
    K = sp.coo_matrix((ke.reshape(-1), (rows, cols)), shape=(n ** 3 * d,) * 2).tocsr()
    K.sum_duplicates()
    return K


def _child_prolongation():
    """Per child c of a coarse element, the 8x8 trilinear weights from the
    coarse corners to the child's corners (EBE_GMG.py:202-224, 226-337)."""
    out = np.zeros((8, 8, 8))
    for c in range(8):
        co = np.array([(c >> 2) & 1, (c >> 1) & 1, c & 1])
        for a in range(8):
            p = co + HEX8[a]                                # position in {0,1,2}^3
            for b in range(8):
                out[c, a, b] = np.prod(1.0 - np.abs(p / 2.0 - HEX8[b]))
    return out


_PCHILD = _child_prolongation()


def coarsen_elements(ke: np.ndarray, n: int, d: int) -> np.ndarray:
    """Galerkin coarse element matrices  Kc_E = sum_children P_c^T K_c P_c
    (EBE_GMG.py:226-337 / EBE_GMG_scalar.py:135-230).  Equivalent to
    P_loc^T K_patch P_loc because each child's corners interpolate only from
    the coarse element's own corners."""
    nc = n // 2
    g = grid_coords(n)
    cid = ((g[:, 0] // 2) * nc + g[:, 1] // 2) * nc + g[:, 2] // 2
    child = (g[:, 0] % 2) * 4 + (g[:, 1] % 2) * 2 + (g[:, 2] % 2)
    k = 8 * d
    out = np.zeros((nc ** 3, k, k))
    I = np.eye(d)
    for c in range(8):
        Pc = np.kron(_PCHILD[c], I)                          # (8d, 8d)
        m = child == c
        contrib = np.einsum("ai,eab,bj->eij", Pc, ke[m], Pc, optimize=True)
        np.add.at(out, cid[m], contrib)
    return out


def prolongation(nf: int, d: int) -> sp.csr_matrix:
    """Global periodic trilinear P: coarse (nf/2)^3 -> fine nf^3
    (EBE_GMG.py:531-647, weights prod(1 - |rem/2 - off|))."""
    nc = nf // 2
    g = grid_coords(nf)
    base, rem = g // 2, g % 2
    rows, cols, vals = [], [], []
    for o in range(8):
        off = np.array([(o >> 2) & 1, (o >> 1) & 1, o & 1])
        t = (base + off) % nc
        w = np.prod(1.0 - np.abs(0.5 * rem - off), axis=1)
        ci = (t[:, 0] * nc + t[:, 1]) * nc + t[:, 2]
        keep = w != 0
        fi = np.arange(nf ** 3)[keep]
        for c in range(d):
            rows.append(fi * d + c)
            cols.append(ci[keep] * d + c)
            vals.append(w[keep])
    P = sp.coo_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                      shape=(nf ** 3 * d, nc ** 3 * d)).tocsr()
    P.sum_duplicates()
    return P


def colors(n: int) -> np.ndarray:
    """Parity colour of each node (EBE_GMG.py:354-374)."""
    g = grid_coords(n)
    return (g[:, 0] % 2) * 4 + (g[:, 1] % 2) * 2 + (g[:, 2] % 2)


# ---------------------------------------------------------------------------
# geometric multigrid (reference algorithm: V-cycles with 8-colour GS)
# ---------------------------------------------------------------------------
class Level:
    def __init__(self, ke: np.ndarray, n: int, d: int):
        self.n, self.d = n, d
        self.ke = ke
        self.K = assemble_K(ke, n, d)
        diag = self.K.diagonal().copy()
        diag[diag == 0] = 1.0                               # EBE_GMG.py:387-388
        self.dinv = 1.0 / diag
        col = np.repeat(colors(n), d)
        self.color_rows = [np.nonzero(col == c)[0] for c in range(8)]
        self.Kc = [self.K[rows] for rows in self.color_rows]
        self.P = None                                       # fine(level-1) <- this level


class Hierarchy:
    """Operator hierarchy of GMGSolver.solve (EBE_GMG.py:790-849) for the
    per-element matrices rho_e * Ke0."""

    def __init__(self, rho: np.ndarray, Ke0: np.ndarray, n: int, d: int, levels: int):
        ke = rho.reshape(-1, 1, 1) * Ke0[None]             # model.py:108
        self.levels = [Level(ke, n, d)]
        for _ in range(1, levels):
            if n % 2 or n < 2:
                break
            ke = coarsen_elements(ke, n, d)
            P = prolongation(n, d)
            n //= 2
            lv = Level(ke, n, d)
            lv.P = P
            self.levels.append(lv)

    def gs_sweeps(self, lv: Level, u, f, sweeps: int, reverse: bool = False):
        """8-colour Gauss-Seidel, omega=1 (EBE_GMG.py:431-459)."""
        order = range(7, -1, -1) if reverse else range(8)
        for _ in range(sweeps):
            for c in order:
                rows = lv.color_rows[c]
                if rows.size == 0:
                    continue
                r = f[rows] - lv.Kc[c] @ u
                u[rows] += lv.dinv[rows, None] * r
        return u

    def vcycle(self, l: int, u, f, smooth_iter, coarse_default: int | None, symmetric: bool = False):
        """One V-cycle (EBE_GMG.py:886-984).  ``coarse_default`` reproduces the
        elastic solver's recursion, which does not forward ``smooth_iter`` and so
        smooths coarser levels with the default of 1 sweep (EBE_GMG.py:955-963);
        the scalar solver forwards it (EBE_GMG_scalar.py:802-811): pass None.

        ``symmetric``: post-smoothing (and the coarsest level's second half)
        runs the colours in reverse order, which makes the cycle a symmetric
        operator (a preconditioner for plain CG); the reference's cycle runs
        them forward both times."""
        lv = self.levels[l]
        if l > 0 and coarse_default is not None:
            nu = coarse_default
        elif isinstance(smooth_iter, (list, tuple)):
            nu = 1 if len(smooth_iter) == 0 else smooth_iter[min(l, len(smooth_iter) - 1)]
        else:
            nu = int(smooth_iter)
        u = self.gs_sweeps(lv, u, f, nu)
        if l == len(self.levels) - 1:
            return self.gs_sweeps(lv, u, f, nu if symmetric else 1, reverse=symmetric)
        r = f - lv.K @ u
        nxt = self.levels[l + 1]
        rc = nxt.P.T @ r
        uc = self.vcycle(l + 1, np.zeros_like(rc), rc, smooth_iter, coarse_default, symmetric)
        u = u + nxt.P @ uc
        return self.gs_sweeps(lv, u, f, nu, reverse=symmetric)


def gmg_solve(hier: Hierarchy, f: np.ndarray, max_iter: int, smooth_iter=(2, 2, 3, 4, 5),
              coarse_default: int | None = 1, rtol: float = 0.0, u0=None, method: str = "vcycle"):
    """V-cycle iteration from u=0 (EBE_GMG.py:758-885).  Returns (u, r, cycles).
    ``rtol`` > 0 stops early once ||r|| <= rtol ||f|| per column (the reference
    has no test; it runs ``max_iter`` cycles).

    ``method="pcg"``: the V-cycle in its symmetric form (post-smoothing in
    reverse colour order; one cycle from zero on the residual) as the
    preconditioner of a conjugate gradient (Polak-Ribiere beta, per load
    case); it reaches residuals the plain cycle stalls above on designs with
    large density contrast.  The converged answer is the same (up to a rigid
    translation, which C^H ignores)."""
    u = np.zeros_like(f) if u0 is None else u0.copy()
    K = hier.levels[0].K
    fn = np.maximum(np.linalg.norm(f, axis=0), 1e-300)
    it = 0
    r = f - K @ u
    if method == "pcg":
        if rtol > 0 and np.all(np.linalg.norm(r, axis=0) <= rtol * fn):
            return u, r, 0
        z = hier.vcycle(0, np.zeros_like(r), r, smooth_iter, coarse_default, True)
        p = z.copy()
        rz = np.sum(r * z, axis=0)
        for it in range(1, max_iter + 1):
            q = K @ p
            pq = np.sum(p * q, axis=0)
            alpha = np.where(pq > 0, rz / np.where(pq > 0, pq, 1.0), 0.0)
            u = u + alpha * p
            r_old = r
            r = r - alpha * q
            if rtol > 0 and np.all(np.linalg.norm(r, axis=0) <= rtol * fn):
                break
            z = hier.vcycle(0, np.zeros_like(r), r, smooth_iter, coarse_default, True)
            beta = np.where(rz != 0, np.sum(z * (r - r_old), axis=0) / np.where(rz != 0, rz, 1.0), 0.0)
            rz = np.sum(r * z, axis=0)
            p = z + beta * p
        return u, f - K @ u, it
    for it in range(1, max_iter + 1):
        u = hier.vcycle(0, u, f, smooth_iter, coarse_default)
        r = f - K @ u
        if rtol > 0 and np.all(np.linalg.norm(r, axis=0) <= rtol * fn):
            break
    return u, r, it


# ---------------------------------------------------------------------------
# homogenization, sensitivities, objectives
# ---------------------------------------------------------------------------
def element_fields(u: np.ndarray, n: int, d: int) -> np.ndarray:
    """Gather per-element DOF blocks (N, 8d, R) (model.py:39-41)."""
    return u[dof_index(n, d)]


def homogenize(u: np.ndarray, rho: np.ndarray, Ke0: np.ndarray, X0: np.ndarray, n: int, d: int):
    """C^H (or kappa^H) = sum_e (X0-u_e)^T rho_e Ke0 (X0-u_e), volume 1
    (model.py:33-44, 47-95)."""
    L = X0[None] - element_fields(u, n, d)
    KL = np.einsum("ij,ejk->eik", Ke0, L, optimize=True)
    return np.einsum("eij,e,eik->jk", L, rho.reshape(-1), KL, optimize=True)


def element_energy(u: np.ndarray, Ke0: np.ndarray, X0: np.ndarray, n: int, d: int) -> np.ndarray:
    """Per-element (X0-u_e)^T Ke0 (X0-u_e): (N,R,R) = dC^H/drho_e at a converged
    solve (the analytic adjoint of the autograd call at main_IHD_v3.py:688)."""
    L = X0[None] - element_fields(u, n, d)
    KL = np.einsum("ij,ejk->eik", Ke0, L, optimize=True)
    return np.einsum("eij,eik->ejk", L, KL, optimize=True)


def _sym_inv(CH):
    C = 0.5 * (CH + CH.T)
    return np.linalg.inv(C + 1e-9 * np.eye(6))


def stiffness_objective(CH):
    """mean(1/S_ii), i=0..2, S=inv(sym(C)+1e-9 I) (utils/objective.py:11-19)."""
    S = _sym_inv(CH)
    return float(np.mean(1.0 / np.diag(S)[:3]))


def shear_objective(CH):
    """mean(1/S_ii), i=3..5 (utils/objective.py:22-30)."""
    S = _sym_inv(CH)
    return float(np.mean(1.0 / np.diag(S)[3:]))


def thermal_objective(kappa):
    """trace(kappa) (utils/objective.py:33-41)."""
    return float(np.trace(kappa))


def _grad_modulus(CH, idx):
    """d/dCH of mean(1/S_ii over idx): with dS = -S dC S on sym(C),
    d(1/S_ii) = S[:,i] S[i,:] / S_ii^2, then symmetrised by C=(CH+CH^T)/2."""
    S = _sym_inv(CH)
    G = np.zeros((6, 6))
    for i in idx:
        G += np.outer(S[:, i], S[i, :]) / S[i, i] ** 2
    G /= len(idx)
    return 0.5 * (G + G.T)


_ALIASES = {"stiff": "stiffness", "stiffness": "stiffness", "e": "stiffness", "young": "stiffness",
            "youngs": "stiffness", "shear": "shear", "g": "shear", "thermal": "thermal",
            "kappa": "thermal", "conductivity": "thermal", "heat": "thermal"}


def parse_objective_spec(spec) -> dict:
    """Weighted-term parser (utils/objective.py:93-157)."""
    import re
    if spec is None or not str(spec).strip():
        return {"shear": 1.0}
    s = str(spec).strip()
    if s.lower() in _ALIASES:
        return {_ALIASES[s.lower()]: 1.0}
    out: dict = {}
    for part in [p for p in re.split(r"[,+]", s.replace(" ", "")) if p]:
        if ":" in part or "=" in part:
            name, w = re.split(r"[:=]", part, maxsplit=1)
            w = float(w)
        elif "*" in part:
            a, b = part.split("*", 1)
            try:
                w, name = float(a), b
            except ValueError:
                w, name = float(b), a
        else:
            name, w = part, 1.0
        key = _ALIASES[name.lower()]
        out[key] = out.get(key, 0.0) + w
    return out


def objective_and_grads(weights: dict, CH, kappa):
    """J = sum_t w_t term_t and (dJ/dCH, dJ/dkappa) (utils/objective.py:180-251)."""
    J = 0.0
    gC = np.zeros((6, 6))
    gK = np.zeros((3, 3))
    for t, w in weights.items():
        if t == "stiffness":
            J += w * stiffness_objective(CH)
            gC += w * _grad_modulus(CH, (0, 1, 2))
        elif t == "shear":
            J += w * shear_objective(CH)
            gC += w * _grad_modulus(CH, (3, 4, 5))
        else:
            J += w * thermal_objective(kappa)
            gK += w * np.eye(3)
    return J, gC, gK


# ---------------------------------------------------------------------------
# filter, OC
# ---------------------------------------------------------------------------
def box_filter_periodic(v: np.ndarray, n: int, k: int = 3) -> np.ndarray:
    """Periodic k^3 box mean (main_IHD_v3.py:342-359)."""
    if k <= 0 or k % 2 == 0:
        raise ValueError(f"filter size must be a positive odd integer, got {k}")
    vol = v.reshape(n, n, n)
    acc = np.zeros_like(vol)
    p = k // 2
    for dx in range(-p, p + 1):
        for dy in range(-p, p + 1):
            for dz in range(-p, p + 1):
                acc += np.roll(vol, (-dx, -dy, -dz), axis=(0, 1, 2))
    return (acc / float(k ** 3)).reshape(v.shape)


def oc_update(x: np.ndarray, dJdx: np.ndarray, volfrac: float, move: float = 0.1,
              xmin: float = 1e-3) -> np.ndarray:
    """60-step OC bisection (main_IHD_v3.py:362-380); returns the x of the last
    bisection step, exactly as the reference does."""
    dJ = np.maximum(dJdx, 1e-12)
    l1, l2 = 1e-12, 1e6
    xn = x
    for _ in range(60):
        lam = 0.5 * (l1 + l2)
        xn = x * np.sqrt(dJ / lam)
        xn = np.minimum(np.maximum(xn, x - move), x + move)
        xn = np.minimum(np.maximum(xn, xmin), 1.0)
        if xn.mean() > volfrac:
            l1 = lam
        else:
            l2 = lam
    return xn


# ---------------------------------------------------------------------------
# seeded synthetic densities (benchmark inputs)
# ---------------------------------------------------------------------------
def seed_density(seed: int, r: int, sigma: float, vf: float, scale: float = 0.25,
                 xmin: float = 1e-3) -> np.ndarray:
    """N(0,1) voxels, periodic Gaussian smoothing (FFT), standardise, affine map
    to mean vf with scale 0.25, clip to [xmin,1], mean-matching rounds until
    |mean - vf| < 1e-12 (at most 200).
    Returns x of shape (r,r,r), float64."""
    z = np.random.default_rng(seed).standard_normal((r, r, r))
    k = np.fft.fftfreq(r)
    k2 = k[:, None, None] ** 2 + k[None, :, None] ** 2 + k[None, None, :] ** 2
    z = np.real(np.fft.ifftn(np.fft.fftn(z) * np.exp(-2.0 * (np.pi ** 2) * (sigma ** 2) * k2)))
    z = (z - z.mean()) / z.std()
    x = np.clip(vf + scale * z, xmin, 1.0)
    for _ in range(200):  # mean matching; converges geometrically unless vf is tiny
        x = np.clip(x - x.mean() + vf, xmin, 1.0)
        if abs(x.mean() - vf) < 1e-12:
            break
    return x


# ---------------------------------------------------------------------------
# one full homogenization + sensitivity evaluation
# ---------------------------------------------------------------------------
def solve_cell(rho: np.ndarray, r: int, elems: Elements | None = None, levels: int = 3,
               max_cycles: int = 200, rtol: float = 1e-12, physics=("elastic", "thermal"),
               smooth_iter=(2, 2, 3, 4, 5), u0: dict | None = None, method: str = "vcycle"):
    """Both physics on one cell: returns dict with CH, kappa, u3, u1 and the
    per-element energies (dC/drho, dkappa/drho).  ``u0`` (keys "u3" / "u1",
    e.g. the previous OC iteration's solutions) is the initial iterate of the
    V-cycles; the converged answer does not depend on it (the reference starts
    from zero, EBE_GMG.py:851-858).  ``method`` as in ``gmg_solve``."""
    elems = elems or Elements(r)
    out = {}
    rho = rho.reshape(-1)
    for ph in physics:
        d = 3 if ph == "elastic" else 1
        Ke0, Fe0, X0 = elems.get(d)
        hier = Hierarchy(rho, Ke0, r, d, levels)
        F = assemble_F(rho, Fe0, r, d)
        key_u = "u3" if d == 3 else "u1"
        start = None if u0 is None else u0.get(key_u)
        u, res, cyc = gmg_solve(hier, F, max_cycles, smooth_iter,
                                coarse_default=1 if d == 3 else None, rtol=rtol, u0=start, method=method)
        H = homogenize(u, rho, Ke0, X0, r, d)
        dH = element_energy(u, Ke0, X0, r, d)
        key = "CH" if d == 3 else "kappa"
        out[key] = H
        out["d" + key] = dH
        out["u3" if d == 3 else "u1"] = u
        out["cycles_" + ph] = cyc
        out["relres_" + ph] = np.linalg.norm(res, axis=0) / np.maximum(np.linalg.norm(F, axis=0), 1e-300)
    return out


def parse_symmetry(symmetry: str):
    """(kind, axes) of a symmetry spec (main_IHD_v3.py:221-256): "none";
    "mirror" with the sorted axes named by x/y/z letters ("octant", "1/8",
    "one_eighth" mean all three); "cubic" for "cubic", "iso", "isotropic"."""
    sym = (symmetry or "none").lower().strip()
    if sym in ("none", ""):
        return "none", []
    if sym in ("octant", "1/8", "one_eighth"):
        sym = "xyz"
    if sym in ("cubic", "iso", "isotropic"):
        return "cubic", [0, 1, 2]
    axes = sorted({i for i, ch in enumerate("xyz") if ch in sym})
    return ("mirror", axes) if axes else ("none", [])


def symmetrize(v: np.ndarray, r: int, kind: str, axes) -> np.ndarray:
    """Group average of an element field (main_IHD_v3.py:259-337): mirror =
    mean over the reflections about the centre planes of `axes`; cubic = mean
    over the 48 axis permutations and reflections.  Index i reflects to r-1-i."""
    if kind == "none":
        return v.reshape(-1).copy()
    vol = v.reshape(r, r, r)
    if kind == "mirror":
        out = vol
        for ax in axes:
            out = 0.5 * (out + np.flip(out, axis=ax))
        return np.ascontiguousarray(out).reshape(-1)
    if kind == "cubic":
        import itertools
        acc = np.zeros_like(vol)
        for p in itertools.permutations((0, 1, 2)):
            w = np.transpose(vol, p)
            for f in itertools.product((0, 1), repeat=3):
                dims = tuple(i for i in range(3) if f[i])
                acc += np.flip(w, axis=dims) if dims else w
        return (acc / 48.0).reshape(-1)
    raise ValueError(f"Unknown symmetry kind: {kind}")


def oc_iteration(x: np.ndarray, r: int, weights: dict, *, volfrac: float, penal: float = 3.0,
                 rho_min: float = 1e-9, move: float = 0.2, xmin: float = 1e-3, filter_k: int = 3,
                 elems: Elements | None = None, levels: int = 3, rtol: float = 1e-12,
                 max_cycles: int = 200, symmetry: str = "none", lambda_print: float = 0.0,
                 overhang_deg: float = 45.0, lambda_cavity: float = 0.0, cavity: dict | None = None,
                 u0: dict | None = None, method: str = "vcycle"):
    """One OC iteration of main_IHD_v3.py:620-716 with the analytic adjoint in
    place of autograd.  With a symmetry, the solve uses the projected design,
    the gradient is projected (the group average is self-adjoint) and so is
    the updated design.  Penalties (:649-686): J = J_raw - lambda_print *
    P_overhang - lambda_cavity * P_cavity, `cavity` holding cavity_penalty's
    keywords.  ``u0`` is passed to ``solve_cell`` as the solves' initial
    iterate (``info["res"]`` of the previous iteration serves); ``method``
    selects the solver as in ``gmg_solve``.  Returns (x_next, info)."""
    kind, axes = parse_symmetry(symmetry)
    x = x.reshape(-1)
    xc = np.clip(symmetrize(np.clip(x, xmin, 1.0), r, kind, axes), xmin, 1.0)
    rho = rho_min + (1.0 - rho_min) * xc ** penal
    phys = []
    if any(t in ("stiffness", "shear") for t in weights):
        phys.append("elastic")
    if "thermal" in weights:
        phys.append("thermal")
    res = solve_cell(rho, r, elems, levels, max_cycles, rtol, tuple(phys), u0=u0, method=method)
    CH = res.get("CH")
    kap = res.get("kappa")
    J, gC, gK = objective_and_grads(weights, CH if CH is not None else np.eye(6),
                                    kap if kap is not None else np.eye(3))
    dJdrho = np.zeros(r ** 3)
    if CH is not None:
        dJdrho += np.einsum("eij,ij->e", res["dCH"], gC)
    if kap is not None:
        dJdrho += np.einsum("eij,ij->e", res["dkappa"], gK)
    J_raw = J
    P_print = P_cav = 0.0
    if lambda_print > 0:
        P_print, gP = overhang_penalty(rho, r, overhang_deg, True)
        J -= lambda_print * P_print
        dJdrho = dJdrho - lambda_print * gP
    if lambda_cavity > 0:
        P_cav, gC = cavity_penalty(rho, r, **(cavity or {}))
        J -= lambda_cavity * P_cav
        dJdrho = dJdrho - lambda_cavity * gC
    dJdx = symmetrize(dJdrho * penal * (1.0 - rho_min) * xc ** (penal - 1.0), r, kind, axes)
    if filter_k and filter_k > 1:
        dJdx = box_filter_periodic(dJdx, r, filter_k)
    x_new = oc_update(x, dJdx, volfrac, move, xmin)
    x_next = np.clip(symmetrize(x_new, r, kind, axes), xmin, 1.0)
    info = dict(J=J, J_raw=J_raw, P_print=P_print, P_cavity=P_cav, CH=CH, kappa=kap, dJdx=dJdx,
                dx_max=float(np.abs(x_next - x).max()),
                dx_mean=float(np.abs(x_next - x).mean()), res=res)
    return x_next, info


# ---------------------------------------------------------------------------
# Manufacturability penalties (utils/printability.py) with their gradients,
# restated with the tie rules of the autograd the reference differentiates
# them with: a max-pool window passes its gradient to the first maximum in
# (x, y, z) scan order; torch.minimum splits it in half between equal
# arguments; relu passes nothing at 0.
# ---------------------------------------------------------------------------
def _pool_windows(t: np.ndarray, rad: int, periodic: bool, pad_val: float):
    """All (2 rad + 1)^d shifted views of t (d = t.ndim) in scan order, each
    paired with the flat source index of every window element (-1 = padding)."""
    d = t.ndim
    n = t.shape
    idx = np.arange(t.size).reshape(n)
    if periodic:
        tp = np.pad(t, rad, mode="wrap")
        ip = np.pad(idx, rad, mode="wrap")
    else:
        tp = np.pad(t, rad, mode="constant", constant_values=pad_val)
        ip = np.pad(idx, rad, mode="constant", constant_values=-1)
    vals, srcs = [], []
    import itertools
    for off in itertools.product(range(2 * rad + 1), repeat=d):
        sl = tuple(slice(o, o + n[k]) for k, o in enumerate(off))
        vals.append(tp[sl])
        srcs.append(ip[sl])
    return np.stack(vals), np.stack(srcs)


def max_pool(t: np.ndarray, rad: int, periodic: bool, pad_val: float = 0.0):
    """(pooled, argmax source index) of a (2 rad+1)^d max pool over a padded
    field: the first maximum in scan order wins (-1 if it is a pad cell)."""
    if rad <= 0:
        return t.copy(), np.arange(t.size).reshape(t.shape)
    vals, srcs = _pool_windows(t, rad, periodic, pad_val)
    k = np.argmax(vals, axis=0)
    pooled = np.take_along_axis(vals, k[None], 0)[0]
    src = np.take_along_axis(srcs, k[None], 0)[0]
    return pooled, src


def _pool_adjoint(g: np.ndarray, src: np.ndarray, size: int) -> np.ndarray:
    out = np.zeros(size)
    m = src.reshape(-1) >= 0
    np.add.at(out, src.reshape(-1)[m], g.reshape(-1)[m])
    return out


def _minimum_grads(a, b, g):
    """Gradients of torch.minimum(a, b) for upstream g (ties split in half)."""
    ga = np.where(a == b, g / 2, g) * (a <= b)
    gb = np.where(a == b, g / 2, g) * (b <= a)
    return ga, gb


def support_radius(overhang_deg: float) -> int:
    """Lateral support radius per layer for an overhang angle from the plate
    (utils/printability.py:76-90): ceil(tan(90 - deg)), at least 1."""
    od = float(np.clip(overhang_deg, 1.0, 89.0))
    return max(1, int(np.ceil(float(np.tan(np.deg2rad(90.0 - od))))))


def overhang_penalty(rho: np.ndarray, r: int, overhang_deg: float = 45.0, periodic_xy: bool = True):
    """(P, dP/drho) of printability_penalty_overhang (utils/printability.py:
    91-134): build direction +z; support(0) = rho(:,:,0); per layer z
    s = maxpool_xy(support(z-1)), P += mean(relu(rho_z - s)),
    support(z) = min(rho_z, s); P /= r - 1."""
    g = rho.reshape(r, r, r)
    rad = support_radius(overhang_deg)
    sup = g[:, :, 0].copy()
    tape = []
    P = 0.0
    for z in range(1, r):
        s, src = max_pool(sup, rad, periodic_xy, 0.0)
        rz = g[:, :, z]
        P += np.maximum(rz - s, 0.0).mean()
        tape.append((s, src, rz))
        sup = np.minimum(rz, s)
    den = max(r - 1, 1)
    P /= den
    grad = np.zeros((r, r, r))
    gsup = np.zeros((r, r))  # gradient arriving at support(z)
    for z in range(r - 1, 0, -1):
        s, src, rz = tape[z - 1]
        grz, gs = _minimum_grads(rz, s, gsup)
        act = (rz - s) > 0
        grz = grz + act / (r * r) / den
        gs = gs - act / (r * r) / den
        grad[:, :, z] += grz
        gsup = _pool_adjoint(gs, src, r * r).reshape(r, r)
    grad[:, :, 0] += gsup
    return P, grad.reshape(-1)


SEED_FACES = ("all", "x", "y", "z", "xy")


def _seed_mask(shape, seed_faces: str) -> np.ndarray:
    sf = str(seed_faces).lower()
    if sf not in SEED_FACES:
        raise ValueError("seed_faces must be one of: all, x, y, z, xy")
    seed = np.zeros(shape)
    if sf in ("all", "x"):
        seed[0], seed[-1] = 1, 1
    if sf in ("all", "y"):
        seed[:, 0], seed[:, -1] = 1, 1
    if sf in ("all", "z", "xy"):
        seed[:, :, 0], seed[:, :, -1] = 1, 1
    return seed


def _cavity(void: np.ndarray, periodic: bool, min_channel_rad: int, rad: int, nsteps: int, seed_faces: str):
    """Trapped-void field relu(void - reach) of the flood fill (utils/
    printability.py:199-220, 293-314) and a backward closure mapping its
    upstream gradient to d/dvoid."""
    shape = void.shape
    size = void.size
    if min_channel_rad > 0:
        er_neg, er_src = max_pool(-void, min_channel_rad, periodic, -1.0)  # erosion = -maxpool(-x), pad 1
        er = -er_neg
        vconn, di_src = max_pool(er, min_channel_rad, periodic, 0.0)       # dilation, pad 0
    else:
        vconn = void
    seed = _seed_mask(shape, seed_faces)
    reach = vconn * seed
    steps = []
    if rad > 0:
        for _ in range(nsteps):
            dil, src = max_pool(reach, rad, periodic, 0.0)
            steps.append((dil, src))
            reach = np.minimum(vconn, dil)
    trapped = np.maximum(void - reach, 0.0)

    def backward(gt: np.ndarray) -> np.ndarray:
        act = (void - reach) > 0
        gvoid = gt * act
        greach = -gt * act
        gvconn = np.zeros(shape)
        for dil, src in reversed(steps):
            gv, gd = _minimum_grads(vconn, dil, greach)
            gvconn += gv
            greach = _pool_adjoint(gd, src, size).reshape(shape)
        gvconn += greach * seed
        if min_channel_rad > 0:
            ger = _pool_adjoint(gvconn, di_src, size).reshape(shape)
            gvoid += _pool_adjoint(ger, er_src, size).reshape(shape)   # d(-maxpool(-x)) routes +g to the argmin
        else:
            gvoid += gvconn
        return gvoid

    return trapped, backward


def cavity_penalty(rho: np.ndarray, r: int, *, void_thresh: float = 0.5, beta: float = 20.0, min_channel_rad: int = 0,
                   rad: int = 1, iters: int = 0, tiles=(1, 1, 1), focus_center: bool = True,
                   seed_faces: str = "all", periodic: bool | None = None):
    """(P, dP/drho) of cavity_penalty_closed_void (tiles (1,1,1); periodic
    flood fill unless periodic=False; utils/printability.py:139-220) or
    cavity_penalty_periodic_array (tiles > 1: the cell tiled into a supercell
    whose boundary is the only outside, never periodic; :226-323)."""
    g = rho.reshape(r, r, r)
    tx, ty, tz = (max(1, int(t)) for t in tiles)
    array = max(tx, ty, tz) > 1
    periodic = (not array) if periodic is None else (bool(periodic) and not array)
    s = 1.0 / (1.0 + np.exp(-float(beta) * (float(void_thresh) - g)))
    void = np.tile(s, (tx, ty, tz)) if array else s
    nsteps = int(iters) if int(iters) > 0 else (max(void.shape) if array else r)
    trapped, backward = _cavity(void, periodic, int(max(0, min_channel_rad)), int(max(0, rad)), nsteps, seed_faces)
    if array and focus_center and tx >= 3 and ty >= 3 and tz >= 3:
        cx, cy, cz = tx // 2, ty // 2, tz // 2
        sl = (slice(cx * r, (cx + 1) * r), slice(cy * r, (cy + 1) * r), slice(cz * r, (cz + 1) * r))
        P = trapped[sl].mean()
        gt = np.zeros(trapped.shape)
        gt[sl] = 1.0 / (r ** 3)
    else:
        P = trapped.mean()
        gt = np.full(trapped.shape, 1.0 / trapped.size)
    gvoid = backward(gt)
    if array:
        gvoid = gvoid.reshape(tx, r, ty, r, tz, r).sum(axis=(0, 2, 4))
    grad = gvoid * (-float(beta)) * s * (1.0 - s)
    return float(P), grad.reshape(-1)
