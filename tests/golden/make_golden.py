"""Generate golden vectors by running the reference implementation (xing-yuu/MAPLE).

Run in a container where the reference source tree is available:

    python tests/golden/make_golden.py /path/to/MAPLE/src [--only=<part>]

It imports the reference package, runs its own functions in FP64 and writes
``tests/golden/*.npz``.  Nothing at test time reads the reference tree: the
tests only read the committed .npz files.

What is recorded (all FP64):
  * element tables: ``hexahedron(r, isotropic_elastic_tensor(1,0.3).double())``
    and ``hexahedron_scalar(r, kappa=float64 1.0)`` (utils/_utils.py:39-196);
  * RHS assembly ``assemble_F_fast`` / ``assemble_F_fast_scalar``;
  * converged homogenization: ``GMGSolver.solve`` / ``GMGSolverScalar.solve``
    with ``dtype=torch.float64`` and enough V-cycles for relres ~1e-14, then the
    energy sums of ``IHD.homogenized_batch_3d`` / ``homogenized_batch_thermal``
    (utils/model.py:33-95);
  * dJ/dx by ``torch.autograd.grad`` through those converged solves
    (main_IHD_v3.py:620-688), for two objective specs;
  * ``avg_filter3d_x_periodic`` and ``oc_update`` on seeded inputs;
  * objective values and their autograd gradients w.r.t. C^H / kappa;
  * a 3-iteration OC trajectory at 8^3 built from the reference's own pieces.
"""
from __future__ import annotations

import json
import os
import sys
import types

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))


def _import_reference(src):
    sys.path.insert(0, src)
    # main_IHD_v3 imports skimage for mesh export only; it is never called here
    sk = types.ModuleType("skimage")
    sk.measure = types.ModuleType("skimage.measure")
    sys.modules.setdefault("skimage", sk)
    sys.modules.setdefault("skimage.measure", sk.measure)
    from maple.core import main_IHD_v3 as M
    from maple.core.utils import _utils as U
    from maple.core.utils import model as Mo
    from maple.core.utils import objective as Ob
    from maple.core.utils.EBE_GMG import GMGSolver
    from maple.core.utils.EBE_GMG_scalar import GMGSolverScalar
    return M, U, Mo, Ob, GMGSolver, GMGSolverScalar


def seed_density(seed, r, sigma, vf, scale=0.25, xmin=1e-3):
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


def main(src, only=None):
    global SRC
    SRC = src
    M, U, Mo, Ob, GMGSolver, GMGSolverScalar = _import_reference(src)
    # torch's default dtype stays float32: the reference's
    # isotropic_elastic_tensor (utils/_utils.py:42) relies on it
    dev = torch.device("cpu")
    ihd = Mo.IHD.__new__(Mo.IHD)
    torch.nn.Module.__init__(ihd)

    def tables(r):
        C = U.isotropic_elastic_tensor(1.0, 0.3).double()
        Ke, Fe, X0 = U.hexahedron(r, C)
        K1, F1, X1 = U.hexahedron_scalar(r, kappa=torch.tensor(1.0, dtype=torch.float64))
        return Ke, Fe, X0, K1, F1, X1

    def homogenize(r, rho, cycles, levels=3, want_u=False):
        """Reference forward in FP64 (differentiable w.r.t. rho)."""
        Ke, Fe, X0, K1, F1, X1 = tables(r)
        batch = M.build_unitcell_batch(dev, r, rho.detach().reshape(r, r, r))
        rr = rho.reshape(-1, 1)
        n = r ** 3
        out = {}
        # elastic (utils/model.py:98-130 with dtype float64)
        F = U.assemble_F_fast(batch["node_index"], Fe, n, rr)
        Ke_ = Ke.unsqueeze(0).expand(n, -1, -1) * rr.reshape(-1, 1, 1)
        us, res = [], []
        g = GMGSolver()
        for i in range(6):
            u, rv = g.solve(Ke_, F[:, :, i], batch["coord"].int(), batch["elem_coords"], batch["node_index"],
                            max_iter=cycles, smooth_iter=[2, 2, 3, 4, 5], max_levels=levels, dtype=torch.float64)
            us.append(u)
            res.append((rv.norm() / F[:, :, i].norm()).item())
        Uel = torch.cat(us, 1)
        out["CH"] = ihd.homogenized_batch_3d(Uel, Ke_, X0, batch["coord"][:, 0], batch["node_index"],
                                             batch["voxel_batch_id"], 1)[0]
        out["relres_elastic"] = np.array(res)
        # thermal (utils/model.py:131-159 with dtype float64)
        Ft = U.assemble_F_fast_scalar(batch["node_index"], F1, n, rr)
        K1_ = K1.unsqueeze(0).expand(n, -1, -1) * rr.reshape(-1, 1, 1)
        gs = GMGSolverScalar()
        ut, res = [], []
        for i in range(3):
            u, rv = gs.solve(K1_, Ft[:, i], batch["coord"].int(), batch["elem_coords"], batch["node_index"],
                             max_iter=cycles, smooth_iter=[2, 2, 3, 4, 5], max_levels=levels, dtype=torch.float64)
            ut.append(u)
            res.append((rv.norm() / Ft[:, i].norm()).item())
        Uth = torch.cat(ut, 1)
        out["kappa"] = ihd.homogenized_batch_thermal(Uth, K1_, X1, batch["coord"][:, 0], batch["node_index"],
                                                     batch["voxel_batch_id"], 1)[0]
        out["relres_thermal"] = np.array(res)
        if want_u:
            out["u_elastic"] = Uel.detach().numpy().reshape(n, 6, 3).transpose(0, 2, 1).copy()  # (N,3,6)
            out["u_thermal"] = Uth.detach().numpy()
            out["F_elastic"] = F.detach().numpy()
            out["F_thermal"] = Ft.detach().numpy()
        return out

    if only == "config0":
        return config0_fixtures(Ob, homogenize)
    if only == "config0pins":
        return config0_pins()
    if only == "config1":
        return config1_fixtures(Ob, homogenize)
    if only == "symmetry":
        return symmetry_fixtures(M, Ob, homogenize, dev)
    if only == "generator":
        return generator_fixtures()
    if only == "print":
        return printability_fixtures(M, Ob, homogenize, dev, src)

    rec = {}
    # ---------------------------------------------------------------- tables
    for r in (8, 16, 32):
        Ke, Fe, X0, K1, F1, X1 = tables(r)
        for k, v in dict(Ke3=Ke, Fe3=Fe, X03=X0, Ke1=K1, Fe1=F1, X01=X1).items():
            rec[f"r{r}_{k}"] = v.numpy()
    np.savez_compressed(os.path.join(HERE, "element_tables.npz"), **rec)

    # ------------------------------------------------- converged homogenization
    specs = {"bi": "stiffness:0.5,thermal:0.5", "tri": "stiffness:0.3333333333333333,shear:0.3333333333333333,"
                                                       "thermal:0.3333333333333333"}
    cases = [(8, 0, 2.0, 0.25), (8, 1, 1.0, 0.30), (16, 0, 2.0, 0.25)]
    for (r, seed, sigma, vf) in cases:
        x = seed_density(seed, r, sigma, vf)
        rec = dict(x=x.reshape(-1), r=r, seed=seed, sigma=sigma, vf=vf)
        penal, rho_min = 3.0, 1e-9
        # the reference's coarsest level is only smoothed, so deeper hierarchies
        # are needed for a converged FP64 solve at 16^3
        cycles, levels = (60, 3) if r == 8 else (70, 5)
        xt = torch.tensor(x.reshape(-1, 1))
        rho = rho_min + (1 - rho_min) * xt ** penal
        out = homogenize(r, rho, cycles, levels=levels, want_u=(r == 8))
        for k, v in out.items():
            rec[k] = v.detach().numpy() if torch.is_tensor(v) else v
        if r == 8:
            # dJ/dx by autograd through the converged solves (main_IHD_v3.py:622-688)
            for tag, spec in specs.items():
                xv = xt.clone().requires_grad_(True)
                xc = xv.clamp(1e-3, 1.0)
                rv = rho_min + (1 - rho_min) * xc ** penal
                o = homogenize(r, rv, cycles, levels=3)
                J = Ob.objective_from_spec(obj=spec, CH=o["CH"], kappa=o["kappa"])
                (g,) = torch.autograd.grad(J, xv)
                rec[f"J_{tag}"] = J.item()
                rec[f"dJdx_{tag}"] = g.numpy().reshape(-1)
        name = f"homog_r{r}_s{seed}.npz"
        np.savez_compressed(os.path.join(HERE, name), **rec)
        print("wrote", name, "relres", out["relres_elastic"].max(), out["relres_thermal"].max())

    # ------------------------------------------------ filter / OC / objectives
    rng = np.random.default_rng(7)
    rec = {}
    for r in (6, 8):
        n = r ** 3
        v = rng.standard_normal(n)
        batch = M.build_unitcell_batch(dev, r, torch.zeros(r, r, r))
        for k in (1, 3, 5):
            rec[f"filter_r{r}_k{k}_in"] = v
            rec[f"filter_r{r}_k{k}_out"] = M.avg_filter3d_x_periodic(torch.tensor(v).reshape(-1, 1),
                                                                       batch["elem_coords"], r, k).numpy().reshape(-1)
    for i, (vf, move, xmin) in enumerate([(0.25, 0.2, 1e-3), (0.1, 0.05, 1e-5), (0.4, 0.2, 1e-3)]):
        n = 512
        x = np.clip(vf + 0.2 * rng.standard_normal(n), xmin, 1.0)
        dJ = np.abs(rng.standard_normal(n)) * 1e-2
        dJ[:5] = -1.0  # negative sensitivities are clamped to 1e-12
        xn = M.oc_update(torch.tensor(x).reshape(-1, 1), torch.tensor(dJ).reshape(-1, 1), volfrac=vf, move=move,
                         xmin=xmin).numpy().reshape(-1)
        rec.update({f"oc{i}_x": x, f"oc{i}_dJ": dJ, f"oc{i}_xnew": xn, f"oc{i}_params": np.array([vf, move, xmin])})
    for i in range(3):
        A = rng.standard_normal((6, 6)) * 0.05
        CH = torch.tensor(A @ A.T + np.eye(6) * (0.1 + 0.1 * i) + 0.01 * rng.standard_normal((6, 6)),
                          requires_grad=True)
        kap = torch.tensor(np.diag(rng.uniform(0.05, 0.3, 3)) + 0.01, requires_grad=True)
        for tag, spec in dict(stiff="stiffness", shear="shear", therm="thermal", bi=specs["bi"],
                              tri=specs["tri"], mixw="0.4*stiffness+0.6*thermal").items():
            J = Ob.objective_from_spec(obj=spec, CH=CH, kappa=kap)
            gC, gK = torch.autograd.grad(J, (CH, kap), allow_unused=True)
            rec[f"obj{i}_{tag}_J"] = J.item()
            rec[f"obj{i}_{tag}_gC"] = gC.numpy() if gC is not None else np.zeros((6, 6))
            rec[f"obj{i}_{tag}_gK"] = gK.numpy() if gK is not None else np.zeros((3, 3))
        rec[f"obj{i}_CH"] = CH.detach().numpy()
        rec[f"obj{i}_kappa"] = kap.detach().numpy()
    for spec in ["stiffness", "0.4*stiffness+0.6*thermal", "shear=0.3+thermal=0.7", "stiffness,thermal",
                 "E:0.5,kappa:0.5", " Shear "]:
        rec["spec::" + spec] = np.array(sorted(Ob.parse_objective_spec(spec).items()), dtype=object).astype(str)
    np.savez_compressed(os.path.join(HERE, "ops.npz"), **rec)

    # ------------------------------------------------------ short OC trajectory
    r, vf, move, xmin, penal, rho_min, fk = 8, 0.25, 0.2, 1e-3, 3.0, 1e-9, 3
    x = torch.tensor(seed_density(0, r, 2.0, vf).reshape(-1, 1))
    batch = M.build_unitcell_batch(dev, r, torch.zeros(r, r, r))
    traj = dict(x0=x.numpy().reshape(-1))
    for it in range(3):
        xv = x.detach().clone().requires_grad_(True)
        rv = rho_min + (1 - rho_min) * xv.clamp(xmin, 1.0) ** penal
        o = homogenize(r, rv, 60, levels=3)
        J = Ob.objective_from_spec(obj=specs["bi"], CH=o["CH"], kappa=o["kappa"])
        (g,) = torch.autograd.grad(J, xv)
        g = M.avg_filter3d_x_periodic(g, batch["elem_coords"], r, fk)
        xn = M.oc_update(x.detach(), g.detach(), volfrac=vf, move=move, xmin=xmin).clamp(xmin, 1.0)
        traj[f"J{it}"] = J.item()
        traj[f"x{it + 1}"] = xn.numpy().reshape(-1)
        x = xn
        print("traj it", it, "J", J.item())
    np.savez_compressed(os.path.join(HERE, "traj_r8.npz"), **traj)


def _oracle():
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from oracle import ihd_oracle as O
    return O


def _reference_terms(Ob, homogenize, r, x, spec, cycles, levels, penal=3.0, rho_min=1e-9, xmin=1e-3):
    """C^H, kappa^H and J of design x by the reference's own FP64 solvers."""
    xt = torch.tensor(np.clip(x, xmin, 1.0).reshape(-1, 1))
    rho = rho_min + (1 - rho_min) * xt ** penal
    o = homogenize(r, rho, cycles, levels=levels)
    J = Ob.objective_from_spec(obj=spec, CH=o["CH"], kappa=o["kappa"])
    return (o["CH"].detach().numpy(), o["kappa"].detach().numpy(), float(J),
            float(max(o["relres_elastic"].max(), o["relres_thermal"].max())))


def config0_fixtures(Ob, homogenize):
    """traj_r32.npz: the plain FP64 method of the 32^3 benchmark configuration
    (seed 0, sigma 2, vf 0.25, J = 0.5 E + 0.5 kappa, move 0.2, 3^3 filter,
    50 OC iterations).  The oracle runs the 50 iterations with its solves
    converged to a relative residual of 1e-12 (warm-started from the previous
    iteration; the converged answer is independent of the start); every
    iteration's J, C^H, kappa^H and |dx| statistics and the designs at
    iterations 1, 10, 25, 49 and 50 are stored, with each iteration's oracle
    residual.  The oracle's solves are its V-cycle in symmetric form used as
    the preconditioner of CG: the reference's plain V-cycle iteration stalls
    near a relative residual of 2e-7 from iteration 41 on (the design then
    holds near-void regions), and so does a flexible CG preconditioned by the
    non-symmetric cycle (3e-8 to 8e-8 after 400 iterations at iterations 42 and
    43); the symmetric one reaches 1e-12 at every iteration.  config0_pins then
    pins the trajectory with the reference's own solvers."""
    import time
    O = _oracle()
    r, vf, spec = 32, 0.25, "stiffness:0.5,thermal:0.5"
    w = O.parse_objective_spec(spec)
    x = O.seed_density(0, r, 2.0, vf).reshape(-1)
    el = O.Elements(r)
    rec = dict(r=r, seed=0, sigma=2.0, vf=vf, move=0.2, filter_k=3, penal=3.0, rho_min=1e-9, xmin=1e-3,
               iters=50, oracle_rtol=1e-12, x0=x.copy())
    Js, CHs, Ks, dmax, dmean, xs, relres = [], [], [], [], [], {}, []
    prev = None
    t0 = time.time()
    for it in range(50):
        if it in (1, 10, 25, 49):
            xs[it] = x.copy()
        xn, info = O.oc_iteration(x, r, w, volfrac=vf, move=0.2, elems=el, levels=5, rtol=1e-12,
                                  max_cycles=2000, u0=prev, method="pcg")
        prev = info["res"]
        Js.append(info["J"])
        CHs.append(info["CH"])
        Ks.append(info["kappa"])
        dmax.append(info["dx_max"])
        dmean.append(info["dx_mean"])
        relres.append(max(prev["relres_elastic"].max(), prev["relres_thermal"].max()))
        print(f"config0 oracle it {it} J {info['J']:.15g} cycles {prev['cycles_elastic']} {prev['cycles_thermal']} "
              f"relres {relres[-1]:.2e} t {time.time() - t0:.0f}s", flush=True)
        x = xn
    rec.update(J=np.array(Js), CH=np.array(CHs), kappa=np.array(Ks), dx_max=np.array(dmax), dx_mean=np.array(dmean),
               oracle_relres=np.array(relres), x50=x.copy())
    for it, xv in xs.items():
        rec[f"x{it}"] = xv
    np.savez_compressed(os.path.join(HERE, "traj_r32.npz"), **rec)
    print("wrote traj_r32.npz (oracle trajectory)")
    config0_pins()


def _oracle_fields(O, r, x, spec, el, levels):
    """The oracle's converged solutions (rtol 1e-12) of design x, as the
    reference's node fields: elastic (N, 3, 6), thermal (N, 3)."""
    rho = 1e-9 + (1 - 1e-9) * np.clip(x, 1e-3, 1.0) ** 3
    res = O.solve_cell(rho, r, el, levels, 1000, 1e-12, ("elastic", "thermal"), method="pcg")
    N = r ** 3
    return res["u3"].reshape(N, 3, 6), res["u1"].reshape(N, 3), res


def _pin_jobs(O, r, spec, xs, levels):
    el = O.Elements(r)
    jobs = []
    for x in xs:
        u3, u1, _ = _oracle_fields(O, r, x, spec, el, levels)
        jobs.append((SRC, spec, r, x, u3, u1, levels))
    return jobs


def config0_pins():
    """The reference's pins of the 32^3 trajectory: at the oracle's designs of
    iterations 0, 1, 10, 25 and 49 the reference's own solvers
    (GMGSolver.solve / GMGSolverScalar.solve in FP64) are started from the
    oracle's converged fields through their init_list hook (sparse tensors
    aligned by node coordinates, EBE_GMG.py:648-757) and run 5 V-cycles; the
    reference's residual of its own operator then says whether the oracle's
    field solves the reference's system (the solution is unique up to a
    rigid translation), and its energy sums give C^H, kappa^H and J."""
    O = _oracle()
    path = os.path.join(HERE, "traj_r32.npz")
    rec = dict(np.load(path, allow_pickle=True))
    r, spec = int(rec["r"]), "stiffness:0.5,thermal:0.5"
    its = (0, 1, 10, 25, 49)
    jobs = _pin_jobs(O, r, spec, [rec["x0"] if it == 0 else rec[f"x{it}"] for it in its], 5)
    import multiprocessing as mp
    with mp.get_context("spawn").Pool(len(jobs)) as pool:
        outs = pool.map(_reference_job, jobs)
    for it, (CH, kap, J, rr) in zip(its, outs):
        rec[f"ref_CH_{it}"], rec[f"ref_kappa_{it}"], rec[f"ref_J_{it}"], rec[f"ref_relres_{it}"] = CH, kap, J, rr
        print(f"config0 reference it {it} J {J:.15g} (oracle {float(rec['J'][it]):.15g}) relres {rr:.2e}",
              flush=True)
    np.savez_compressed(path, **rec)
    print("wrote traj_r32.npz")


SRC = None  # the reference source tree of this run (set by main)


def _reference_job(args):
    """One reference evaluation in a fresh process (spawned): C^H, kappa^H, J
    and the relative residual of design x, the reference's solvers started from
    the given fields (u3 (N, 3, 6), u1 (N, 3)) through init_list."""
    import types
    src, spec, r, x, u3, u1, levels = args
    cycles = 5
    torch.set_num_threads(1)
    M, U, Mo, Ob, GMGSolver, GMGSolverScalar = _import_reference(src)
    dev = torch.device("cpu")
    ihd = Mo.IHD.__new__(Mo.IHD)
    torch.nn.Module.__init__(ihd)

    def homogenize(r_, rho, cycles_, levels=3):
        C = U.isotropic_elastic_tensor(1.0, 0.3).double()
        Ke, Fe, X0 = U.hexahedron(r_, C)
        K1, F1, X1 = U.hexahedron_scalar(r_, kappa=torch.tensor(1.0, dtype=torch.float64))
        batch = M.build_unitcell_batch(dev, r_, rho.detach().reshape(r_, r_, r_))
        rr = rho.reshape(-1, 1)
        n = r_ ** 3
        out = {}
        F = U.assemble_F_fast(batch["node_index"], Fe, n, rr)
        Ke_ = Ke.unsqueeze(0).expand(n, -1, -1) * rr.reshape(-1, 1, 1)
        idx = batch["coord"].long()

        def init(field):  # the reference's sparse-tensor hook: indices [b,x,y,z], features
            return [types.SimpleNamespace(indices=idx, features=torch.tensor(field, dtype=torch.float64))]

        us, res = [], []
        for i in range(6):
            u, rv = GMGSolver().solve(Ke_, F[:, :, i], batch["coord"].int(), batch["elem_coords"], batch["node_index"],
                                      max_iter=cycles_, smooth_iter=[2, 2, 3, 4, 5], max_levels=levels,
                                      init_list=init(u3[:, :, i]), dtype=torch.float64)
            us.append(u)
            res.append((rv.norm() / F[:, :, i].norm()).item())
        out["CH"] = ihd.homogenized_batch_3d(torch.cat(us, 1), Ke_, X0, batch["coord"][:, 0], batch["node_index"],
                                             batch["voxel_batch_id"], 1)[0]
        out["relres_elastic"] = np.array(res)
        Ft = U.assemble_F_fast_scalar(batch["node_index"], F1, n, rr)
        K1_ = K1.unsqueeze(0).expand(n, -1, -1) * rr.reshape(-1, 1, 1)
        ut, res = [], []
        for i in range(3):
            u, rv = GMGSolverScalar().solve(K1_, Ft[:, i], batch["coord"].int(), batch["elem_coords"],
                                            batch["node_index"], max_iter=cycles_, smooth_iter=[2, 2, 3, 4, 5],
                                            max_levels=levels, init_list=init(u1[:, i:i + 1]),
                                            dtype=torch.float64)
            ut.append(u)
            res.append((rv.norm() / Ft[:, i].norm()).item())
        out["kappa"] = ihd.homogenized_batch_thermal(torch.cat(ut, 1), K1_, X1, batch["coord"][:, 0],
                                                     batch["node_index"], batch["voxel_batch_id"], 1)[0]
        out["relres_thermal"] = np.array(res)
        return out

    return _reference_terms(Ob, homogenize, r, x, spec, cycles, levels)


def config1_fixtures(Ob, homogenize):
    """spot_r64.npz: the 64^3 precision configuration (seed 0, sigma 4,
    vf 0.25, J = (E + G + kappa)/3).  The oracle runs OC iteration 0 from the
    seeded design (solves to a relative residual of 1e-12) and evaluates
    iteration 1's design; the reference's own FP64 GMG solvers evaluate C^H,
    kappa^H and J at both designs."""
    import time
    O = _oracle()
    r, vf = 64, 0.25
    spec = "stiffness:0.3333333333333333,shear:0.3333333333333333,thermal:0.3333333333333333"
    w = O.parse_objective_spec(spec)
    x0 = O.seed_density(0, r, 4.0, vf).reshape(-1)
    el = O.Elements(r)
    t0 = time.time()
    x1, info0 = O.oc_iteration(x0, r, w, volfrac=vf, move=0.2, elems=el, levels=6, rtol=1e-12, max_cycles=400)
    print(f"config1 oracle it 0 J {info0['J']:.15g} t {time.time() - t0:.0f}s", flush=True)
    _, info1 = O.oc_iteration(x1, r, w, volfrac=vf, move=0.2, elems=el, levels=6, rtol=1e-12, max_cycles=400,
                              u0=info0["res"])
    print(f"config1 oracle it 1 J {info1['J']:.15g} t {time.time() - t0:.0f}s", flush=True)
    rec = dict(r=r, seed=0, sigma=4.0, vf=vf, move=0.2, filter_k=3, penal=3.0, rho_min=1e-9, xmin=1e-3,
               oracle_rtol=1e-12, x1=x1,
               J=np.array([info0["J"], info1["J"]]), CH=np.array([info0["CH"], info1["CH"]]),
               kappa=np.array([info0["kappa"], info1["kappa"]]))
    for it, xv in ((0, x0), (1, x1)):
        CH, kap, J, rr = _reference_terms(Ob, homogenize, r, xv, spec, cycles=90, levels=6)
        rec[f"ref_CH_{it}"], rec[f"ref_kappa_{it}"], rec[f"ref_J_{it}"], rec[f"ref_relres_{it}"] = CH, kap, J, rr
        print(f"config1 reference it {it} J {J:.15g} relres {rr:.2e} t {time.time() - t0:.0f}s", flush=True)
    np.savez_compressed(os.path.join(HERE, "spot_r64.npz"), **rec)
    print("wrote spot_r64.npz")


def printability_fixtures(M, Ob, homogenize, dev, src):
    """print.npz: the reference's printability / cavity penalties
    (utils/printability.py) and their autograd gradients w.r.t. rho on two 8^3
    fields (one continuous, one clipped SIMP design full of exact ties), and a
    3-iteration OC trajectory with both penalties (lambda 0.9 each, the
    experiment scripts' values) from the reference's own pieces."""
    from maple.core.utils import printability as Pr
    r = 8
    rng = np.random.default_rng(21)
    fields = {
        "cont": rng.random(r ** 3),
        "simp": 1e-9 + (1 - 1e-9) * np.clip(seed_density(3, r, 1.5, 0.3) + 0.3 * rng.standard_normal(r ** 3)
                                             .reshape(r, r, r), 1e-3, 1.0).reshape(-1) ** 3,
    }
    rec = {}
    cases = []
    for deg in (45.0, 20.0):
        for per in (True, False):
            cases.append(("over", dict(overhang_deg=deg, periodic_xy=per)))
    closed = [dict(), dict(min_channel_rad=1), dict(rad=0), dict(rad=2, iters=3), dict(seed_faces="x"),
              dict(seed_faces="xy", void_thresh=0.3, beta=10.0), dict(periodic_xyz=False, min_channel_rad=1)]
    for kw in closed:
        cases.append(("closed", kw))
    arrays = [dict(tiles_xyz=(2, 2, 2), min_channel_rad=1), dict(tiles_xyz=(2, 2, 2), min_channel_rad=3),
              dict(tiles_xyz=(3, 3, 3), focus_center=True), dict(tiles_xyz=(3, 3, 3), focus_center=False, iters=5),
              dict(tiles_xyz=(2, 1, 3), seed_faces="z")]
    for kw in arrays:
        cases.append(("array", kw))
    for fname, f in fields.items():
        rec[f"field_{fname}"] = f
        for i, (kind, kw) in enumerate(cases):
            rho = torch.tensor(f.reshape(r, r, r), requires_grad=True)
            if kind == "over":
                P = Pr.printability_penalty_overhang(rho, **kw)
            elif kind == "closed":
                P = Pr.cavity_penalty_closed_void(rho, **kw)
            else:
                P = Pr.cavity_penalty_periodic_array(rho, **kw)
            (gr,) = torch.autograd.grad(P, rho)
            rec[f"{fname}_{i}_P"] = P.item()
            rec[f"{fname}_{i}_grad"] = gr.numpy().reshape(-1)
    rec["cases"] = np.array([json.dumps([k, kw]) for k, kw in cases])
    # OC trajectory with both penalties (main_IHD_v3.py:649-688)
    vf, move, xmin, penal, rho_min, fk = 0.25, 0.2, 1e-3, 3.0, 1e-9, 3
    lp, lc = 0.9, 0.9
    spec_obj = "stiffness:0.5,thermal:0.5"
    batch = M.build_unitcell_batch(dev, r, torch.zeros(r, r, r))
    ec = batch["elem_coords"]
    x = torch.tensor(seed_density(0, r, 2.0, vf).reshape(-1, 1))
    rec["traj_x0"] = x.numpy().reshape(-1)
    for it in range(3):
        xv = x.detach().clone().requires_grad_(True)
        rv = rho_min + (1 - rho_min) * xv.clamp(xmin, 1.0) ** penal
        o = homogenize(r, rv, 60, levels=3)
        J_raw = Ob.objective_from_spec(obj=spec_obj, CH=o["CH"], kappa=o["kappa"])
        grid = rv.reshape(r, r, r)
        Pp = Pr.printability_penalty_overhang(grid, overhang_deg=45.0, periodic_xy=True)
        Pc = Pr.cavity_penalty_periodic_array(grid, tiles_xyz=(2, 2, 2), focus_center=True, void_thresh=0.5,
                                              beta=20.0, min_channel_rad=1, rad=1, iters=0, seed_faces="all")
        J = J_raw - lp * Pp - lc * Pc
        (g,) = torch.autograd.grad(J, xv)
        g = M.avg_filter3d_x_periodic(g, ec, r, fk)
        xn = M.oc_update(x.detach(), g.detach(), volfrac=vf, move=move, xmin=xmin).clamp(xmin, 1.0)
        rec[f"traj_J{it}"] = J.item()
        rec[f"traj_Jraw{it}"] = J_raw.item()
        rec[f"traj_Pp{it}"] = Pp.item()
        rec[f"traj_Pc{it}"] = Pc.item()
        rec[f"traj_x{it + 1}"] = xn.numpy().reshape(-1)
        x = xn
        print("print traj", it, J.item(), Pp.item(), Pc.item())
    np.savez_compressed(os.path.join(HERE, "print.npz"), **rec)


def symmetry_fixtures(M, Ob, homogenize, dev):
    """sym.npz: parse_symmetry on several spellings, symmetrize_vec of a random
    8^3 field for each kind, and 3-iteration 8^3 OC trajectories with cubic and
    "xy" mirror symmetry built from the reference's own pieces
    (main_IHD_v3.py:620-716 with lambda_print = lambda_cavity = 0)."""
    rec = {}
    for spec in ["none", "", "x", "xy", "yz", "xz", "xyz", "octant", "1/8", "cubic", "iso", "isotropic", "z"]:
        kind, axes = M.parse_symmetry(spec)
        rec["parse::" + spec] = np.array([kind] + [str(a) for a in axes])
    r = 8
    batch = M.build_unitcell_batch(dev, r, torch.zeros(r, r, r))
    ec = batch["elem_coords"]
    v = torch.tensor(np.random.default_rng(11).standard_normal((r ** 3, 1)))
    rec["field"] = v.numpy().reshape(-1)
    for spec in ["x", "xy", "yz", "xyz", "cubic"]:
        kind, axes = M.parse_symmetry(spec)
        rec["sym::" + spec] = M.symmetrize_vec(v, ec, res=r, kind=kind, axes=axes).numpy().reshape(-1)
    vf, move, xmin, penal, rho_min, fk = 0.25, 0.2, 1e-3, 3.0, 1e-9, 3
    spec_obj = "stiffness:0.5,thermal:0.5"
    for spec in ["cubic", "xy"]:
        kind, axes = M.parse_symmetry(spec)
        x = torch.tensor(seed_density(0, r, 2.0, vf).reshape(-1, 1))
        x = M.symmetrize_vec(x, ec, res=r, kind=kind, axes=axes).clamp(xmin, 1.0)
        rec[f"traj_{spec}_x0"] = x.numpy().reshape(-1)
        for it in range(3):
            xv = x.detach().clone().requires_grad_(True)
            xu = M.symmetrize_vec(xv.clamp(xmin, 1.0), ec, res=r, kind=kind, axes=axes).clamp(xmin, 1.0)
            rv = rho_min + (1 - rho_min) * xu ** penal
            o = homogenize(r, rv, 60, levels=3)
            J = Ob.objective_from_spec(obj=spec_obj, CH=o["CH"], kappa=o["kappa"])
            (g,) = torch.autograd.grad(J, xv)
            g = M.avg_filter3d_x_periodic(g, ec, r, fk)
            xn = M.oc_update(x.detach(), g.detach(), volfrac=vf, move=move, xmin=xmin)
            xn = M.symmetrize_vec(xn, ec, res=r, kind=kind, axes=axes).clamp(xmin, 1.0)
            rec[f"traj_{spec}_J{it}"] = J.item()
            rec[f"traj_{spec}_x{it + 1}"] = xn.numpy().reshape(-1)
            x = xn
            print("sym traj", spec, it, J.item())
    np.savez_compressed(os.path.join(HERE, "sym.npz"), **rec)


GENERATOR_CONFIGS = {
    "full": dict(cond_dim=7, out_res=32, base_res=4, latent_dim=256, base_channels=128),
    "small": dict(cond_dim=7, out_res=16, base_res=4, latent_dim=64, base_channels=32),
}


def generator_fixtures():
    """Stage2DensityGenerator (core/stage2/density_generator.py:123-197) with
    seeded weights, and the Pareto worker's warm-start helpers
    (pareto/densify_pareto_property_network_32.py:1031-1052), run from the
    reference's own modules.  Densities are stored every 7th voxel plus
    per-sample FP64 sums and sums of squares of the full field."""
    from maple.core.stage2.density_generator import Stage2DensityGenerator
    from maple.pareto import densify_pareto_property_network_32 as D
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from oracle.generator_oracle import synthetic_state_dict
    rec = {}
    for tag, cfg in GENERATOR_CONFIGS.items():
        model = Stage2DensityGenerator(**cfg, use_noise_encoder=False)
        model.load_state_dict(synthetic_state_dict(seed=11, **cfg))  # strict: names and shapes agree
        model.eval()
        cond = np.random.default_rng(5).uniform(0.0, 1.0, (3, cfg["cond_dim"])).astype(np.float32)
        eta = np.array([0.25, 0.75], dtype=np.float32)
        with torch.no_grad():
            rho = model(torch.from_numpy(cond), None).numpy().reshape(3, -1)
            lat = model.encode_latent(torch.from_numpy(cond), None)
            mix = model.decode_latent(torch.sum(lat[:2] * torch.from_numpy(eta).reshape(-1, 1), dim=0,
                                                keepdim=True)).numpy().reshape(1, -1)
        rec[f"{tag}_cond"] = cond
        rec[f"{tag}_eta"] = eta
        rec[f"{tag}_latent"] = lat.numpy()
        for name, a in (("rho", rho), ("mix", mix)):
            rec[f"{tag}_{name}_sub"] = a[:, ::7].copy()
            rec[f"{tag}_{name}_sum"] = a.astype(np.float64).sum(1)
            rec[f"{tag}_{name}_sumsq"] = (a.astype(np.float64) ** 2).sum(1)
        print("generator", tag, rho.mean(), rho.min(), rho.max())
    vol = np.random.default_rng(9).uniform(-0.1, 1.1, (12, 12, 12)).astype(np.float32)
    rec["warm_in"] = vol
    for passes in (0, 1, 3):
        rec[f"smooth_{passes}"] = D.binomial_smooth_periodic_torch(torch.from_numpy(vol), passes).numpy()
    for i, (t, iters) in enumerate(((0.3, 8), (0.05, 1), (0.9, 20), (0.25, 0))):
        rec[f"match_{i}"] = D.match_mean_clamped_torch(torch.from_numpy(vol), t, 1e-5, iters).numpy()
        rec[f"match_{i}_args"] = np.array([t, iters], dtype=np.float64)
    rec["fieldnames"] = np.array(D.FIELDNAMES)
    rec["condition_columns"] = np.array(D.CONDITION_COLUMNS)
    np.savez_compressed(os.path.join(HERE, "generator.npz"), **rec)


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--only=")]
    only = next((a.split("=", 1)[1] for a in sys.argv[1:] if a.startswith("--only=")), None)
    if len(args) != 1:
        sys.exit("usage: python tests/golden/make_golden.py <reference src dir> [--only=config0|config1|print|"
                 "symmetry|generator]")
    main(args[0], only)
