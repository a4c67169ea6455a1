"""GPU parity of the sm_100a kernels against the FP64 oracle and the golden
vectors recorded from the reference (called through the C ABI)."""
import numpy as np
import pytest
import torch

from oracle import ihd_oracle as O

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


def T(a):
    return torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=DEV)


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def simp(x, p=3.0, rmin=1e-9):
    return rmin + (1 - rmin) * np.clip(x, 1e-3, 1.0) ** p


@pytest.fixture(scope="module")
def ctx8(lib):
    from maple_b200.core import HomogenizationContext
    c = HomogenizationContext(8, ncells=2)
    yield c
    c.close()


@pytest.fixture(scope="module")
def dens8(golden):
    g0, g1 = golden("homog_r8_s0.npz"), golden("homog_r8_s1.npz")
    return (g0, g1), np.stack([simp(g0["x"]), simp(g1["x"])])


def test_matvec_elastic_and_thermal(ctx8, dens8):
    _, rho = dens8
    r, N = 8, 512
    rng = np.random.default_rng(0)
    e = O.Elements(r)
    for phys, d, R, Ke0 in (("elastic", 3, 6, e.Ke3), ("thermal", 1, 3, e.Ke1)):
        u = rng.standard_normal((2, R, d, N))
        y = ctx8.matvec(phys, T(rho), T(u)).cpu().numpy()
        for b in range(2):
            K = O.assemble_K(rho[b].reshape(-1, 1, 1) * Ke0[None], r, d)
            umat = u[b].transpose(2, 1, 0).reshape(N * d, R)
            ref = (K @ umat).reshape(N, d, R).transpose(2, 1, 0)
            assert rel(y[b], ref) < 1e-13, (phys, b)


def test_assemble_rhs(ctx8, dens8):
    _, rho = dens8
    e = O.Elements(8)
    for phys, d, R, Fe in (("elastic", 3, 6, e.Fe3), ("thermal", 1, 3, e.Fe1)):
        F = ctx8.assemble_rhs(phys, T(rho)).cpu().numpy()
        for b in range(2):
            ref = O.assemble_F(rho[b], Fe, 8, d).reshape(512, d, R).transpose(2, 1, 0)
            assert rel(F[b], ref) < 1e-13


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-10), ("mixed", 1e-9)])
def test_homogenization_matches_reference(ctx8, dens8, precision, tol):
    (g0, g1), rho = dens8
    for phys, key in (("elastic", "CH"), ("thermal", "kappa")):
        ctx8.set_density(phys, T(rho), precision)
        info = ctx8.solve(phys, precision, rtol=1e-12, maxit=300)
        assert (info.status & 1).all(), info
        H = ctx8.homogenize(phys).cpu().numpy()
        assert rel(H[0], g0[key]) < tol, (phys, precision)
        assert rel(H[1], g1[key]) < tol, (phys, precision)


def test_solution_field_matches_reference(ctx8, dens8):
    (g0, _), rho = dens8
    ctx8.set_density("elastic", T(rho), "fp64")
    ctx8.solve("elastic", "fp64", rtol=1e-13, maxit=300)
    u = ctx8.solution("elastic").cpu().numpy()[0]          # (6, 3, N)
    ug = g0["u_elastic"].transpose(2, 1, 0)                 # (6, 3, N)
    du = (u - u.mean(-1, keepdims=True)) - (ug - ug.mean(-1, keepdims=True))
    assert np.abs(du).max() / np.abs(ug).max() < 1e-9


@pytest.mark.parametrize("tag,w", [("bi", (0.5, 0.0, 0.5)), ("tri", (1 / 3, 1 / 3, 1 / 3))])
def test_sensitivity_matches_autograd(ctx8, dens8, tag, w):
    (g0, g1), rho = dens8
    H = {}
    for phys in ("elastic", "thermal"):
        ctx8.set_density(phys, T(rho), "fp64")
        ctx8.solve(phys, "fp64", rtol=1e-13, maxit=300)
        H[phys] = ctx8.homogenize(phys).cpu().numpy()
    weights = {"stiffness": w[0], "shear": w[1], "thermal": w[2]}
    weights = {k: v for k, v in weights.items() if v}
    gC = np.zeros((2, 6, 6))
    gK = np.zeros((2, 3, 3))
    for b in range(2):
        _, gC[b], gK[b] = O.objective_and_grads(weights, H["elastic"][b], H["thermal"][b])
    dJdrho = ctx8.sensitivity(T(gC), T(gK)).cpu().numpy()
    for b, g in enumerate((g0, g1)):
        if f"dJdx_{tag}" not in g:
            continue
        dJdx = dJdrho[b] * 3 * (1 - 1e-9) * np.clip(g["x"], 1e-3, 1) ** 2
        assert rel(dJdx, g[f"dJdx_{tag}"]) < 1e-8


@pytest.mark.parametrize("r", [6, 8])
@pytest.mark.parametrize("k", [1, 3, 5])
def test_box_filter(lib, golden, r, k):
    from maple_b200.core import box_filter
    g = golden("ops.npz")
    out = box_filter(T(g[f"filter_r{r}_k{k}_in"][None]), r, k).cpu().numpy()[0]
    assert rel(out, g[f"filter_r{r}_k{k}_out"]) < 1e-14


def test_oc_update_matches_reference(ctx8, golden, lib):
    from maple_b200.core import HomogenizationContext
    g = golden("ops.npz")
    # cases 0 and 2 share move/xmin: one batched call
    x = np.stack([g["oc0_x"], g["oc2_x"]])
    dJ = np.stack([g["oc0_dJ"], g["oc2_dJ"]])
    vf = np.array([g["oc0_params"][0], g["oc2_params"][0]])
    xn, stats = ctx8.oc_update(T(x), T(dJ), T(vf), move=0.2, xmin=1e-3)
    xn = xn.cpu().numpy()
    assert np.abs(xn[0] - g["oc0_xnew"]).max() < 1e-10
    assert np.abs(xn[1] - g["oc2_xnew"]).max() < 1e-10
    st = stats.cpu().numpy()
    assert abs(st[0, 0] - np.abs(xn[0] - x[0]).max()) < 1e-15
    assert abs(st[0, 1] - np.abs(xn[0] - x[0]).mean()) < 1e-14
    c1 = HomogenizationContext(8, ncells=1)
    vf1, mv1, xm1 = g["oc1_params"]
    xn1, _ = c1.oc_update(T(g["oc1_x"][None]), T(g["oc1_dJ"][None]), T(np.array([vf1])), move=mv1, xmin=xm1)
    assert np.abs(xn1.cpu().numpy()[0] - g["oc1_xnew"]).max() < 1e-10
    c1.close()


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-8), ("mixed", 1e-7)])
def test_oc_step_trajectory(lib, golden, precision, tol):
    """Three fused OC iterations on device follow the reference trajectory."""
    from maple_b200.core import HomogenizationContext
    g = golden("traj_r8.npz")
    c = HomogenizationContext(8, ncells=1)
    x = T(g["x0"][None])
    w = T(np.array([[0.5, 0.0, 0.5]]))
    vf = T(np.array([0.25]))
    for it in range(3):
        out = c.oc_step(x, w, vf, penal=3.0, rho_min=1e-9, move=0.2, xmin=1e-3, filter_k=3, precision=precision,
                        rtol=1e-12, maxit=300, warm=True)
        J = out["J"].cpu().numpy()[0]
        assert abs(J - float(g[f"J{it}"])) / abs(J) < tol * 1e-1
        xn = out["x_next"].cpu().numpy()[0]
        assert np.abs(xn - g[f"x{it + 1}"]).max() < tol
        x = out["x_next"].clone()
    c.close()


def test_r16_matches_reference(lib, golden):
    from maple_b200.core import HomogenizationContext
    g = golden("homog_r16_s0.npz")
    c = HomogenizationContext(16, ncells=1)
    rho = T(simp(g["x"])[None])
    for phys, key in (("elastic", "CH"), ("thermal", "kappa")):
        c.set_density(phys, rho, "fp64")
        info = c.solve(phys, "fp64", rtol=1e-12, maxit=300)
        assert (info.status & 1).all()
        assert rel(c.homogenize(phys).cpu().numpy()[0], g[key]) < 1e-9
    c.close()


@pytest.mark.parametrize("r,fixtures", [(8, ("homog_r8_s0.npz", "homog_r8_s1.npz")), (16, ("homog_r16_s0.npz",))])
def test_refinement_mode_matches_reference(lib, golden, r, fixtures):
    """The FP32-inner-PCG / FP64-refinement form of the mixed solve reaches the
    reference's converged C^H and kappa^H like the flexible form."""
    from maple_b200.core import HomogenizationContext
    gs = [golden(f) for f in fixtures]
    c = HomogenizationContext(r, ncells=len(gs))
    c.set_mixed_mode("refine")
    rho = T(np.stack([simp(g["x"]) for g in gs]))
    for phys, key in (("elastic", "CH"), ("thermal", "kappa")):
        c.set_density(phys, rho, "mixed")
        info = c.solve(phys, "mixed", rtol=1e-12, maxit=500)
        assert (info.status == 1).all(), info
        H = c.homogenize(phys).cpu().numpy()
        for b, g in enumerate(gs):
            assert rel(H[b], g[key]) < 1e-9, (phys, b)
    c.close()


def test_solid_cell_known_answer(lib):
    from maple_b200.core import HomogenizationContext
    c = HomogenizationContext(8, ncells=1)
    rho = torch.ones((1, 512), dtype=torch.float64, device=DEV)
    for phys, ref in (("elastic", O.isotropic_elastic_tensor(1.0, 0.3)), ("thermal", np.eye(3))):
        c.set_density(phys, rho, "fp64")
        c.solve(phys, "fp64", rtol=1e-12, maxit=50)
        assert rel(c.homogenize(phys).cpu().numpy()[0], ref) < 1e-12
    c.close()


def test_deterministic(ctx8, dens8):
    _, rho = dens8
    out = []
    for _ in range(2):
        ctx8.set_density("elastic", T(rho), "mixed")
        ctx8.solve("elastic", "mixed", rtol=1e-10, maxit=300)
        out.append(ctx8.homogenize("elastic").cpu().numpy())
    assert np.array_equal(out[0], out[1])


def test_bad_arguments(lib):
    from maple_b200 import MapleError
    from maple_b200.core import HomogenizationContext
    with pytest.raises(MapleError):
        HomogenizationContext(5, ncells=1)
    c = HomogenizationContext(8, ncells=1)
    with pytest.raises(ValueError):
        c.set_density("elastic", torch.ones((1, 100), dtype=torch.float64, device=DEV))
    with pytest.raises(ValueError):
        c.set_density("elastic", torch.ones((1, 512), dtype=torch.float32, device=DEV))
    with pytest.raises(MapleError):
        c.solve("elastic", "fp64")  # no density loaded yet
    c.close()


def test_multigrid_quality_iteration_counts(lib):
    """A CPU emulation of this exact MG-PCG (Chebyshev degree 2 block-Jacobi
    smoothing on every level, Galerkin levels down to 4^3, dense FP64
    coarsest) needs 25 elastic and 13 thermal iterations to rtol 1e-10 on this
    32^3 density from zero; a defective level (operator, transfer or smoother)
    shows up as extra iterations.  The context is set to that configuration."""
    from maple_b200.core import HomogenizationContext
    r = 32
    x = O.seed_density(0, r, 2.0, 0.25)
    rho = T(simp(x).reshape(1, -1))
    c = HomogenizationContext(r, ncells=1)
    c.set_options(cheb_degree=2, coarse_degree=2)
    H = {}
    for prec in ("fp64", "mixed"):
        for phys, cap in (("elastic", 30), ("thermal", 16)):
            c.set_density(phys, rho, prec)
            info = c.solve(phys, prec, rtol=1e-10, maxit=300)
            assert info.status[0] & 1
            assert info.iters[0] <= cap + (3 if prec == "mixed" else 0), (prec, phys, info.iters[0])
            H[(prec, phys)] = c.homogenize(phys).cpu().numpy()[0]
    for phys in ("elastic", "thermal"):
        assert rel(H[("mixed", phys)], H[("fp64", phys)]) < 1e-9
    c.close()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_coarse_stencil_kernels_agree(lib, precision):
    """The three coarse-level stencil kernels solve alike: the shared-memory
    tile kernel (nine and split off), the split-offset kernel (every level with
    n >= 8) and the nine-thread kernel (every level): the same C^H / kappa^H to
    summation-order accuracy and iteration counts within one, on two different
    cells in one context."""
    from maple_b200.core import HomogenizationContext
    r = 32
    rho = T(np.stack([simp(O.seed_density(s, r, 2.0, 0.25)).reshape(-1) for s in (0, 1)]))
    out = {}
    for name, nine, split in (("tile", 0, 0), ("split", 0, 8), ("nine", 64, 0)):
        c = HomogenizationContext(r, ncells=2)
        c.set_stencil_nine(nine)
        c.set_stencil_split(split)
        for phys in ("elastic", "thermal"):
            c.set_density(phys, rho, precision)
            info = c.solve(phys, precision, rtol=1e-10, maxit=300)
            assert (info.status & 1).all()
            out[(name, phys)] = (c.homogenize(phys).cpu().numpy(), info.iters.copy())
        c.close()
    for phys in ("elastic", "thermal"):
        H0, it0 = out[("tile", phys)]
        for name in ("split", "nine"):
            H1, it1 = out[(name, phys)]
            for b in range(2):
                assert rel(H1[b], H0[b]) < (1e-12 if precision == "fp64" else 1e-9), (name, phys, b)
            assert np.abs(it1.astype(int) - it0.astype(int)).max() <= 1, (name, phys, it0, it1)


@pytest.mark.parametrize("r", [16, 32])
@pytest.mark.parametrize("coarse_degree", [0, 1, 5])
def test_fused_tail_matches_separate_launches(lib, r, coarse_degree):
    """The one-launch bottom of the FP32 V-cycle (8^3 level, restriction, 4^3
    coarsest solve, prolongation; a cluster of 8 CTAs per cell) computes what
    the separate launches compute, bit for bit: the same solutions, C^H /
    kappa^H and iteration counts, with an inactive cell between two active
    ones.  r = 16 puts the fused level at level 1, r = 32 at level 2;
    Chebyshev degrees 1 and 5 cover the smoothing loops' ends."""
    from maple_b200.core import HomogenizationContext
    rho = T(np.stack([simp(O.seed_density(s, r, 2.0, 0.3)).reshape(-1) for s in (3, 4, 5)]))
    out = {}
    for fused in (False, True):
        c = HomogenizationContext(r, ncells=3)
        c.set_options(coarse_degree=coarse_degree)
        c.set_tail_fused(fused)
        c.set_active([1, 0, 1])
        c.profile(True)
        for phys in ("elastic", "thermal"):
            c.set_density(phys, rho, "mixed")
            info = c.solve(phys, "mixed", rtol=1e-10, maxit=300)
            assert (info.status[[0, 2]] & 1).all()
            out[(fused, phys)] = (c.homogenize(phys).cpu().numpy(), info.iters.copy(),
                                  c.solution(phys)[[0, 2]].clone())
        names = c.profile_read()
        ran = any(k.startswith("k_tail_cycle") for k in names)
        assert ran == fused, sorted(names)
        c.close()
    for phys in ("elastic", "thermal"):
        H0, it0, u0 = out[(False, phys)]
        H1, it1, u1 = out[(True, phys)]
        assert torch.equal(u0, u1), (phys, (u0 - u1).abs().max().item())
        for b in (0, 2):
            assert np.array_equal(H1[b], H0[b]), (phys, b)
            assert it1[b] == it0[b], (phys, b, it0, it1)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("r", [16, 32])
def test_pdl_matches_plain_launches(lib, precision, r):
    """Programmatic dependent launch of the coarse sweeps, transfers and the
    fused tail changes only when kernels start: solutions and iteration counts
    are bit-identical to plain launches, for graph replays and eager runs,
    with an inactive cell."""
    from maple_b200.core import HomogenizationContext
    rho = T(np.stack([simp(O.seed_density(s, r, 2.0, 0.3)).reshape(-1) for s in (6, 7, 8)]))
    out = {}
    for pdl in (False, True):
        for graphs in (False, True):
            c = HomogenizationContext(r, ncells=3)
            c.set_pdl(pdl)
            c.set_graphs(graphs)
            c.set_active([1, 0, 1])
            for phys in ("elastic", "thermal"):
                c.set_density(phys, rho, precision)
                info = c.solve(phys, precision, rtol=1e-10, maxit=300)
                assert (info.status[[0, 2]] & 1).all()
                out[(pdl, graphs, phys)] = (info.iters.copy(), c.solution(phys)[[0, 2]].clone())
            c.close()
    for phys in ("elastic", "thermal"):
        it0, u0 = out[(False, False, phys)]
        for key in ((False, True), (True, False), (True, True)):
            it1, u1 = out[key + (phys,)]
            assert torch.equal(u0, u1), (phys, key, (u0 - u1).abs().max().item())
            assert np.array_equal(it0[[0, 2]], it1[[0, 2]]), (phys, key)


@pytest.mark.parametrize("form", ["fp64", "flexible", "refine", "reliable"])
def test_device_loop_matches_host_loop(lib, form):
    """The device-side PCG loop (conditional graph node, one host wait per
    solve) runs the same iterations as the per-iteration graph replays with a
    host convergence check after each: bit-identical solutions and iteration
    counts, with an inactive cell, and the same stop at an iteration cap."""
    from maple_b200.core import HomogenizationContext, launch_count
    r = 16
    precision = "fp64" if form == "fp64" else "mixed"
    rho = T(np.stack([simp(O.seed_density(s, r, 2.0, 0.3)).reshape(-1) for s in (11, 12, 13)]))
    out = {}
    launches = {}
    for loop in (None, False, True):  # None: eager, no graphs
        c = HomogenizationContext(r, ncells=3)
        if loop is None:
            c.set_graphs(False)
        else:
            c.set_device_loop(loop)
        n0 = launch_count()
        if form != "fp64":
            c.set_mixed_mode(form)
        c.set_active([1, 0, 1])
        for phys in ("elastic", "thermal"):
            c.set_density(phys, rho, precision)
            info = c.solve(phys, precision, rtol=1e-10, maxit=300)
            assert (info.status[[0, 2]] & 1).all()
            out[(loop, phys)] = (info.iters.copy(), c.solution(phys)[[0, 2]].clone())
            # capped: the loop stops at maxit with the cells unconverged
            c.set_density(phys, rho, precision)
            capped = c.solve(phys, precision, rtol=1e-14, maxit=4)
            out[(loop, phys, "cap")] = (capped.iters.copy(), capped.status.copy(), c.solution(phys)[[0, 2]].clone())
        launches[loop] = launch_count() - n0
        assert c.device_loop_state() == (1 if loop else 0)
        c.close()
    # Launch counts: per-iteration graph replays launch what the eager runs
    # launch.  With conditional nodes the device loop adds its counting kernel
    # per iteration, and a reliable-update iteration runs its replacement (an
    # IF node) only when one is due, where the others launch it predicated.
    assert launches[False] == launches[None], launches
    if form == "reliable":
        assert launches[True] < launches[None], launches
    else:
        assert launches[True] > launches[None], launches
    for phys in ("elastic", "thermal"):
        it0, u0 = out[(False, phys)]
        it1, u1 = out[(True, phys)]
        assert torch.equal(u0, u1), (phys, (u0 - u1).abs().max().item())
        assert np.array_equal(it0[[0, 2]], it1[[0, 2]]), (phys, it0, it1)
        c0, s0, v0 = out[(False, phys, "cap")]
        c1, s1, v1 = out[(True, phys, "cap")]
        assert np.array_equal(c0[[0, 2]], c1[[0, 2]]) and np.array_equal(s0[[0, 2]], s1[[0, 2]]), (phys, c0, c1)
        assert torch.equal(v0, v1)


def test_reliable_form_hands_slow_cells_to_flexible(lib):
    """The reliable-update form: its answer matches the flexible form and
    plain FP64 to the tolerance; a cell still unconverged after the handover
    count continues in the flexible form from its iterate and converges, the
    iterations of both parts counted, within the same limit."""
    from maple_b200.core import HomogenizationContext
    r = 16
    rho = T(np.stack([simp(O.seed_density(s, r, 2.0, 0.3)).reshape(-1) for s in (21, 22)]))
    sol = {}
    for form, handover in (("fp64", None), ("flexible", None), ("reliable", 120), ("reliable", 5)):
        c = HomogenizationContext(r, ncells=2)
        prec = "fp64" if form == "fp64" else "mixed"
        if form != "fp64":
            c.set_mixed_mode(form)
        if handover:
            c.set_reliable_options(1e-3, handover)
        for phys in ("elastic", "thermal"):
            c.set_density(phys, rho, prec)
            info = c.solve(phys, prec, rtol=1e-10, maxit=300)
            assert (info.status == 1).all(), (form, handover, phys, info.status)
            if handover == 5:
                assert (info.iters > 5).all()
            sol[(form, handover, phys)] = (c.solution(phys), info.iters.copy())
        c.close()
    def mean_free(u):  # the periodic solution is defined up to a translation
        return u - u.mean(dim=-1, keepdim=True)

    for phys in ("elastic", "thermal"):
        ref, it_ref = sol[("fp64", None, phys)]
        ref = mean_free(ref)
        for key in (("flexible", None), ("reliable", 120), ("reliable", 5)):
            u, it = sol[key + (phys,)]
            err = ((mean_free(u) - ref).norm() / ref.norm()).item()
            assert err < 1e-8, (key, phys, err)
        # the reliable form keeps the Krylov space: about the FP64 iteration count
        assert np.all(sol[("reliable", 120, phys)][1] <= it_ref + 3), (phys, sol[("reliable", 120, phys)][1], it_ref)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_graph_replay_matches_eager(lib, precision):
    """The captured PCG iteration replays the same launches: identical results
    and iteration counts with graphs on and off."""
    from maple_b200.core import HomogenizationContext
    r = 16
    rho = T(simp(O.seed_density(1, r, 2.0, 0.3)).reshape(1, -1))
    out = []
    for graphs in (False, True):
        c = HomogenizationContext(r, ncells=1)
        c.set_graphs(graphs)
        res = []
        for phys in ("elastic", "thermal"):
            c.set_density(phys, rho, precision)
            info = c.solve(phys, precision, rtol=1e-10, maxit=200)
            res.append((int(info.iters[0]), c.homogenize(phys).cpu().numpy()))
        out.append(res)
        c.close()
    for (i0, h0), (i1, h1) in zip(out[0], out[1]):
        assert i0 == i1
        assert np.array_equal(h0, h1)


def test_precision_switch_on_one_context(lib):
    """A context used first in mixed precision and then in FP64 (and back)
    gives the results of contexts used in one precision only."""
    from maple_b200.core import HomogenizationContext
    r = 16
    rho = T(simp(O.seed_density(3, r, 2.0, 0.25)).reshape(1, -1))
    ref = {}
    for prec in ("fp64", "mixed"):
        c = HomogenizationContext(r, ncells=1)
        c.set_density("elastic", rho, prec)
        c.solve("elastic", prec, rtol=1e-12, maxit=300)
        ref[prec] = c.homogenize("elastic").cpu().numpy()
        c.close()
    c = HomogenizationContext(r, ncells=1)
    for prec in ("mixed", "fp64", "mixed"):
        c.set_density("elastic", rho, prec)
        c.solve("elastic", prec, rtol=1e-12, maxit=300)
        assert rel(c.homogenize("elastic").cpu().numpy(), ref[prec]) < 1e-11, prec
    c.close()


def test_concurrent_physics_match_sequential(lib):
    """OC steps with the elastic and thermal solves running at the same time
    (two streams, two host threads) give bit-identical results to the same
    steps run one physics after the other."""
    from maple_b200.core import HomogenizationContext
    r, B = 16, 2
    x0 = np.stack([O.seed_density(s, r, 2.0, 0.3).reshape(-1) for s in (4, 5)])
    w = T(np.array([[0.4, 0.2, 0.4], [1 / 3, 1 / 3, 1 / 3]]))
    vf = T(np.array([0.3, 0.3]))
    runs = []
    for concurrent in (False, True):
        c = HomogenizationContext(r, ncells=B)
        c.set_concurrency(concurrent)
        x = T(x0)
        rec = []
        for _ in range(3):
            out = c.oc_step(x, w, vf, precision="mixed", rtol=1e-10, warm=True)
            x = out["x_next"].clone()
            rec.append((out["J"].cpu().numpy(), x.cpu().numpy(), np.array(out["iters"])))
        runs.append(rec)
        c.close()
    for (j0, x0_, i0), (j1, x1, i1) in zip(*runs):
        assert np.array_equal(j0, j1) and np.array_equal(x0_, x1) and np.array_equal(i0, i1)


def test_symmetrize_matches_reference(lib, golden):
    """maple_symmetrize and the symmetrize_vec drop-in against the reference's
    symmetrize_vec on a random 8^3 field, for mirror axes and the cube group."""
    from maple_b200.core import symmetrize
    from maple_b200.optimize import build_unitcell_batch, parse_symmetry, symmetrize_vec
    g = golden("sym.npz")
    batch = build_unitcell_batch(DEV, 8, torch.zeros(8, 8, 8, device=DEV))
    v = T(g["field"].reshape(1, -1))
    for spec in ["x", "xy", "yz", "xyz", "cubic"]:
        kind, axes = parse_symmetry(spec)
        out = symmetrize(v, 8, kind, axes).cpu().numpy().reshape(-1)
        assert np.abs(out - g["sym::" + spec]).max() < 1e-14, spec
        dv = symmetrize_vec(v.reshape(-1, 1), batch["elem_coords"], 8, kind, axes)
        assert dv.shape == (512, 1) and np.abs(dv.cpu().numpy().reshape(-1) - g["sym::" + spec]).max() < 1e-14


@pytest.mark.parametrize("spec", ["cubic", "xy"])
def test_symmetric_oc_step_trajectory(lib, golden, spec):
    """Three fused OC steps with a symmetry projection follow the reference's
    trajectory (solve at the projected design, projected gradient, projected
    update)."""
    from maple_b200.core import HomogenizationContext
    from maple_b200.optimize import parse_symmetry
    g = golden("sym.npz")
    ctx = HomogenizationContext(8, ncells=1)
    ctx.set_symmetry(*parse_symmetry(spec))
    x = T(g[f"traj_{spec}_x0"].reshape(1, -1))
    w, vf = T(np.array([[0.5, 0.0, 0.5]])), T(np.array([0.25]))
    for it in range(3):
        out = ctx.oc_step(x, w, vf, precision="fp64", rtol=1e-12, warm=True)
        ref_J = g[f"traj_{spec}_J{it}"]
        assert abs(float(out["J"][0]) - ref_J) < 1e-8 * abs(ref_J), (spec, it)
        x_next = out["x_next"].cpu().numpy().reshape(-1)
        assert np.abs(x_next - g[f"traj_{spec}_x{it + 1}"]).max() < 1e-7, (spec, it)
        dx = np.abs(x_next - x.cpu().numpy().reshape(-1))
        assert abs(float(out["stats"][0, 0]) - dx.max()) < 1e-14 and abs(float(out["stats"][0, 1]) - dx.mean()) < 1e-14
        x = out["x_next"].clone()
    ctx.close()


@pytest.mark.parametrize("r", [8, 16])
def test_coarse_element_matrices_match_oracle(lib, r):
    """Every level's Galerkin element matrices (k_level1_elements,
    k_coarsen_elements) against the oracle's per-coarse-element P^T K P
    (utils/EBE_GMG.py:226-337, utils/EBE_GMG_scalar.py:135-230)."""
    from maple_b200.core import HomogenizationContext
    xs = [O.seed_density(s, r, 2.0, 0.3).reshape(-1) for s in (3, 4)]
    rho = np.stack([simp(x) for x in xs])
    c = HomogenizationContext(r, ncells=2)
    el = O.Elements(r)
    for phys, d in (("elastic", 3), ("thermal", 1)):
        c.set_density(phys, T(rho), "mixed" if r == 16 else "fp64")
        Ke0 = el.get(d)[0]
        for b in range(2):
            ke, n = rho[b].reshape(-1, 1, 1) * Ke0[None], r
            for level in range(1, c.levels):
                ke = O.coarsen_elements(ke, n, d)
                n //= 2
                got = c.level_elements(phys, level)[b].cpu().numpy()
                assert rel(got, ke) < 1e-12, (phys, b, level)
    c.close()


@pytest.mark.parametrize("nc,K", [(2, 3), (4, 18), (8, 3)])
def test_grid_transfers_match_oracle_prolongation(lib, nc, K):
    """k_restrict and k_prolong_add against the oracle's assembled periodic
    trilinear P (utils/EBE_GMG.py:38-79, 531-647), element by element."""
    from maple_b200.core import transfer
    rng = np.random.default_rng(nc * 100 + K)
    nf = 2 * nc
    P = O.prolongation(nf, 1)  # per component: the same weights for every field
    fine = rng.standard_normal((2, K, nf ** 3))
    coarse = rng.standard_normal((2, K, nc ** 3))
    base = rng.standard_normal((2, K, nf ** 3))
    rc = transfer("restrict", T(fine)).cpu().numpy()
    uf = transfer("prolong_add", T(coarse), out=T(base)).cpu().numpy()
    for b in range(2):
        for k in range(K):
            assert rel(rc[b, k], P.T @ fine[b, k]) < 1e-14, (b, k)
            assert rel(uf[b, k], base[b, k] + P @ coarse[b, k]) < 1e-14, (b, k)


def test_element_batched_tensor_core_matvec(lib):
    """The element-batched operator on tcgen05 (TF32 contraction of all
    elements and load cases, the reference's EBE form) against the FP64
    stencil operator, to the TF32 rounding."""
    from maple_b200 import _lib
    from maple_b200.core import HomogenizationContext
    import ctypes as C
    r, B = 16, 2
    N = r ** 3
    rho = np.stack([simp(O.seed_density(s, r, 2.0, 0.3).reshape(-1)) for s in (5, 6)])
    c = HomogenizationContext(r, ncells=B)
    c.set_density("elastic", T(rho), "mixed")
    rng = np.random.default_rng(3)
    u = rng.standard_normal((B, 6, 3, N))
    y64 = c.matvec("elastic", T(rho), T(u)).cpu().numpy()
    u32 = torch.tensor(u, dtype=torch.float32, device=DEV).contiguous()
    y32 = torch.empty_like(u32)
    rows = torch.empty(B * N * 6 * 24, dtype=torch.float32, device=DEV)
    outw = torch.empty_like(rows)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    _lib.check(lib.maple_matvec_ebe_tc(c._h, C.c_void_p(u32.data_ptr()), C.c_void_p(y32.data_ptr()),
                                       C.c_void_p(rows.data_ptr()), C.c_void_p(outw.data_ptr()), stream))
    err = np.abs(y32.cpu().numpy() - y64).max() / np.abs(y64).max()
    assert err < 5e-3, err
    c.close()


def test_extrapolated_warm_start_keeps_the_answer(lib):
    """maple_set_extrapolation only changes where the OC step's solves start:
    the trajectory is the same to the solver tolerance."""
    from maple_b200.core import HomogenizationContext
    r, B = 16, 2
    x0 = np.stack([O.seed_density(s, r, 2.0, 0.3).reshape(-1) for s in (1, 2)])
    w = T(np.array([[1 / 3, 1 / 3, 1 / 3], [0.5, 0.0, 0.5]]))
    vf = T(np.full(B, 0.3))
    out = {}
    for theta in (0.0, 1.0):
        c = HomogenizationContext(r, ncells=B)
        c.set_extrapolation(theta)
        x, Js, its = T(x0), [], 0
        for _ in range(6):
            o = c.oc_step(x, w, vf, precision="mixed", rtol=1e-12, maxit=1000, warm=True)
            x = o["x_next"].clone()
            Js.append(o["J"].cpu().numpy())
            its += int(o["iters"].sum())
        out[theta] = (np.array(Js), x.cpu().numpy(), its)
        c.close()
    assert rel(out[1.0][0], out[0.0][0]) < 1e-10
    assert np.abs(out[1.0][1] - out[0.0][1]).max() < 1e-8
