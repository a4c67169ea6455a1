"""The FP64 oracle against the golden vectors produced by the reference code.

These pin the oracle: every later GPU parity test compares against it (or
directly against the same golden vectors).
"""
import numpy as np
import pytest

from oracle import ihd_oracle as O


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b))) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("r", [8, 16, 32])
def test_element_tables(golden, r):
    g = golden("element_tables.npz")
    e = O.Elements(r)
    for name, mine in dict(Ke3=e.Ke3, Fe3=e.Fe3, X03=e.X03, Ke1=e.Ke1, Fe1=e.Fe1, X01=e.X01).items():
        assert rel(mine, g[f"r{r}_{name}"]) < 1e-12, name


def test_assemble_rhs(golden):
    g = golden("homog_r8_s0.npz")
    r = 8
    e = O.Elements(r)
    rho = 1e-9 + (1 - 1e-9) * g["x"] ** 3
    F3 = O.assemble_F(rho, e.Fe3, r, 3)                      # (N*3, 6)
    assert rel(F3.reshape(-1, 3, 6), g["F_elastic"]) < 1e-13
    F1 = O.assemble_F(rho, e.Fe1, r, 1)
    assert rel(F1, g["F_thermal"]) < 1e-13


@pytest.mark.parametrize("case", ["homog_r8_s0.npz", "homog_r8_s1.npz"])
def test_converged_homogenization(golden, case):
    g = golden(case)
    r = int(g["r"])
    rho = 1e-9 + (1 - 1e-9) * g["x"] ** 3
    res = O.solve_cell(rho, r, levels=3, max_cycles=200, rtol=1e-14)
    assert rel(res["CH"], g["CH"]) < 1e-10
    assert rel(res["kappa"], g["kappa"]) < 1e-10
    if "u_elastic" in g:
        u = res["u3"].reshape(-1, 3, 6)
        ug = g["u_elastic"]
        # both are converged solutions; they may differ by a rigid translation
        du = (u - u.mean(0)) - (ug - ug.mean(0))
        assert np.abs(du).max() / np.abs(ug).max() < 1e-9


def test_converged_homogenization_r16(golden):
    g = golden("homog_r16_s0.npz")
    assert g["relres_elastic"].max() < 1e-8 and g["relres_thermal"].max() < 1e-8
    rho = 1e-9 + (1 - 1e-9) * g["x"] ** 3
    res = O.solve_cell(rho, 16, levels=4, max_cycles=200, rtol=1e-13)
    assert rel(res["CH"], g["CH"]) < 1e-9
    assert rel(res["kappa"], g["kappa"]) < 1e-9


@pytest.mark.parametrize("tag,weights", [("bi", {"stiffness": 0.5, "thermal": 0.5}),
                                         ("tri", {"stiffness": 1 / 3, "shear": 1 / 3, "thermal": 1 / 3})])
def test_analytic_sensitivity_matches_autograd(golden, tag, weights):
    """dJ/dx from the analytic adjoint equals the reference's autograd through
    converged solves (main_IHD_v3.py:688)."""
    g = golden("homog_r8_s0.npz")
    r = 8
    x = g["x"]
    rho = 1e-9 + (1 - 1e-9) * x ** 3
    res = O.solve_cell(rho, r, levels=3, max_cycles=200, rtol=1e-14)
    J, gC, gK = O.objective_and_grads(weights, res["CH"], res["kappa"])
    assert abs(J - float(g[f"J_{tag}"])) / abs(J) < 1e-10
    dJdrho = np.einsum("eij,ij->e", res["dCH"], gC) + np.einsum("eij,ij->e", res["dkappa"], gK)
    dJdx = dJdrho * 3 * (1 - 1e-9) * x ** 2
    assert rel(dJdx, g[f"dJdx_{tag}"]) < 1e-8


@pytest.mark.parametrize("r", [6, 8])
@pytest.mark.parametrize("k", [1, 3, 5])
def test_box_filter(golden, r, k):
    g = golden("ops.npz")
    out = O.box_filter_periodic(g[f"filter_r{r}_k{k}_in"], r, k)
    assert rel(out, g[f"filter_r{r}_k{k}_out"]) < 1e-14


def test_box_filter_rejects_even():
    with pytest.raises(ValueError):
        O.box_filter_periodic(np.zeros(8), 2, 2)


@pytest.mark.parametrize("i", [0, 1, 2])
def test_oc_update(golden, i):
    g = golden("ops.npz")
    vf, move, xmin = g[f"oc{i}_params"]
    xn = O.oc_update(g[f"oc{i}_x"], g[f"oc{i}_dJ"], vf, move, xmin)
    assert np.abs(xn - g[f"oc{i}_xnew"]).max() < 1e-12


@pytest.mark.parametrize("i", [0, 1, 2])
@pytest.mark.parametrize("tag,spec", [("stiff", "stiffness"), ("shear", "shear"), ("therm", "thermal"),
                                      ("bi", "stiffness:0.5,thermal:0.5"),
                                      ("tri", "stiffness:0.3333333333333333,shear:0.3333333333333333,"
                                              "thermal:0.3333333333333333"),
                                      ("mixw", "0.4*stiffness+0.6*thermal")])
def test_objectives_and_gradients(golden, i, tag, spec):
    g = golden("ops.npz")
    w = O.parse_objective_spec(spec)
    J, gC, gK = O.objective_and_grads(w, g[f"obj{i}_CH"], g[f"obj{i}_kappa"])
    assert abs(J - float(g[f"obj{i}_{tag}_J"])) <= 1e-12 * max(1.0, abs(J))
    assert np.abs(gC - g[f"obj{i}_{tag}_gC"]).max() < 1e-9 * max(1.0, np.abs(gC).max())
    assert np.abs(gK - g[f"obj{i}_{tag}_gK"]).max() < 1e-12


def test_spec_parser(golden):
    g = golden("ops.npz")
    for key in g.files:
        if not key.startswith("spec::"):
            continue
        spec = key[len("spec::"):]
        mine = sorted((k, str(float(v))) for k, v in O.parse_objective_spec(spec).items())
        ref = [(a, str(float(b))) for a, b in g[key]]
        assert mine == ref, spec


def test_oc_trajectory(golden):
    """Three OC iterations (main_IHD_v3.py:620-716) match the reference run."""
    g = golden("traj_r8.npz")
    x = g["x0"]
    e = O.Elements(8)
    for it in range(3):
        x, info = O.oc_iteration(x, 8, {"stiffness": 0.5, "thermal": 0.5}, volfrac=0.25, move=0.2, elems=e,
                                 levels=3, rtol=1e-14)
        assert abs(info["J"] - float(g[f"J{it}"])) / abs(info["J"]) < 1e-10
        assert np.abs(x - g[f"x{it + 1}"]).max() < 1e-8


def test_seed_density_properties():
    for vf in (0.01, 0.25, 0.4):
        x = O.seed_density(3, 16, 2.0, vf)
        assert x.shape == (16, 16, 16)
        assert x.min() >= 1e-3 and x.max() <= 1.0
        assert abs(x.mean() - vf) < 1e-6


def test_solid_cell_known_answer():
    """A solid cell homogenizes to the isotropic C and kappa = I."""
    r = 6
    res = O.solve_cell(np.ones(r ** 3), r, levels=2, max_cycles=50, rtol=1e-13)
    C = O.isotropic_elastic_tensor(1.0, 0.3)
    assert rel(res["CH"], C) < 1e-12
    assert rel(res["kappa"], np.eye(3)) < 1e-12


def test_symmetry_parse_and_projection_match_reference(golden):
    g = golden("sym.npz")
    for key in g.files:
        if key.startswith("parse::"):
            spec = key.split("::", 1)[1]
            kind, axes = O.parse_symmetry(spec)
            assert [kind] + [str(a) for a in axes] == list(g[key]), spec
    for spec in ["x", "xy", "yz", "xyz", "cubic"]:
        kind, axes = O.parse_symmetry(spec)
        out = O.symmetrize(g["field"], 8, kind, axes)
        assert np.abs(out - g["sym::" + spec]).max() < 1e-14, spec
        assert np.abs(O.symmetrize(out, 8, kind, axes) - out).max() < 1e-14  # a projection


@pytest.mark.parametrize("spec", ["cubic", "xy"])
def test_symmetric_trajectory_matches_reference(golden, spec):
    g = golden("sym.npz")
    x = g[f"traj_{spec}_x0"]
    for it in range(3):
        x, info = O.oc_iteration(x, 8, {"stiffness": 0.5, "thermal": 0.5}, volfrac=0.25, symmetry=spec, rtol=1e-12)
        assert abs(info["J"] - g[f"traj_{spec}_J{it}"]) < 1e-8 * abs(g[f"traj_{spec}_J{it}"]), (spec, it)
        assert np.abs(x - g[f"traj_{spec}_x{it + 1}"]).max() < 1e-7, (spec, it)


def test_dropin_parse_symmetry_matches_reference(golden):
    from maple_b200.optimize import parse_symmetry
    g = golden("sym.npz")
    for key in g.files:
        if key.startswith("parse::"):
            kind, axes = parse_symmetry(key.split("::", 1)[1])
            assert [kind] + [str(a) for a in axes] == list(g[key])


def _print_case(kind, kw, rho, r=8):
    """Oracle call for one fixture case (reference keyword names)."""
    if kind == "over":
        return O.overhang_penalty(rho, r, kw.get("overhang_deg", 45.0), kw.get("periodic_xy", True))
    tiles = tuple(kw.get("tiles_xyz", (1, 1, 1)))
    return O.cavity_penalty(rho, r, void_thresh=kw.get("void_thresh", 0.5), beta=kw.get("beta", 20.0),
                            min_channel_rad=kw.get("min_channel_rad", 0), rad=kw.get("rad", 1),
                            iters=kw.get("iters", 0), tiles=tiles, focus_center=kw.get("focus_center", True),
                            seed_faces=kw.get("seed_faces", "all"), periodic=kw.get("periodic_xyz", None))


def _print_cases(golden):
    import json
    g = golden("print.npz")
    return g, [json.loads(c) for c in g["cases"]]


@pytest.mark.parametrize("field", ["cont", "simp"])
def test_printability_penalties_match_reference_autograd(golden, field):
    g, cases = _print_cases(golden)
    rho = g[f"field_{field}"]
    for i, (kind, kw) in enumerate(cases):
        P, grad = _print_case(kind, kw, rho)
        ref_P, ref_g = g[f"{field}_{i}_P"], g[f"{field}_{i}_grad"]
        assert abs(P - ref_P) <= 1e-13 * max(1.0, abs(ref_P)), (i, kind, kw)
        assert np.abs(grad - ref_g).max() <= 1e-12 * max(1e-300, np.abs(ref_g).max()), (i, kind, kw)


PRINT_TRAJ_CAVITY = dict(void_thresh=0.5, beta=20.0, min_channel_rad=1, rad=1, iters=0, tiles=(2, 2, 2),
                         focus_center=True, seed_faces="all")


def test_penalised_trajectory_matches_reference(golden):
    g = golden("print.npz")
    x = g["traj_x0"]
    for it in range(3):
        x, info = O.oc_iteration(x, 8, {"stiffness": 0.5, "thermal": 0.5}, volfrac=0.25, rtol=1e-12,
                                 lambda_print=0.9, overhang_deg=45.0, lambda_cavity=0.9, cavity=PRINT_TRAJ_CAVITY)
        assert abs(info["J"] - g[f"traj_J{it}"]) < 1e-8 * abs(g[f"traj_J{it}"]), it
        assert abs(info["P_print"] - g[f"traj_Pp{it}"]) < 1e-10 and abs(info["P_cavity"] - g[f"traj_Pc{it}"]) < 1e-10
        assert np.abs(x - g[f"traj_x{it + 1}"]).max() < 1e-7, it


def test_oracle_meets_the_32cube_reference_pins(golden):
    """The 32^3 trajectory fixture: the oracle's own evaluation of the design
    of iteration 10 reproduces the recorded J, C^H and kappa^H, and these agree
    with the reference's solvers at that design (its residual there is tiny)."""
    g = golden("traj_r32.npz")
    r = int(g["r"])
    w = O.parse_objective_spec("stiffness:0.5,thermal:0.5")
    _, info = O.oc_iteration(g["x10"], r, w, volfrac=float(g["vf"]), move=0.2, levels=5, rtol=1e-12,
                             max_cycles=2000, method="pcg")
    assert abs(info["J"] - float(g["J"][10])) < 1e-12 * float(g["J"][10])
    assert np.abs(info["CH"] - g["CH"][10]).max() < 1e-11 * np.abs(g["CH"][10]).max()
    assert abs(info["J"] - float(g["ref_J_10"])) < 1e-12 * float(g["J"][10])
    assert np.abs(info["kappa"] - g["ref_kappa_10"]).max() < 1e-11 * np.abs(g["ref_kappa_10"]).max()
    for it in (0, 1, 10, 25, 49):
        assert float(g[f"ref_relres_{it}"]) < 1e-12


def test_port_follows_the_32cube_trajectory(golden):
    """The multithreaded C port (the bench's CPU path) follows the first three
    iterations of the 32^3 trajectory fixture."""
    from oracle import port as P
    g = golden("traj_r32.npz")
    P.build()
    P.set_threads(4)
    r = int(g["r"])
    w = O.parse_objective_spec("stiffness:0.5,thermal:0.5")
    cell = P.Cell(r, 5)
    x = g["x0"]
    for it in range(3):
        x, info = P.oc_iteration(x, cell, w, volfrac=float(g["vf"]), rtol=1e-12, max_cycles=2000, warm=True,
                                 method="pcg")
        assert abs(info["J"] - float(g["J"][it])) < 1e-12 * float(g["J"][it]), it
        if it == 0:
            assert np.abs(x - g["x1"]).max() < 1e-12
