"""Parity of the CUDA path with the reference (golden fixtures made by the
reference itself) and with the C restatement in oracle/ on the same inputs.

Bars: bit-identical for geometry, gradients, assembled matrices and
right-hand sides and corrected fluxes; for whole SIMPLE iterations, whose
linear solves use parallel dot products, U, p and phi within 1e-6 relative
L2 (the reported differences sit far below it).
"""
import dataclasses

import numpy as np
import pytest

import _cases as K
import _oracle as O

pytestmark = pytest.mark.gpu

REL_TOL = 1e-6  # relative L2, U / p / phi after K SIMPLE iterations (FP64)


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def mesh_from_fixture(g):
    import chuanflow_b200 as cf
    pats = [(str(n), str(t), int(s), int(z)) for n, t, s, z in
            zip(g["patch_names"], g["patch_types"], g["patch_start"], g["patch_size"])]
    return cf.PolyMesh(g["points"], g["face_offsets"], g["face_verts"], g["owner"], g["neighbour"], pats)


@pytest.mark.parametrize("fixture", ["mesh_tets22.npz", "mesh_hex41.npz"])
def test_gradients_bit_exact(golden, fixture):
    import chuanflow_b200 as cf
    g = golden(fixture)
    mesh = mesh_from_fixture(g)
    case = cf.SimpleCase(mesh)
    for fname in K.POLY_FIELDS:
        t, b = g[f"T_{fname}"], g[f"B_{fname}"]
        for s in ("linear", "corrected", "leastSquares"):
            got = case.gradient(t, b, s)
            assert np.array_equal(got, g[f"grad_fn_{s}_{fname}"]), (fixture, fname, s)
            got = case.gradient(t, b, s, vol_quirk=True)
            assert np.array_equal(got, g[f"grad_vol_{s}_{fname}"]), (fixture, fname, s, "vol")


@pytest.mark.parametrize("order", ["identity", "colour", "rcm", "rcm-colour"])
def test_equations_bit_exact(golden, order):
    """Momentum and pressure assembly, gradients, rAUf, div(phi), continuity
    and the flux correction of one outer iteration equal the reference's, in
    every device cell numbering."""
    g = golden("eqns_cavity.npz")
    mesh, case = K.cavity_product(6, 5, 4, order=order)
    assert np.array_equal(mesh.addressing()["points"], g["points"])
    case.upload(g["in_U"], g["in_p"], g["in_phi"])
    ctl = K.controls_from(K.cavity_case(6, 5, 4))
    out = case.probe_equations(ctl, g["in_xprobe"])
    assert np.array_equal(out["gradPn"], g["gradPn"])
    for q in range(3):
        assert np.array_equal(out["U_diag"][q], g[f"U_diag{q}"]), q
        assert np.array_equal(out["U_h0"][q], g[f"U_h0_{q}"]), q
        assert np.array_equal(out["U_h1"][q], g[f"U_h1_{q}"]), q
    for k in ("rAUf", "divPhi", "contErr", "p_diag", "p_h0", "p_h1", "phiCorrected"):
        assert np.array_equal(out[k], g[k]), k
    assert np.array_equal(out["gradPFull"], g["gradPFull"])


def test_simple_channel_matches_reference(golden):
    """4 SIMPLE iterations of the jittered channel (non-orthogonal, nonOrth 2,
    pRelaxStart) against the reference's own run."""
    g = golden("simple_channel.npz")
    mesh, case = K.channel_product(10, 6, 5)
    assert np.array_equal(mesh.addressing()["points"], g["points"])
    res = case.solve(K.controls_from(K.channel_case(10, 6, 5)))
    U, p, phi = case.download()
    assert res.iterations == int(g["iterations"])
    for a, b, name in ((U, g["U"], "U"), (p, g["p"], "p"), (phi, g["phi"], "phi")):
        assert rel(a, b) < REL_TOL, (name, rel(a, b))
    assert abs(res.final_continuity_error - float(g["continuity"])) <= 1e-6 * abs(float(g["continuity"]))


def test_simple_channel_time_term_matches_reference(golden):
    """SIMPLE with the reference's time term (SimpleControls::dt and
    uTimeOld, simpleSolver.cpp:75-97): six one-sweep calls with dt 0.05, each
    taking the velocity it starts from as the old time level, against the
    reference's own six calls; and the reference's refusals of a time step
    without an old velocity and the reverse."""
    import dataclasses
    import chuanflow_b200 as cf
    g = golden("simple_channel_dt.npz")
    mesh, case = K.channel_product(10, 6, 5)
    ctl = dataclasses.replace(K.controls_from(K.channel_case(10, 6, 5)), max_iterations=1, dt=0.05, u_time_old=1)
    for _ in range(int(g["iterations"])):
        res = case.solve(ctl)
        assert not res.diverged
    U, p, phi = case.download()
    for a, b, name in ((U, g["U"], "U"), (p, g["p"], "p"), (phi, g["phi"], "phi")):
        assert rel(a, b) < REL_TOL, (name, rel(a, b))
    assert abs(res.final_continuity_error - float(g["continuity"])) <= 1e-6 * abs(float(g["continuity"]))
    with pytest.raises(cf.CfgError, match="no velocity at the previous time level"):
        case.solve(dataclasses.replace(ctl, u_time_old=0))
    with pytest.raises(cf.CfgError, match="no time step"):
        case.solve(dataclasses.replace(ctl, dt=0.0))


@pytest.mark.parametrize("cells,jitter,pin,iters", [((8, 8, 8), 0.0, -1, 5), ((12, 12, 12), 0.1, 0, 8)])
def test_simple_cavity_matches_oracle(cells, jitter, pin, iters):
    """The lid-driven cavity: orthogonal (the reference's own set-up) and
    jittered with a pressure reference cell."""
    oc = K.cavity_case(*cells, jitter=jitter, iters=iters, linear_tol=1e-10, nu=0.0025)
    oc.p_ref_cell = pin
    U0, p0, phi0, r0 = oc.run()
    mesh, case = K.cavity_product(*cells, jitter=jitter)
    res = case.solve(K.controls_from(oc))
    U, p, phi = case.download()
    assert res.iterations == r0.iterations
    assert rel(U, U0) < REL_TOL, rel(U, U0)
    assert rel(p - p.mean(), p0 - p0.mean()) < REL_TOL, rel(p - p.mean(), p0 - p0.mean())
    assert rel(phi, phi0) < REL_TOL, rel(phi, phi0)


@pytest.mark.parametrize("fixture,method", [("solve_cg.npz", "cg"), ("solve_bicgstab.npz", "bicgstab")])
def test_sparse_solvers_match_reference(golden, fixture, method):
    import chuanflow_b200 as cf
    g = golden(fixture)
    fn = cf.solve_cg if method == "cg" else cf.solve_bicgstab
    x, rep = fn(g["row_start"], g["cols"], g["vals"], g["b"], g["x0"], float(g["tol"]), int(g["max_iter"]))
    assert rep.converged == bool(g["converged"])
    assert abs(rep.iterations - int(g["iterations"])) <= 1
    assert rel(x, g["x"]) < 1e-9
    assert rep.initial_residual == float(g["initial"])


@pytest.mark.parametrize("order", ["identity", "colour", "rcm-colour"])
def test_dic_factor_and_apply_bit_exact(golden, order):
    """The multicolour DIC of the device pressure matrix equals the oracle's
    restatement of the same definition (oracle/cfo.c) on the same matrix, in
    any device cell numbering."""
    g = golden("eqns_cavity.npz")
    mesh, case = K.cavity_product(6, 5, 4, order=order)
    case.upload(g["in_U"], g["in_p"], g["in_phi"])
    oc = K.cavity_case(6, 5, 4)
    out = case.probe_equations(K.controls_from(oc), g["in_xprobe"])
    rs, cols, vals = oc.pressure_csr(out["rAUf"])
    colour, nc, rdinv, apply = O.dic(rs, cols, vals)
    r = np.random.default_rng(3).normal(size=mesh.n_cells)
    z, rd, ncol = case.probe_dic(r)
    assert ncol == nc == 2
    assert np.array_equal(rd, rdinv)
    assert np.array_equal(z, apply(r))


@pytest.mark.parametrize("cells,jitter", [((12, 12, 12), 0.1), ((9, 7, 5), 0.0)])
def test_simple_cavity_dic_matches_oracle(cells, jitter):
    oc = K.cavity_case(*cells, jitter=jitter, iters=6, linear_tol=1e-10, nu=0.0025)
    oc.p_ref_cell = 0
    oc.p_precond = 1
    U0, p0, phi0, r0 = oc.run()
    mesh, case = K.cavity_product(*cells, jitter=jitter)
    res = case.solve(K.controls_from(oc, p_preconditioner="DIC"))
    U, p, phi = case.download()
    assert res.iterations == r0.iterations
    assert abs(res.p_inner_iterations - r0.pItersTotal) <= 2 * 6 * 2
    assert rel(U, U0) < REL_TOL and rel(p, p0) < REL_TOL and rel(phi, phi0) < REL_TOL


def test_simple_cavity_amg_pressure_matches_oracle():
    """SIMPLE with the FP32-AMG flexible-CG pressure solve against the
    oracle's DIC run: the pressure solves stop at the same 1e-10 infinity-norm
    test, so the outer iterations agree to the SIMPLE bar."""
    oc = K.cavity_case(10, 9, 8, jitter=0.1, iters=6, linear_tol=1e-10, nu=0.0025)
    oc.p_ref_cell = 0
    oc.p_precond = 1
    U0, p0, phi0, r0 = oc.run()
    mesh, case = K.cavity_product(10, 9, 8, jitter=0.1)
    res = case.solve(K.controls_from(oc, p_preconditioner="AMG"))
    U, p, phi = case.download()
    assert res.iterations == r0.iterations
    assert res.p_inner_iterations * 2 < r0.pItersTotal, (res.p_inner_iterations, r0.pItersTotal)
    assert rel(U, U0) < REL_TOL and rel(p, p0) < REL_TOL and rel(phi, phi0) < REL_TOL


@pytest.mark.parametrize("order", ["colour", "rcm-colour"])
@pytest.mark.parametrize("method", ["jacobi64", "dic64", "ir32"])
def test_poisson_solves_match_oracle(method, order):
    """The pressure-Poisson study system (unit face coefficient, Neumann,
    one reference cell) on a Delaunay tet mesh: every method reaches the
    requested FP64 true residual and the oracle's FP64 solution."""
    from chuanflow_b200 import meshgen
    mesh, pts, tets = meshgen.tet_mesh(10, 0.1, 2)
    import chuanflow_b200 as cf
    case = cf.SimpleCase(mesh, order=order)
    case.poisson_setup(ref_cell=0)
    rng = np.random.default_rng(1)
    b = rng.normal(size=mesh.n_cells)
    b -= b.mean()
    x, rep = case.poisson_solve(b, method, tol=1e-10)
    assert rep["converged"] and rep["true_rel_residual"] <= 1e-10
    a = mesh.addressing()
    om = O.OMesh(a["points"], a["face_offsets"], a["face_verts"], a["owner"], a["neighbour"],
                 [p[0] for p in mesh.patches], [p[1] for p in mesh.patches], [p[2] for p in mesh.patches],
                 [p[3] for p in mesh.patches])
    oc = O.Case(om, u_type=["fixedValue"] * mesh.n_patches, u_value=[(0, 0, 0)] * mesh.n_patches,
                p_type=["zeroGradient"] * mesh.n_patches, p_value=[0] * mesh.n_patches, nu=1.0)
    oc.p_ref_cell = 0
    rs, cols, vals = oc.pressure_csr(np.ones(mesh.n_faces))
    x0, r0 = O.solve("cg", rs, cols, vals, b, np.zeros(mesh.n_cells), 1e-15, 20000)
    assert rel(x, x0) < 1e-7, rel(x, x0)


def test_full_size_cavity_matches_oracle_checksums(golden):
    """The 2M-cell jittered cavity of bench.py (128^3, pressure reference cell
    0) after one outer iteration from rest, against the C restatement's run
    (the reference itself has no reference cell): inner iteration counts,
    continuity, field checksums and 4096 seeded cell and face samples."""
    import bench
    g = golden("simple_cavity128.npz")
    mesh, case, ctl = bench.make_cavity_case(int(g["n"]), 0, "Jacobi")
    assert np.array_equal(mesh.addressing()["points"].sum(0), g["points_sum"])
    ctl.max_iterations = int(g["iters"])
    ctl.linear_tol = float(g["linear_tol"])
    r = case.solve(ctl)
    U, p, phi = case.download()
    assert r.iterations == int(g["iterations"])
    assert abs(r.final_continuity_error - float(g["continuity"])) <= 1e-6 * abs(float(g["continuity"]))
    # checksums relative to the sums of magnitudes (the recirculating flow's
    # signed sums nearly cancel)
    assert np.all(np.abs(U.sum(0) - g["U_sum"]) <= REL_TOL * np.abs(U).sum(0))
    assert abs(p.sum() - g["p_sum"]) <= REL_TOL * np.abs(p).sum()
    assert abs(np.abs(phi).sum() - g["phi_abs_sum"]) <= REL_TOL * g["phi_abs_sum"]
    assert rel(U[g["cells"]], g["U_cells"]) < REL_TOL
    assert rel(p[g["cells"]], g["p_cells"]) < REL_TOL
    assert rel(phi[g["faces"]], g["phi_faces"]) < REL_TOL
    # the inner counts: the solves stop where a 2M-term dot product crosses
    # the tolerance, so a different summation order moves them a little
    assert abs(r.u_inner_iterations - int(g["u_inner"])) <= 0.1 * int(g["u_inner"])
    assert abs(r.p_inner_iterations - int(g["p_inner"])) <= 0.1 * int(g["p_inner"])


def channel40_product(schemes=None):
    import chuanflow_b200 as cf
    mesh = cf.PolyMesh.block((0, 0, 0), (2.0, 0.1, 0.1), (40, 20, 20),
                             {s: (n, t) for s, n, t in zip(K.SIDES, K.CHANNEL_NAMES, K.CHANNEL_TYPES)})
    case = cf.SimpleCase(mesh, 0, schemes)
    case.set_patch_bc("U", "inlet", "fixedValue", (0.1, 0, 0))
    case.set_patch_bc("p", "inlet", "zeroGradient", 0.0)
    case.set_patch_bc("U", "outlet", "zeroGradient", (0, 0, 0))
    case.set_patch_bc("p", "outlet", "fixedValue", 0.0)
    for n in ("bottom", "top", "front", "back"):
        case.set_patch_bc("U", n, "fixedValue", (0, 0, 0))
        case.set_patch_bc("p", n, "zeroGradient", 0.0)
    case.init_flux()
    return mesh, case


def test_config1_channel_matches_reference(golden):
    """The 16,000-cell channel (40x20x20, 2 x 0.1 x 0.1 m, Re 100) for all
    300 outer iterations of the workload at the reference's stable
    relaxation, against its own run of them."""
    import chuanflow_b200 as cf
    g = golden("simple_channel40.npz")
    mesh, case = channel40_product()
    ctl = cf.SimpleControls(max_iterations=int(g["iters"]), relax_u=0.9, relax_p=0.03, p_relax_start=0.02,
                            non_orth_correctors=2, linear_tol=1e-10, nu=1e-4)
    r = case.solve(ctl)
    U, p, phi = case.download()
    assert r.iterations == int(g["ref_iterations"])
    assert abs(r.final_continuity_error - float(g["ref_continuity"])) <= 1e-6 * float(g["ref_continuity"])
    assert rel(U[g["cells"]], g["ref_U_cells"]) < REL_TOL and rel(p[g["cells"]], g["ref_p_cells"]) < REL_TOL
    assert rel(phi[g["faces"]], g["ref_phi_faces"]) < REL_TOL
    assert np.all(np.abs(U.sum(0) - g["ref_U_sum"]) <= REL_TOL * np.abs(U).sum(0))


def test_config1_linear_upwind_dic_matches_oracle(golden):
    """The same channel as the workload names it -- linear-upwind convection,
    Gauss linear gradients, relaxation 0.7 / 0.3, DIC-PCG to 1e-8 -- against
    the C restatement (no reference counterpart)."""
    import chuanflow_b200 as cf
    g = golden("simple_channel40.npz")
    mesh, case = channel40_product(cf.Schemes(div="linearUpwind", grad="linear"))
    ctl = cf.SimpleControls(max_iterations=int(g["lu_iters"]), relax_u=0.7, relax_p=0.3, p_relax_start=0.02,
                            non_orth_correctors=2, linear_tol=1e-8, nu=1e-4, p_preconditioner="DIC")
    r = case.solve(ctl)
    U, p, phi = case.download()
    assert r.iterations == int(g["lu_iterations"])
    assert rel(U[g["cells"]], g["lu_U_cells"]) < REL_TOL and rel(p[g["cells"]], g["lu_p_cells"]) < REL_TOL
    assert rel(phi[g["faces"]], g["lu_phi_faces"]) < REL_TOL


def test_poiseuille_verification_case_converges_like_the_reference(golden, tmp_path):
    """The reference's own converged-state check (tests/check_poiseuille.py
    on tests/cases/poiseuilleChannel): its case file run end to end through
    cfg_run_case_file to the outer stop of its simple{} block stops at the
    reference's iteration, with U, p and phi within the FP64 bar of the
    reference's run, and passes the check's bands -- |v| < 5e-3 downstream,
    the parabola within 0.012, the centreline within 8% and the column flux
    within 2%."""
    import chuanflow_b200 as cf
    g = golden("poiseuille.npz")
    path = tmp_path / "case.dict"
    path.write_text(K.poiseuille_dict())
    res, counts, (U, p, phi) = cf.run_case_file(path, fields=True)
    assert res.converged and not res.diverged
    assert res.iterations == int(g["iterations"])
    assert rel(U, g["U"]) < REL_TOL and rel(p, g["p"]) < REL_TOL and rel(phi, g["phi"]) < REL_TOL
    mesh = cf.PolyMesh.block((0, 0, 0), (4.0, 0.2, 0.1), (100, 20, 1))
    b = K.poiseuille_bands(mesh.geometry()["C"], U)
    assert b["column"] == 20
    assert b["v_max"] < 5e-3 and b["profile_err"] < 0.012
    assert abs(b["centreline"] / 0.15 - 1.0) < 0.08 and b["flux_err"] < 0.02


@pytest.mark.parametrize("theta", [0.0, 0.25])
def test_headline_amg_pressure_fields_match_fp64_oracle(theta):
    """The headline's configuration (bench.make_case: the jittered channel,
    the reference's channel relaxation, nonOrth 1, tolerance 1e-8) at 64 x 8
    x 8 cells, with the FP32-AMG flexible-CG pressure solve (its hierarchy
    aggregated plainly, theta 0, or by strength of connection, theta 0.25),
    over 12 outer iterations from rest, against the C restatement's FP64
    DIC-PCG run of the same iterations: every field within the FP64 bar
    (relative L2) and no iteration diverged."""
    import bench
    n, iters = 8, 12
    m = K._block((0, 0, 0), bench.LENGTH, bench.dims(n), K.CHANNEL_NAMES, K.CHANNEL_TYPES, bench.JITTER, bench.SEED)
    oc = O.Case(m, u_type=["fixedValue", "zeroGradient"] + ["fixedValue"] * 4,
                u_value=[(bench.U_IN, 0, 0)] + [(0, 0, 0)] * 5, p_type=["zeroGradient", "fixedValue"] +
                ["zeroGradient"] * 4, p_value=[0] * 6, nu=bench.NU, max_iterations=iters, linear_tol=1e-8,
                non_orth=1, **bench.RELAX)
    oc.p_precond = 1
    U0, p0, phi0, r0 = oc.run()
    mesh, case, ctl = bench.make_case(n, 0, "AMG", theta)
    assert np.array_equal(mesh.addressing()["points"], m.points)
    for k in range(iters):
        r = case.solve(ctl)
        assert not r.diverged, k
    U, p, phi = case.download()
    errs = {"U": rel(U, U0), "p": rel(p, p0), "phi": rel(phi, phi0)}
    assert all(v < REL_TOL for v in errs.values()), errs


def test_simple_cavity_mixed_precision_pressure_matches_fp64_oracle():
    """SIMPLE with the mixed-precision pressure solve (the matrix rounded to
    FP32, FP32 DIC-PCG corrections inside FP64 iterative refinement whose
    residual and infinity-norm test are FP64) against the oracle's FP64
    DIC run of the same outer iterations.  The refinement stops on the same
    FP64 test, so every field stays within the FP64 bar; stated per field:
    U, p and phi each within 1e-6 relative L2."""
    oc = K.cavity_case(12, 11, 10, jitter=0.1, iters=6, linear_tol=1e-10, nu=0.0025)
    oc.p_ref_cell = 0
    oc.p_precond = 1
    U0, p0, phi0, r0 = oc.run()
    mesh, case = K.cavity_product(12, 11, 10, jitter=0.1)
    res = case.solve(K.controls_from(oc, p_preconditioner="IR32"))
    U, p, phi = case.download()
    assert res.iterations == r0.iterations and not res.diverged
    assert rel(U, U0) < 1e-6, rel(U, U0)
    assert rel(p, p0) < 1e-6, rel(p, p0)
    assert rel(phi, phi0) < 1e-6, rel(phi, phi0)


def test_headline_amg_momentum_fields_match_fp64_oracle():
    """The headline channel at 64 x 8 x 8 with both linear solves
    preconditioned by FP32 AMG V-cycles inside FP64 Krylov loops (flexible CG
    for the pressure; BiCGStab with M = the momentum matrix's V-cycle for the
    three velocity components) over 12 outer iterations from rest, against
    the C restatement's FP64 run (Jacobi-BiCGStab, DIC-PCG): each solve stops
    on the reference's FP64 |r|inf / |b|inf < 1e-8 test, so every field stays
    within the FP64 bar; the momentum solves take fewer BiCGStab iterations
    than with the reference's Jacobi preconditioner."""
    import bench
    n, iters = 8, 12
    m = K._block((0, 0, 0), bench.LENGTH, bench.dims(n), K.CHANNEL_NAMES, K.CHANNEL_TYPES, bench.JITTER, bench.SEED)
    oc = O.Case(m, u_type=["fixedValue", "zeroGradient"] + ["fixedValue"] * 4,
                u_value=[(bench.U_IN, 0, 0)] + [(0, 0, 0)] * 5, p_type=["zeroGradient", "fixedValue"] +
                ["zeroGradient"] * 4, p_value=[0] * 6, nu=bench.NU, max_iterations=iters, linear_tol=1e-8,
                non_orth=1, **bench.RELAX)
    oc.p_precond = 1
    U0, p0, phi0, r0 = oc.run()
    inner = {}
    for up in ("Jacobi", "AMG"):
        mesh, case, ctl = bench.make_case(n, 0, "AMG")
        ctl = dataclasses.replace(ctl, u_preconditioner=up)
        inner[up] = 0
        for k in range(iters):
            r = case.solve(ctl)
            assert not r.diverged, k
            inner[up] += r.u_inner_iterations
        U, p, phi = case.download()
        errs = {"U": rel(U, U0), "p": rel(p, p0), "phi": rel(phi, phi0)}
        assert all(v < REL_TOL for v in errs.values()), (up, errs)
    assert inner["AMG"] < inner["Jacobi"], inner
