"""The FP32 aggregation-AMG preconditioner (chuanflow_b200/csrc/amg.cu) on
the pressure-Poisson study system of a Delaunay tet mesh, against the numpy
restatement in tests/_amg_ref.py: the same hierarchy (levels and rows), one
V-cycle within FP32 accuracy, and the FP64 flexible CG it preconditions
reaching the requested true residual and the oracle's solution, in a small
fraction of the Jacobi-PCG iterations."""
import numpy as np
import pytest
import scipy.sparse as sp

import _amg_ref as R
import _oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def _system(n=12, seed=2):
    import chuanflow_b200 as cf
    from chuanflow_b200 import meshgen
    mesh, pts, tets = meshgen.tet_mesh(n, 0.1, seed)
    case = cf.SimpleCase(mesh)
    case.poisson_setup(ref_cell=0)
    a = mesh.addressing()
    om = O.OMesh(a["points"], a["face_offsets"], a["face_verts"], a["owner"], a["neighbour"],
                 [p[0] for p in mesh.patches], [p[1] for p in mesh.patches], [p[2] for p in mesh.patches],
                 [p[3] for p in mesh.patches])
    oc = O.Case(om, u_type=["fixedValue"] * mesh.n_patches, u_value=[(0, 0, 0)] * mesh.n_patches,
                p_type=["zeroGradient"] * mesh.n_patches, p_value=[0] * mesh.n_patches, nu=1.0)
    oc.p_ref_cell = 0
    rs, cols, vals = oc.pressure_csr(np.ones(mesh.n_faces))
    A = sp.csr_matrix((vals, cols, rs), shape=(mesh.n_cells, mesh.n_cells))
    return mesh, case, A, (rs, cols, vals)


def test_amg_hierarchy_and_vcycle_match_restatement():
    mesh, case, A, _ = _system()
    info = case.poisson_amg_setup()
    H = R.Hierarchy(A)
    assert info["levels"] == len(H.rows)
    assert info["rows"] == H.rows[:8]
    rng = np.random.default_rng(3)
    for _ in range(2):
        r = rng.standard_normal(mesh.n_cells)
        z = case.poisson_amg_apply(r)
        assert rel(z, H.apply(r).astype(np.float64)) < 1e-4


@pytest.mark.parametrize("method", ["fcg_amg", "fcg_amg_mpnn"])
def test_fcg_amg_reaches_oracle_solution(method):
    mesh, case, A, (rs, cols, vals) = _system()
    if method == "fcg_amg_mpnn":
        case.mpnn_create(layers=2, seed=1)
    rng = np.random.default_rng(1)
    b = rng.standard_normal(mesh.n_cells)
    b -= b.mean()
    x, rep = case.poisson_solve(b, method, tol=1e-10)
    assert rep["converged"] and rep["true_rel_residual"] <= 1e-10
    x0, r0 = O.solve("cg", rs, cols, vals, b, np.zeros(mesh.n_cells), 1e-15, 20000)
    assert rel(x, x0) < 1e-7
    if method == "fcg_amg":
        # the V-cycle alone: no fallback, a fraction of Jacobi-PCG's iterations
        assert rep["outer_iterations"] == 1
        _, jac = case.poisson_solve(b, "jacobi64", tol=1e-10)
        assert rep["inner_iterations"] * 4 < jac["inner_iterations"], (rep["inner_iterations"],
                                                                       jac["inner_iterations"])


def test_three_vector_vcycle_equals_single_vcycles():
    """The V-cycle the AMG momentum BiCGStab applies (three right-hand sides
    over one matrix read) gives each component the single V-cycle's result
    bit for bit, and leaves a component flagged done untouched."""
    mesh, case, A, _ = _system()
    case.poisson_amg_setup()
    rng = np.random.default_rng(7)
    r3 = rng.standard_normal((3, mesh.n_cells))
    z3 = case.poisson_amg_apply3(r3)
    for q in range(3):
        assert np.array_equal(z3[q], case.poisson_amg_apply(r3[q])), q
    keep = rng.standard_normal((3, mesh.n_cells))
    z3b = case.poisson_amg_apply3(r3, keep, done=(0, 1, 0))
    assert np.array_equal(z3b[1], keep[1])
    assert np.array_equal(z3b[0], z3[0]) and np.array_equal(z3b[2], z3[2])


def test_vcycle_with_sell_levels_matches_restatement():
    """Coarse levels of 32768 rows or more run their sweeps one thread per
    row on a SELL-32 copy of their operator, each row summed in its column
    order.  On a 444k-tet Poisson system (first coarse level about 64k rows)
    the three-vector V-cycle equals the single one bit for bit; one V-cycle
    agrees with the numpy restatement within 1e-3 relative, the size of the
    FP32 conditioning here (the restatement's own output moves by 5.9e-4
    when its finest FP32 values are perturbed by one part in 1.6e7); and the
    flexible CG it preconditions reaches a 1e-10 true residual in the
    V-cycle's usual count of iterations, a fraction of Jacobi-PCG's."""
    mesh, case, A, (rs, cols, vals) = _system(n=40, seed=4)
    info = case.poisson_amg_setup()
    assert info["rows"][1] >= 32768, info["rows"]
    H = R.Hierarchy(A)
    assert info["rows"] == H.rows[:8]
    rng = np.random.default_rng(11)
    r3 = rng.standard_normal((3, mesh.n_cells))
    r3 -= r3.mean(axis=1, keepdims=True)
    z3 = case.poisson_amg_apply3(r3)
    for q in range(3):
        z = case.poisson_amg_apply(r3[q])
        assert np.array_equal(z3[q], z), q
        assert rel(z, H.apply(r3[q]).astype(np.float64)) < 1e-3
    x, rep = case.poisson_solve(r3[0], "fcg_amg", tol=1e-10)
    assert rep["converged"] and rep["true_rel_residual"] <= 1e-10 and rep["outer_iterations"] == 1
    _, jac = case.poisson_solve(r3[0], "jacobi64", tol=1e-10)
    assert rep["inner_iterations"] * 4 < jac["inner_iterations"], (rep["inner_iterations"], jac["inner_iterations"])


def _channel_poisson(theta, cells=(96, 12, 12)):
    """The Poisson system of the jittered channel with the headline's cell
    aspect (2.5x longer than wide: couplings across 6.25x those along),
    fixed p at the outlet, with the pressure hierarchy aggregated at theta."""
    import _cases as K
    L = (2.0, 0.1, 0.1)
    mesh, case = K.channel_product(*cells, jitter=0.1, seed=7, L=L)
    if theta:
        case.amg_strength(theta)
    case.poisson_setup()
    oc = K.channel_case(*cells, jitter=0.1, seed=7, L=L)
    rs, cols, vals = oc.pressure_csr(np.ones(mesh.n_faces))
    return mesh, case, sp.csr_matrix((vals, cols, rs), shape=(mesh.n_cells, mesh.n_cells))


def test_strength_hierarchy_matches_restatement_and_cuts_iterations():
    """Strength-of-connection aggregation (theta 0.25) on the anisotropic
    channel: the device hierarchy has the restatement's levels and rows, one
    V-cycle agrees within FP32 accuracy, and the flexible CG it preconditions
    reaches a 1e-10 true residual in fewer iterations than with the plain
    hierarchy; the threshold is fixed once the hierarchy is built."""
    import chuanflow_b200 as cf
    mesh, case, A = _channel_poisson(0.25)
    info = case.poisson_amg_setup()
    H = R.Hierarchy(A, 0.25)
    assert info["levels"] == len(H.rows) and info["rows"] == H.rows[:8], (info, H.rows)
    assert info["rows"] != R.Hierarchy(A).rows[:8]
    rng = np.random.default_rng(5)
    r = rng.standard_normal(mesh.n_cells)
    assert rel(case.poisson_amg_apply(r), H.apply(r).astype(np.float64)) < 1e-4
    r3 = rng.standard_normal((3, mesh.n_cells))
    z3 = case.poisson_amg_apply3(r3)
    for q in range(3):
        assert np.array_equal(z3[q], case.poisson_amg_apply(r3[q])), q
    x, rep = case.poisson_solve(r, "fcg_amg", tol=1e-10)
    assert rep["converged"] and rep["true_rel_residual"] <= 1e-10
    case.amg_strength(0.25)  # the same threshold again is accepted
    with pytest.raises(cf.CfgError, match="built already"):
        case.amg_strength(0.5)
    _, plain, _ = _channel_poisson(0.0)
    x0, rep0 = plain.poisson_solve(r, "fcg_amg", tol=1e-10)
    assert rel(x, x0) < 1e-8
    assert 5 * rep["inner_iterations"] < 4 * rep0["inner_iterations"], (rep["inner_iterations"],
                                                                       rep0["inner_iterations"])
