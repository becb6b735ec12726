"""The restatement of the AMG preconditioner (tests/_amg_ref.py, the checker
of the device V-cycle) on its own, on the CPU: on the pressure-Poisson
system of a small Delaunay tet mesh its hierarchy coarsens about 7x per
level down to at most 128 rows, and a flexible CG preconditioned by its
V-cycle reaches a 1e-10 relative residual in a fraction of Jacobi-PCG's
iterations (the oracle's solveCG restatement)."""
import numpy as np
import scipy.sparse as sp

import _amg_ref as R
import _oracle as O


def _system(n=10, seed=2):
    from chuanflow_b200 import meshgen
    mesh, pts, tets = meshgen.tet_mesh(n, 0.1, seed)
    a = mesh.addressing()
    om = O.OMesh(a["points"], a["face_offsets"], a["face_verts"], a["owner"], a["neighbour"],
                 [p[0] for p in mesh.patches], [p[1] for p in mesh.patches], [p[2] for p in mesh.patches],
                 [p[3] for p in mesh.patches])
    oc = O.Case(om, u_type=["fixedValue"] * mesh.n_patches, u_value=[(0, 0, 0)] * mesh.n_patches,
                p_type=["zeroGradient"] * mesh.n_patches, p_value=[0] * mesh.n_patches, nu=1.0)
    oc.p_ref_cell = 0
    rs, cols, vals = oc.pressure_csr(np.ones(mesh.n_faces))
    return sp.csr_matrix((vals, cols, rs), shape=(mesh.n_cells, mesh.n_cells)), (rs, cols, vals)


def fcg(A, b, M, tol, maxit=500):
    x = np.zeros_like(b)
    r = b.copy()
    z = M(r)
    p = z.copy()
    bn = np.linalg.norm(b)
    for it in range(1, maxit + 1):
        q = A @ p
        pq = p @ q
        alpha = (p @ r) / pq
        x += alpha * p
        r -= alpha * q
        if np.linalg.norm(r) / bn <= tol:
            return x, it
        z = M(r).astype(np.float64)
        p = z - (z @ q) / pq * p
    return x, maxit


def test_restated_amg_coarsens_and_preconditions():
    A, (rs, cols, vals) = _system()
    H = R.Hierarchy(A)
    assert H.rows[-1] <= R.DENSE_MAX
    for a, b in zip(H.rows, H.rows[1:]):
        assert 4 * b < a  # aggregates of several cells each
    rng = np.random.default_rng(1)
    b = rng.standard_normal(A.shape[0])
    b -= b.mean()
    x, it = fcg(A, b, lambda r: H.apply(r), 1e-10)
    assert np.linalg.norm(b - A @ x) / np.linalg.norm(b) <= 1e-10
    _, rep = O.solve("cg", rs, cols, vals, b, np.zeros(A.shape[0]), 1e-10, 20000)
    assert 4 * it < rep.iterations, (it, rep.iterations)


def _channel_system(cells=(96, 12, 12), jitter=0.1):
    """The pressure system of a jittered channel whose cells are 2.5x longer
    than wide (the 2M-cell channel's aspect): couplings across the channel
    6.25x those along it; fixed p at the outlet."""
    import _cases as K
    names = ["inlet", "outlet", "bottom", "top", "front", "back"]
    mn, mx = (0.0, 0.0, 0.0), (2.0, 0.1, 0.1)
    om = O.block_mesh(mn, mx, cells, names, ["wall"] * 6)
    om = om.with_points(K.jitter_points(om.points, cells, mn, mx, jitter, 7))
    np_ = len(names)
    oc = O.Case(om, u_type=["fixedValue"] * np_, u_value=[(0, 0, 0)] * np_,
                p_type=["fixedValue" if n == "outlet" else "zeroGradient" for n in names],
                p_value=[0] * np_, nu=1e-4)
    rs, cols, vals = oc.pressure_csr(np.ones(om.nF))
    return sp.csr_matrix((vals, cols, rs), shape=(om.nC, om.nC))


def test_strength_aggregation_follows_the_strong_couplings():
    A = _channel_system()
    plain, strong = R.Hierarchy(A), R.Hierarchy(A, 0.25)
    # theta 0 is plain aggregation
    assert R.Hierarchy(A, 0.0).rows == plain.rows
    agg0, _ = R.aggregate(A.tocsr(), 0.25)
    # every aggregate of the finest level lies within one cross-section
    # (cells of one x-index), since couplings along x are weak
    nx = 96
    xi = np.arange(A.shape[0]) % nx
    for a in np.unique(agg0)[:200]:
        assert np.ptp(xi[agg0 == a]) == 0
    rng = np.random.default_rng(4)
    b = rng.standard_normal(A.shape[0])
    _, it_plain = fcg(A, b, plain.apply, 1e-8)
    _, it_strong = fcg(A, b, strong.apply, 1e-8)
    assert 3 * it_strong < 2 * it_plain, (it_strong, it_plain)


def test_strength_aggregation_at_least_halves_every_level():
    # each row's largest coupling is always strong, so every first-phase
    # aggregate holds its root and at least one neighbour: even theta 1
    # (only the largest coupling kept) halves each level
    A = _channel_system((24, 6, 6))
    for theta in (0.25, 0.5, 1.0):
        rows = R.Hierarchy(A, theta).rows
        assert rows[-1] <= R.DENSE_MAX
        for a, b in zip(rows, rows[1:]):
            assert 2 * b <= a, (theta, rows)
