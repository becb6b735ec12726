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
