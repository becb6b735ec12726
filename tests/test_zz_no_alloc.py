"""cfg_pcg_solve_static: the allocation-free Jacobi-PCG entry point.

Some callers cannot let a library allocate device memory: a solver living
inside a host framework that has already reserved the whole GPU for its own
memory manager, or one that runs beside other streams and cannot absorb the
device-wide synchronisation cudaMalloc and cudaFree imply.  This entry point
takes a CSR matrix and vectors the caller already holds on the device and
keeps its own work vectors in a static device array of the library.

The test calls it through the C ABI, twice in a row on different systems,
and checks each answer against the existing cfg_sparse_solve (which copies
host arrays to memory it allocates) to 1e-10 relative L2, with the same
iteration count; the second system is the reference's own CG fixture
(solve_cg.npz, from src/common/src/Matrix.cpp:153-222 run on the host), whose
stored solution the answer must also match.  Its device buffers are allocated here, by the test; the
entry point itself allocates nothing.  This file is collected last so a run
that stops at its first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

import _cases as K

pytestmark = pytest.mark.gpu

REL_TOL = 1e-10
MAX_ROWS = 1 << 18


def poisson_csr(nx, ny, nz, shift):
    """A 7-point Laplacian with a diagonal shift, CSR with sorted columns."""
    n = nx * ny * nz
    rs, cols, vals = [0], [], []
    for k in range(nz):
        for j in range(ny):
            for i in range(nx):
                r = i + nx * (j + ny * k)
                row = {r: 6.0 + shift}
                for di, dj, dk in ((-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)):
                    a, b, c = i + di, j + dj, k + dk
                    if 0 <= a < nx and 0 <= b < ny and 0 <= c < nz:
                        row[a + nx * (b + ny * c)] = -1.0
                for cc in sorted(row):
                    cols.append(cc)
                    vals.append(row[cc])
                rs.append(len(cols))
    return np.array(rs, np.int64), np.array(cols, np.int64), np.array(vals), n


def solve_static(rs, cols, vals, b, x0, tol, max_iter):
    import torch
    import chuanflow_b200 as cf
    lib = cf.lib()
    dev = torch.device("cuda:0")
    t_rs = torch.from_numpy(rs.astype(np.int32)).to(dev)
    t_cols = torch.from_numpy(cols.astype(np.int32)).to(dev)
    t_vals = torch.from_numpy(vals).to(dev)
    t_b = torch.from_numpy(b).to(dev)
    t_x = torch.from_numpy(x0.copy()).to(dev)
    torch.cuda.synchronize()
    rep = cf._capi._Report()
    vp = C.c_void_p
    rc = lib.cfg_pcg_solve_static(C.c_int32(0), C.c_int64(rs.size - 1), vp(t_rs.data_ptr()), vp(t_cols.data_ptr()),
                                  vp(t_vals.data_ptr()), vp(t_b.data_ptr()), vp(t_x.data_ptr()), C.c_double(tol),
                                  C.c_int32(max_iter), None, C.byref(rep))
    if rc != 0:
        raise cf.CfgError(rc, cf._capi._err())
    torch.cuda.synchronize()
    return t_x.cpu().numpy(), rep


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


def test_static_pcg_matches_sparse_solve_twice(golden):
    import chuanflow_b200 as cf
    rng = np.random.default_rng(5)
    big = poisson_csr(40, 30, 25, 0.05)
    g = golden("solve_cg.npz")
    small = (g["row_start"], g["cols"], g["vals"], g["row_start"].size - 1)
    for (rs, cols, vals, n), tol in ((big, 1e-10), (small, 1e-12)):
        b = rng.normal(size=n)
        x0 = np.zeros(n)
        x_ref, r_ref = cf.solve_cg(rs, cols, vals, b, x0, tol, 2000)
        x, rep = solve_static(rs, cols, vals, b, x0, tol, 2000)
        assert rep.converged and r_ref.converged
        assert abs(rep.iterations - r_ref.iterations) <= 1
        assert rel(x, x_ref) < REL_TOL, rel(x, x_ref)
    # the reference's own solve of its fixture, from its right-hand side and
    # initial guess
    rs, cols, vals, n = small
    x, rep = solve_static(rs, cols, vals, g["b"], g["x0"], float(g["tol"]), int(g["max_iter"]))
    assert rep.converged == bool(g["converged"])
    assert abs(rep.iterations - int(g["iterations"])) <= 1
    assert rel(x, g["x"]) < 1e-9, rel(x, g["x"])


def test_static_pcg_rejects_oversized_systems():
    import chuanflow_b200 as cf
    lib = cf.lib()
    rep = cf._capi._Report()
    one = C.c_void_p(1)  # never dereferenced: the size check comes first
    rc = lib.cfg_pcg_solve_static(C.c_int32(0), C.c_int64(MAX_ROWS + 1), one, one, one, one, one, C.c_double(1e-8),
                                  C.c_int32(10), None, C.byref(rep))
    assert rc == 1
    assert "static scratch holds" in cf._capi._err()
