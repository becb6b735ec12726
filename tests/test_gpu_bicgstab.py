"""Jacobi-BiCGStab on the device against the C restatement of
solveBiCGStab (Matrix.cpp:224-319) on matrices that reach each compiled row
width (rows of at most 7, 8 to 16 and more than 16 entries) and the tDenom
breakdown exit (t = A s^ = 0 after the first half step).

The device forms s^ per column inside its second SpMV and updates x once
per iteration; the bars are those of the reference's fixtures:
iteration counts within one (parallel dot products) and x within 1e-9
relative L2, and the breakdown case exactly.
"""
import numpy as np
import pytest

import _oracle as O

pytestmark = pytest.mark.gpu


def rel(a, b):
    nb = np.linalg.norm(b)
    return np.linalg.norm(a - b) / (nb if nb > 0 else 1.0)


def random_csr(n, lo, hi, seed):
    """Nonsymmetric, diagonally dominant rows of lo..hi entries (diagonal
    included), columns ascending as the reference's CSR build leaves them."""
    rng = np.random.default_rng(seed)
    rs, cols, vals = [0], [], []
    for i in range(n):
        k = int(rng.integers(lo, hi + 1)) - 1
        off = rng.choice(np.delete(np.arange(n), i), size=k, replace=False)
        c = np.sort(np.concatenate([off, [i]]))
        v = -rng.uniform(0.1, 1.0, size=c.size)
        v[c == i] = 0.0
        v[c == i] = np.abs(v).sum() * rng.uniform(1.05, 1.5)
        cols.extend(c.tolist())
        vals.extend(v.tolist())
        rs.append(len(cols))
    return np.array(rs, np.int64), np.array(cols, np.int64), np.array(vals)


@pytest.mark.parametrize("lo,hi", [(3, 7), (8, 16), (17, 24)])
def test_bicgstab_row_widths_match_oracle(lo, hi):
    import chuanflow_b200 as cf
    n = 3000
    rs, cols, vals = random_csr(n, lo, hi, seed=lo)
    rng = np.random.default_rng(99)
    b = rng.standard_normal(n)
    x0 = np.zeros(n)
    xo, ro = O.solve("bicgstab", rs, cols, vals, b, x0, 1e-10, 500)
    xd, rd = cf.solve_bicgstab(rs, cols, vals, b, x0, 1e-10, 500)
    assert ro.converged and rd.converged
    assert abs(rd.iterations - ro.iterations) <= 1
    assert rel(xd, xo) < 1e-9
    assert rd.initial_residual == ro.initialResidual


def test_bicgstab_breakdown_exit_matches_oracle():
    """A = D with power-of-two entries: v = A D^-1 r = r exactly, so alpha is
    1, s = 0 and tDenom = 0; the exit keeps x + alpha z = b / D and reports
    |s|inf = 0 after one iteration."""
    import chuanflow_b200 as cf
    n = 1000
    rng = np.random.default_rng(5)
    d = 2.0 ** rng.integers(-2, 3, size=n)
    rs = np.arange(n + 1, dtype=np.int64)
    cols = np.arange(n, dtype=np.int64)
    b = rng.standard_normal(n)
    x0 = np.zeros(n)
    xo, ro = O.solve("bicgstab", rs, cols, d, b, x0, 1e-12, 50)
    xd, rd = cf.solve_bicgstab(rs, cols, d, b, x0, 1e-12, 50)
    assert (ro.iterations, bool(ro.converged), ro.finalResidual) == (1, True, 0.0)
    assert (rd.iterations, rd.converged, rd.final_residual) == (1, True, 0.0)
    assert np.array_equal(xd, xo)
    assert np.array_equal(xd, b / d)
