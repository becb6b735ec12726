"""Test infrastructure: a numpy restatement of chuanflow_b200/csrc/amg.cu,
the aggregation-AMG V-cycle the GPU applies as the pressure preconditioner
(no reference counterpart).  Same aggregation (rows in order, entries in
row order; plain, or over the strong entries only), Galerkin sums in FP64
stored in FP32, FP32 damped Jacobi with
w = 0.8, coarse correction scaled by 2.0, coarsest level (<= 128 rows)
inverted densely with a 1e-6 max|diag| shift."""
import numpy as np
import scipy.sparse as sp

OMEGA = np.float32(0.8)
SCALE = np.float32(2.0)
DENSE_MAX = 128


def strong_entries(A, theta):
    """Per CSR entry: the diagonal, or |a_ij| >= theta * max_{k != i} |a_ik|."""
    ip, ind, val = A.indptr, A.indices, A.data
    link = np.zeros(ind.size, bool)
    for i in range(A.shape[0]):
        cs, vs = ind[ip[i]:ip[i + 1]], np.abs(val[ip[i]:ip[i + 1]])
        off = cs != i
        mx = vs[off].max() if off.any() else 0.0
        link[ip[i]:ip[i + 1]] = (cs == i) | (vs >= theta * mx)
    return link


def aggregate(A, theta=0.0):
    """Plain aggregation over every entry, or (theta > 0) over the strong
    entries only, falling back to plain when that coarsens by less than half."""
    n = A.shape[0]
    ip, ind = A.indptr, A.indices
    link = strong_entries(A, theta) if theta > 0 else np.ones(ind.size, bool)
    agg = -np.ones(n, np.int64)
    na = 0
    for i in range(n):
        if agg[i] >= 0:
            continue
        nb = ind[ip[i]:ip[i + 1]][link[ip[i]:ip[i + 1]]]
        if (agg[nb] >= 0).any():
            continue
        agg[nb] = na
        agg[i] = na
        na += 1
    for i in range(n):
        if agg[i] >= 0:
            continue
        for j, on in zip(ind[ip[i]:ip[i + 1]], link[ip[i]:ip[i + 1]]):
            if on and agg[j] >= 0 and j != i:
                agg[i] = agg[j]
                break
        if agg[i] < 0:
            agg[i] = na
            na += 1
    if theta > 0 and na > n // 2:
        return aggregate(A, 0.0)
    return agg, na


class Hierarchy:
    def __init__(self, A, theta=0.0):
        """A: the FP64 CSR operator (rows in device order, columns ascending);
        theta: the strength threshold of the aggregation (0: plain)."""
        self.levels = []
        cur = A.tocsr()
        cur.sort_indices()
        first = True
        while first or cur.shape[0] > DENSE_MAX:
            first = False
            agg, na = aggregate(cur, theta)
            n = cur.shape[0]
            P = sp.csr_matrix((np.ones(n), (np.arange(n), agg)), shape=(n, na))
            coarse = (P.T @ cur @ P).tocsr()
            coarse.sort_indices()
            self.levels.append({"A": cur.astype(np.float32), "dinv": (1.0 / cur.diagonal()).astype(np.float32),
                                "agg": agg, "P": P.astype(np.float32)})
            cur = coarse
        n = cur.shape[0]
        m = cur.toarray()
        m[np.diag_indices(n)] += 1e-6 * np.abs(cur.diagonal()).max()
        self.dense = np.linalg.inv(m).astype(np.float32)
        self.rows = [lv["A"].shape[0] for lv in self.levels] + [n]

    def apply(self, r, level=0):
        if level == len(self.levels):
            return self.dense @ r.astype(np.float32)
        lv = self.levels[level]
        A, dinv, P = lv["A"], lv["dinv"], lv["P"]
        b = r.astype(np.float32)
        x = OMEGA * dinv * b
        res = b - A @ x
        xc = self.apply(P.T @ res, level + 1)
        y = x + SCALE * (P @ xc)
        return y + OMEGA * dinv * (b - A @ y)
