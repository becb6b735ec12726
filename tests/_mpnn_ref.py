"""FP64 PyTorch (CPU) restatement of the learned pressure preconditioner:
the autograd oracle its device forward and backward kernels are checked
against.  Test infrastructure only.

    s = rms(r); h0 = relu(w0 r/s + b0)
    per layer: m = C h (C_ij = -a_ij / a_ii off the diagonal),
               h += relu(bf(h) A^T + bf(m) B^T + b)
    z = r / diag(A) + s (h . wout)
    loss = |A z - r|^2 / |r|^2, or with a target t (A t = r) e.Ae / t.At, e = z - t
bf() rounds to BF16 (round to nearest even), the tensor cores' operands; its
gradient passes through unchanged.
Parameter layout: w0[32], b0[32], per layer A[32x32] (row = output unit),
B[32x32], b[32], then wout[32]."""
import numpy as np

H = 32


def off_layer(l):
    return 2 * H + l * (2 * H * H + H)


def n_params(L):
    return off_layer(L) + H


def bf16_round(w):
    """Round float32 values to bfloat16 (round to nearest even), as floats."""
    w = np.ascontiguousarray(w, np.float32)
    u = w.view(np.uint32).astype(np.uint64)
    lsb = (u >> 16) & 1
    u = ((u + 0x7FFF + lsb) >> 16) << 16
    return u.astype(np.uint32).view(np.float32)


def bf16_st(x):
    """x rounded to BF16 with a pass-through gradient."""
    import torch
    return x + (x.to(torch.bfloat16).to(torch.float64) - x).detach()


def loss_and_grad(rs, cols, vals, r, w, L, t=None):
    import torch
    n = rs.size - 1
    rows = np.repeat(np.arange(n), np.diff(rs))
    A = torch.sparse_coo_tensor(np.stack([rows, cols]), vals, (n, n), dtype=torch.float64).coalesce()
    diag = np.zeros(n)
    on = rows == cols
    np.add.at(diag, rows[on], vals[on])
    off = ~on
    Cm = torch.sparse_coo_tensor(np.stack([rows[off], cols[off]]), -vals[off] / diag[rows[off]], (n, n),
                                 dtype=torch.float64).coalesce()
    wt = torch.tensor(np.asarray(w, np.float64), requires_grad=True)
    rt = torch.tensor(r, dtype=torch.float64)
    dt = torch.tensor(diag, dtype=torch.float64)
    s = torch.sqrt((rt * rt).sum() / n)
    h = torch.relu((rt / s)[:, None] * wt[0:H][None, :] + wt[H:2 * H][None, :])
    for l in range(L):
        o = off_layer(l)
        Aw = wt[o:o + H * H].reshape(H, H)
        Bw = wt[o + H * H:o + 2 * H * H].reshape(H, H)
        b = wt[o + 2 * H * H:o + 2 * H * H + H]
        m = torch.sparse.mm(Cm, h)
        h = h + torch.relu(bf16_st(h) @ Aw.T + bf16_st(m) @ Bw.T + b)
    wout = wt[off_layer(L):off_layer(L) + H]
    z = rt / dt + s * (h @ wout)
    if t is None:
        res = torch.sparse.mm(A, z[:, None])[:, 0] - rt
        loss = (res * res).sum() / (rt * rt).sum()
    else:
        tt = torch.tensor(t, dtype=torch.float64)
        e = z - tt
        loss = (e * torch.sparse.mm(A, e[:, None])[:, 0]).sum() / (tt * torch.sparse.mm(A, tt[:, None])[:, 0]).sum()
    loss.backward()
    return float(loss), wt.grad.numpy(), z.detach().numpy()
