// Kernels of the SIMPLE path.  Every kernel that has a reference
// counterpart evaluates the same IEEE operations in the same order as the
// reference's serial loop for each output element (compiled with
// -fmad=false), so its results are bit-identical; the only differences left
// are the orders of the global dot-product reductions inside the linear
// solvers, which are deterministic tree reductions here.
#pragma once

#include "dev.cuh"

namespace cfg
{

/// Sparse matrix rows in SELL-32 layout: rows 32s..32s+31 form slice s; the
/// k-th entry of row 32s+l sits at start[s] + 32k + l; col < 0 pads.
struct DMat
{
    int n;
    const int* start;
    const int* col;
};

struct Grad3
{
    V3P g[3];
};
struct CGrad3
{
    CV3P g[3];
};

#define ROW_LOOP(c, n) for (int c = blockIdx.x * TPB + threadIdx.x; c < (n); c += gridDim.x * TPB)

// ---------------------------------------------------------------------------
// Gauss gradient (src/3d/src/discrete/gradScheme.cpp:15-96), gathered per
// cell over its faces in ascending face order, which is the order in which
// the reference's face loop adds into that cell.
// ---------------------------------------------------------------------------

/// Pass 0: V grad = sum_f Sf T_f.  Internal T_f: bounded owner weight
/// (quirk = 0: makeFaceValueFn, interpolate.cpp:334-355, and the corrected
/// scheme's reconstruction) or the volScalarField face value (quirk = 1,
/// volFields.cpp:96-111: the clamped owner-to-face fraction weights the owner).
template <int NC>
__global__ void __launch_bounds__(TPB) k_grad_gauss0(DMesh m, CV3P x, BcTab bc, int quirk, Grad3 out)
{
    ROW_LOOP(c, m.nC)
    {
        const int sl = c >> 5, lane = c & 31;
        double s[NC][3];
        double xc[NC];
#pragma unroll
        for (int q = 0; q < NC; ++q)
        {
            s[q][0] = s[q][1] = s[q][2] = 0.0;
            xc[q] = x.c[q][c];
        }
        const int e1 = m.cfStart[sl + 1];
        for (int e = m.cfStart[sl] + lane; e < e1; e += 32)
        {
            const int code = m.cfCode[e];
            if (code < 0) break;
            const int f = code >> 1, side = code & 1, other = m.cfOther[e];
            const double sx = m.sfx[f], sy = m.sfy[f], sz = m.sfz[f];
#pragma unroll
            for (int q = 0; q < NC; ++q)
            {
                double val;
                if (f < m.nI)
                {
                    const double xot = x.c[q][other];
                    const double xo = side ? xot : xc[q];
                    const double xn = side ? xc[q] : xot;
                    const double w = quirk ? m.wq[f] : m.ow[f];
                    val = w * xo + (1.0 - w) * xn;
                }
                else
                {
                    val = bc.c[q][other] * xc[q] + bc.k[q][other];
                }
                const double fx = sx * val, fy = sy * val, fz = sz * val;
                if (!side) { s[q][0] += fx; s[q][1] += fy; s[q][2] += fz; }
                else { s[q][0] -= fx; s[q][1] -= fy; s[q][2] -= fz; }
            }
        }
        const double v = m.V[c];
#pragma unroll
        for (int q = 0; q < NC; ++q)
        {
            out.g[q].c[0][c] = s[q][0] / v;
            out.g[q].c[1][c] = s[q][1] / v;
            out.g[q].c[2][c] = s[q][2] / v;
        }
    }
}

/// One skew-correction pass of the corrected scheme (gradScheme.cpp:59-95).
template <int NC>
__global__ void __launch_bounds__(TPB) k_grad_gauss_corr(DMesh m, CV3P x, BcTab bc, CGrad3 gin, Grad3 out)
{
    ROW_LOOP(c, m.nC)
    {
        const int sl = c >> 5, lane = c & 31;
        double s[NC][3];
        double xc[NC];
#pragma unroll
        for (int q = 0; q < NC; ++q)
        {
            s[q][0] = s[q][1] = s[q][2] = 0.0;
            xc[q] = x.c[q][c];
        }
        const int e1 = m.cfStart[sl + 1];
        for (int e = m.cfStart[sl] + lane; e < e1; e += 32)
        {
            const int code = m.cfCode[e];
            if (code < 0) break;
            const int f = code >> 1, side = code & 1, other = m.cfOther[e];
            const double sx = m.sfx[f], sy = m.sfy[f], sz = m.sfz[f];
            if (f < m.nI)
            {
                const int o = side ? other : c, n = side ? c : other;
                const double w = m.ow[f], w1 = 1.0 - w;
                const double kx = m.skx[f], ky = m.sky[f], kz = m.skz[f];
#pragma unroll
                for (int q = 0; q < NC; ++q)
                {
                    const double xo = side ? x.c[q][o] : xc[q];
                    const double xn = side ? xc[q] : x.c[q][n];
                    double tf = w * xo + w1 * xn;
                    const double gx = gin.g[q].c[0][o] * w + gin.g[q].c[0][n] * w1;
                    const double gy = gin.g[q].c[1][o] * w + gin.g[q].c[1][n] * w1;
                    const double gz = gin.g[q].c[2][o] * w + gin.g[q].c[2][n] * w1;
                    tf += gx * kx + gy * ky + gz * kz;
                    const double fx = sx * tf, fy = sy * tf, fz = sz * tf;
                    if (!side) { s[q][0] += fx; s[q][1] += fy; s[q][2] += fz; }
                    else { s[q][0] -= fx; s[q][1] -= fy; s[q][2] -= fz; }
                }
            }
            else
            {
#pragma unroll
                for (int q = 0; q < NC; ++q)
                {
                    const double tf = bc.c[q][other] * xc[q] + bc.k[q][other];
                    s[q][0] += sx * tf;
                    s[q][1] += sy * tf;
                    s[q][2] += sz * tf;
                }
            }
        }
        const double v = m.V[c];
#pragma unroll
        for (int q = 0; q < NC; ++q)
        {
            out.g[q].c[0][c] = s[q][0] / v;
            out.g[q].c[1][c] = s[q][1] / v;
            out.g[q].c[2][c] = s[q][2] / v;
        }
    }
}

// ---------------------------------------------------------------------------
// leastSquares gradient (gradScheme.cpp:106-239)
// ---------------------------------------------------------------------------

struct Sym3
{
    double xx = 0, xy = 0, xz = 0, yy = 0, yz = 0, zz = 0;
    __device__ void add(double dx, double dy, double dz, double w)
    {
        xx += w * dx * dx;
        xy += w * dx * dy;
        xz += w * dx * dz;
        yy += w * dy * dy;
        yz += w * dy * dz;
        zz += w * dz * dz;
    }
    __device__ void solve(double bx, double by, double bz, double& ox, double& oy, double& oz) const
    {
        const double t = smax((xx + yy + zz) / 3.0, 1e-300);
        const double e = 1e-12 * t;
        const double XX = xx + e, YY = yy + e, ZZ = zz + e;
        const double c11 = YY * ZZ - yz * yz;
        const double c12 = xz * yz - xy * ZZ;
        const double c13 = xy * yz - YY * xz;
        const double c22 = XX * ZZ - xz * xz;
        const double c23 = xy * xz - XX * yz;
        const double c33 = XX * YY - xy * xy;
        const double det = XX * c11 + xy * c12 + xz * c13;
        if (det <= 0 || !isfinite(det))
        {
            ox = oy = oz = 0.0;
            return;
        }
        ox = (c11 * bx + c12 * by + c13 * bz) / det;
        oy = (c12 * bx + c22 * by + c23 * bz) / det;
        oz = (c13 * bx + c23 * by + c33 * bz) / det;
    }
};

__device__ __forceinline__ double mag3(double x, double y, double z) { return sqrt(x * x + y * y + z * z); }

/// Stage 1: the neighbour-cell bootstrap fit.
template <int NC>
__global__ void __launch_bounds__(TPB) k_grad_ls1(DMesh m, CV3P x, BcTab bc, Grad3 out)
{
    ROW_LOOP(c, m.nC)
    {
        const int sl = c >> 5, lane = c & 31;
        Sym3 cm;
        double r[NC][3];
        double xc[NC];
#pragma unroll
        for (int q = 0; q < NC; ++q)
        {
            r[q][0] = r[q][1] = r[q][2] = 0.0;
            xc[q] = x.c[q][c];
        }
        const double ccx = m.cx[c], ccy = m.cy[c], ccz = m.cz[c];
        const int e1 = m.cfStart[sl + 1];
        for (int e = m.cfStart[sl] + lane; e < e1; e += 32)
        {
            const int code = m.cfCode[e];
            if (code < 0) break;
            const int f = code >> 1, side = code & 1, other = m.cfOther[e];
            if (f < m.nI)
            {
                const int o = side ? other : c, n = side ? c : other;
                const double dx = m.cx[n] - m.cx[o], dy = m.cy[n] - m.cy[o], dz = m.cz[n] - m.cz[o];
                const double wn = 1.0 / smax(mag3(dx, dy, dz), 1e-300);
                cm.add(dx, dy, dz, wn);
#pragma unroll
                for (int q = 0; q < NC; ++q)
                {
                    const double xo = side ? x.c[q][o] : xc[q];
                    const double xn = side ? xc[q] : x.c[q][n];
                    const double dPhi = (xn - xo) * wn;
                    r[q][0] += dx * dPhi;
                    r[q][1] += dy * dPhi;
                    r[q][2] += dz * dPhi;
                }
            }
            else
            {
                const double dx = m.fcx[f] - ccx, dy = m.fcy[f] - ccy, dz = m.fcz[f] - ccz;
                const double wf = 1.0 / smax(mag3(dx, dy, dz), 1e-300);
                cm.add(dx, dy, dz, wf);
#pragma unroll
                for (int q = 0; q < NC; ++q)
                {
                    const double dPhi = ((bc.c[q][other] * xc[q] + bc.k[q][other]) - xc[q]) * wf;
                    r[q][0] += dx * dPhi;
                    r[q][1] += dy * dPhi;
                    r[q][2] += dz * dPhi;
                }
            }
        }
#pragma unroll
        for (int q = 0; q < NC; ++q)
            cm.solve(r[q][0], r[q][1], r[q][2], out.g[q].c[0][c], out.g[q].c[1][c], out.g[q].c[2][c]);
    }
}

/// Stage 2: face values from the bootstrap gradient, then the face fit.
template <int NC>
__global__ void __launch_bounds__(TPB) k_grad_ls2(DMesh m, CV3P x, BcTab bc, CGrad3 g0, Grad3 out)
{
    ROW_LOOP(c, m.nC)
    {
        const int sl = c >> 5, lane = c & 31;
        Sym3 fm;
        double r[NC][3];
        double xc[NC];
#pragma unroll
        for (int q = 0; q < NC; ++q)
        {
            r[q][0] = r[q][1] = r[q][2] = 0.0;
            xc[q] = x.c[q][c];
        }
        const double ccx = m.cx[c], ccy = m.cy[c], ccz = m.cz[c];
        const int e1 = m.cfStart[sl + 1];
        for (int e = m.cfStart[sl] + lane; e < e1; e += 32)
        {
            const int code = m.cfCode[e];
            if (code < 0) break;
            const int f = code >> 1, side = code & 1, other = m.cfOther[e];
            const double fx = m.fcx[f], fy = m.fcy[f], fz = m.fcz[f];
            const double dx = fx - ccx, dy = fy - ccy, dz = fz - ccz;
            const double w = 1.0 / smax(mag3(dx, dy, dz), 1e-300);
            fm.add(dx, dy, dz, w);
#pragma unroll
            for (int q = 0; q < NC; ++q)
            {
                double vf;
                if (f < m.nI)
                {
                    const int o = side ? other : c, n = side ? c : other;
                    const double xo = side ? x.c[q][o] : xc[q];
                    const double xn = side ? xc[q] : x.c[q][n];
                    const double po = xo + (g0.g[q].c[0][o] * (fx - m.cx[o]) + g0.g[q].c[1][o] * (fy - m.cy[o]) +
                                            g0.g[q].c[2][o] * (fz - m.cz[o]));
                    const double pn = xn + (g0.g[q].c[0][n] * (fx - m.cx[n]) + g0.g[q].c[1][n] * (fy - m.cy[n]) +
                                            g0.g[q].c[2][n] * (fz - m.cz[n]));
                    vf = 0.5 * (po + pn);
                }
                else
                {
                    vf = bc.c[q][other] * xc[q] + bc.k[q][other];
                }
                const double a = (vf - xc[q]) * w;
                r[q][0] += dx * a;
                r[q][1] += dy * a;
                r[q][2] += dz * a;
            }
        }
#pragma unroll
        for (int q = 0; q < NC; ++q)
            fm.solve(r[q][0], r[q][1], r[q][2], out.g[q].c[0][c], out.g[q].c[1][c], out.g[q].c[2][c]);
    }
}

// ---------------------------------------------------------------------------
// Sparse matrix-vector products
// ---------------------------------------------------------------------------

/// One row of y = A x for NC vectors sharing A; entries in the reference
/// CSR's column order (SparseMatrix::product, Matrix.cpp:119-133).  W is a
/// compile-time bound on the row length: all column indices and values of
/// the row are loaded first and then all gathers issued, so a thread keeps W
/// independent loads in flight instead of walking a dependent chain.  W = 0
/// walks rows of any length.  Entries are added in order, skipping only the
/// trailing pads, so the sum is the reference's.  T = float forms each
/// product in single precision and accumulates in double.
template <int W, int NC, class T = double>
__device__ __forceinline__ void spmv_row(const DMat& A, const T* __restrict__ val, int c, const T* const (&x)[NC],
                                         double (&y)[NC])
{
#pragma unroll
    for (int q = 0; q < NC; ++q) y[q] = 0.0;
    const int sl = c >> 5, lane = c & 31;
    const int e0 = __ldg(A.start + sl) + lane, e1 = __ldg(A.start + sl + 1);
    if constexpr (W > 0)
    {
        // entries in groups of at most 8 (wide rows stay in registers)
        constexpr int CH = W > 8 ? 8 : W;
#pragma unroll
        for (int k0 = 0; k0 < W; k0 += CH)
        {
            int col[CH];
            T v[CH];
#pragma unroll
            for (int k = 0; k < CH; ++k)
            {
                const int e = e0 + 32 * (k0 + k);
                col[k] = (k0 + k < W && e < e1) ? __ldg(A.col + e) : -1;
                v[k] = (k0 + k < W && e < e1) ? __ldg(val + e) : T(0);
            }
            T xv[NC][CH];
#pragma unroll
            for (int k = 0; k < CH; ++k)
#pragma unroll
                for (int q = 0; q < NC; ++q) xv[q][k] = col[k] >= 0 ? __ldg(x[q] + col[k]) : T(0);
#pragma unroll
            for (int k = 0; k < CH; ++k)
                if (col[k] >= 0)
#pragma unroll
                    for (int q = 0; q < NC; ++q) y[q] += static_cast<double>(v[k] * xv[q][k]);
        }
    }
    else
    {
        for (int e = e0; e < e1; e += 32)
        {
            const int col = A.col[e];
            if (col < 0) break;
            const T v = val[e];
#pragma unroll
            for (int q = 0; q < NC; ++q) y[q] += static_cast<double>(v * x[q][col]);
        }
    }
}

/// One row of y = A x where the NC values of x at a column are formed by
/// `gather(col, xv)` from several arrays, in the same entry order and with
/// the same skipping as spmv_row.
template <int W, int NC, class Gather>
__device__ __forceinline__ void spmv_row_gather(const DMat& A, const double* __restrict__ val, int c, double (&y)[NC],
                                                Gather gather)
{
#pragma unroll
    for (int q = 0; q < NC; ++q) y[q] = 0.0;
    const int sl = c >> 5, lane = c & 31;
    const int e0 = __ldg(A.start + sl) + lane, e1 = __ldg(A.start + sl + 1);
    if constexpr (W > 0)
    {
        // entries in groups of at most 8, so that the gathers of wide rows
        // stay in registers; the sum still runs in entry order
        constexpr int CH = W > 8 ? 8 : W;
#pragma unroll
        for (int k0 = 0; k0 < W; k0 += CH)
        {
            int col[CH];
            double v[CH];
#pragma unroll
            for (int k = 0; k < CH; ++k)
            {
                const int e = e0 + 32 * (k0 + k);
                col[k] = (k0 + k < W && e < e1) ? __ldg(A.col + e) : -1;
                v[k] = (k0 + k < W && e < e1) ? __ldg(val + e) : 0.0;
            }
#pragma unroll
            for (int k = 0; k < CH; ++k)
                if (col[k] >= 0)
                {
                    double xv[NC];
                    gather(col[k], xv);
#pragma unroll
                    for (int q = 0; q < NC; ++q) y[q] += v[k] * xv[q];
                }
        }
    }
    else
    {
        for (int e = e0; e < e1; e += 32)
        {
            const int col = A.col[e];
            if (col < 0) break;
            const double v = val[e];
            double xv[NC];
            gather(col, xv);
#pragma unroll
            for (int q = 0; q < NC; ++q) y[q] += v * xv[q];
        }
    }
}

/// The solver kernels' row loop: a grid-stride loop, so a warp's rows stay
/// contiguous and the grid can be sized for the GPU rather than the system
/// (fewer blocks means fewer per-block reduction epilogues and partials).
/// RPT is the rows per thread of the default grid, ceil(n / (RPT * TPB)).
constexpr int RPT = 2;
/// Blocks per SM the solver kernels are compiled to fit (registers <= 64),
/// so a grid of 4 blocks per SM runs in one wave.
constexpr int kSolverMinBlocks = 4;
#define FOR_ROWS(c, n) \
    for (int c = blockIdx.x * ::cfg::TPB + threadIdx.x; c < (n); c += gridDim.x * ::cfg::TPB)

inline CV3P cv(const V3P& v) { return CV3P{{v.c[0], v.c[1], v.c[2]}}; }

/// The non-orthogonal corrector of assembleLaplacian (laplacianScheme.cpp:217-263):
/// rhs = base + sum over faces in order of +-gamma_f (cfVec . grad_f), with
/// grad_f the owner-weighted face interpolation of the cell gradients.
template <int NC>
__global__ void __launch_bounds__(TPB) k_corrector(DMesh m, const double* __restrict__ gamma, CGrad3 g, CV3P base,
                                                   V3P rhs)
{
    ROW_LOOP(c, m.nC)
    {
        const int sl = c >> 5, lane = c & 31;
        double r[NC];
#pragma unroll
        for (int q = 0; q < NC; ++q) r[q] = base.c[q][c];
        const int e1 = m.cfStart[sl + 1];
        for (int e = m.cfStart[sl] + lane; e < e1; e += 32)
        {
            const int code = m.cfCode[e];
            if (code < 0) break;
            const int f = code >> 1, side = code & 1;
            const double cvx = m.cvx[f], cvy = m.cvy[f], cvz = m.cvz[f], gm = gamma[f];
            if (f < m.nI)
            {
                const int other = m.cfOther[e];
                const int o = side ? other : c, n = side ? c : other;
                const double w = m.ow[f], w1 = 1.0 - w;
#pragma unroll
                for (int q = 0; q < NC; ++q)
                {
                    const double gx = g.g[q].c[0][o] * w + g.g[q].c[0][n] * w1;
                    const double gy = g.g[q].c[1][o] * w + g.g[q].c[1][n] * w1;
                    const double gz = g.g[q].c[2][o] * w + g.g[q].c[2][n] * w1;
                    const double corr = gm * (cvx * gx + cvy * gy + cvz * gz);
                    r[q] = side ? r[q] + (-corr) : r[q] + corr;
                }
            }
            else
            {
#pragma unroll
                for (int q = 0; q < NC; ++q)
                {
                    const double corr =
                        gm * (cvx * g.g[q].c[0][c] + cvy * g.g[q].c[1][c] + cvz * g.g[q].c[2][c]);
                    r[q] = r[q] + corr;
                }
            }
        }
#pragma unroll
        for (int q = 0; q < NC; ++q) rhs.c[q][c] = r[q];
    }
}

}  // namespace cfg
