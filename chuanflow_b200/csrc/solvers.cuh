// Jacobi-preconditioned CG and BiCGStab (src/common/src/Matrix.cpp:153-319)
// as sequences of row kernels with device-resident scalars.  The global dot
// products are block partials plus a fixed-order reduction done by the block
// that finishes last (no block ever waits for another); that block also
// advances the solver's scalar state, which the next kernel reads.
#pragma once

#include "ctx.h"
#include "kernels.cuh"

namespace cfg
{

__device__ __forceinline__ double inv_diag_cg(double d) { return (fabs(d) > 1e-300) ? 1.0 / d : 1.0; }
__device__ __forceinline__ float inv_diag_cg(float d) { return (fabs(static_cast<double>(d)) > 1e-300) ? 1.0f / d : 1.0f; }
__device__ __forceinline__ double inv_diag_bicg(double d) { return (d > 1e-300) ? 1.0 / d : 1.0; }

// ------------------------- device-side solver loops -----------------------
// Inside a captured CUDA graph a solver loop cannot poll its state from the
// host: the iterations run as the body of a conditional while-node, and the
// body's last kernel decides whether it runs again.

/// The solver state cleared and its limits set, by a kernel (a captured
/// graph cannot copy them from a host struct).
static __global__ void k_state_reset(SolveState* st, double tol, int maxIter, int nComp, int normType)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    unsigned char* b = reinterpret_cast<unsigned char*>(st);
    for (size_t i = 0; i < sizeof(SolveState); ++i) b[i] = 0;
    st->tol = tol;
    st->maxIter = maxIter;
    st->nComp = nComp;
    st->normType = normType;
}

/// The while-condition of a device-side solver loop: run the body again
/// while the solve is not done, for at most maxBodies bodies (each body
/// advances at least one iteration until the state's own maxIter test marks
/// the solve done, so the bound is only a backstop).
static __global__ void k_loop_cond(cudaGraphConditionalHandle h, const SolveState* st, int* count, int maxBodies)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const int c = *count + 1;
    *count = c;
    cudaGraphSetConditional(h, (!st->allDone && c < maxBodies) ? 1u : 0u);
}

/// A finished solve's iteration counts added to acc (component sum), and
/// its non-convergence counted in acc[1].
static __global__ void k_state_tally(const SolveState* st, int nComp, double* acc)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    for (int q = 0; q < nComp; ++q)
    {
        acc[0] += st->it[q];
        acc[1] += st->conv[q] ? 0.0 : 1.0;
    }
}

/// the residual norm of the stopping test from |r|inf and sum r^2
__device__ __forceinline__ double resid_norm(const SolveState* st, double inf, double sumsq)
{
    return st->normType ? sqrt(sumsq) : inf;
}

// ------------------------------- CG ---------------------------------------
// T is the type of the matrix values and vectors (double: the reference's
// FP64 solve; float: the inner solves of the mixed-precision refinement).
// Dot products and norms accumulate in double either way.

/// r = b - A x; z = D^-1 r; p = z; initial residual, |b|, and r.z.
template <int W, class T = double>
__global__ void __launch_bounds__(TPB, kSolverMinBlocks) k_cg_init(DMat A, const T* __restrict__ val, const T* __restrict__ diag,
                                                 const T* __restrict__ b, const T* __restrict__ x, T* __restrict__ r,
                                                 T* __restrict__ p, double* partials, SolveState* st)
{
    double mx[3] = {0.0, 0.0, 0.0};  // |r|, |b|, nan flag
    double sm[3] = {0.0, 0.0, 0.0};  // r.z, r.r, b.b
    const T* xs[1] = {x};
    FOR_ROWS(c, A.n)
    {
        double y[1];
        spmv_row<W, 1, T>(A, val, c, xs, y);
        const T bi = b[c];
        const T ri = static_cast<T>(static_cast<double>(bi) - y[0]);
        r[c] = ri;
        const T zi = inv_diag_cg(diag[c]) * ri;
        p[c] = zi;
        if (isnan(static_cast<double>(ri))) mx[2] = 1.0;
        mx[0] = smax(mx[0], fabs(static_cast<double>(ri)));
        if (isnan(static_cast<double>(bi))) mx[2] = 1.0;
        mx[1] = smax(mx[1], fabs(static_cast<double>(bi)));
        sm[0] += static_cast<double>(ri * zi);
        sm[1] += static_cast<double>(ri) * static_cast<double>(ri);
        sm[2] += static_cast<double>(bi) * static_cast<double>(bi);
    }
    block_max<3>(mx);
    __syncthreads();
    block_sum<3>(sm);
    const int G = gridDim.x;
    if (threadIdx.x == 0)
    {
        partials[blockIdx.x] = mx[0];
        partials[G + blockIdx.x] = mx[1];
        partials[2 * G + blockIdx.x] = mx[2];
        partials[3 * G + blockIdx.x] = sm[0];
        partials[4 * G + blockIdx.x] = sm[1];
        partials[5 * G + blockIdx.x] = sm[2];
    }
    if (!last_block(&st->ticket[0])) return;
    double fm[3], fs[3];
    final_max<3>(partials, G, fm);
    __syncthreads();
    final_sum<3>(partials + 3 * G, G, fs);
    if (threadIdx.x == 0)
    {
        st->ticket[0] = 0;
        const double init = fm[2] > 0 ? NAN : resid_norm(st, fm[0], fs[1]);
        const double bn = smax(st->normType ? sqrt(fs[2]) : fm[1], 1e-300);
        st->init[0] = init;
        st->bnorm[0] = bn;
        st->it[0] = 0;
        st->conv[0] = 0;
        st->done[0] = 0;
        st->fin[0] = 0.0;
        st->rz[0] = fs[0];
        if (init / bn < st->tol)
        {
            st->conv[0] = 1;
            st->done[0] = 1;
            st->fin[0] = init;
        }
        else if (st->maxIter <= 0)
        {
            st->done[0] = 1;
        }
        st->allDone = st->done[0];
    }
}

/// Ap = A p and p.Ap; breakdown test and alpha (Matrix.cpp:187-194).
template <int W, class T = double>
__global__ void __launch_bounds__(TPB, kSolverMinBlocks) k_cg_spmv(DMat A, const T* __restrict__ val, const T* __restrict__ p,
                                                 T* __restrict__ Ap, double* partials, SolveState* st)
{
    if (st->allDone) return;
    double sm[1] = {0.0};
    const T* xs[1] = {p};
    FOR_ROWS(c, A.n)
    {
        double y[1];
        spmv_row<W, 1, T>(A, val, c, xs, y);
        const T ay = static_cast<T>(y[0]);
        Ap[c] = ay;
        sm[0] += static_cast<double>(p[c] * ay);
    }
    block_sum<1>(sm);
    if (threadIdx.x == 0) partials[blockIdx.x] = sm[0];
    if (!last_block(&st->ticket[0])) return;
    double fs[1];
    final_sum<1>(partials, gridDim.x, fs);
    if (threadIdx.x == 0)
    {
        st->ticket[0] = 0;
        const double pAp = fs[0];
        const double rz = st->rz[0];
        st->pAp[0] = pAp;
        if (pAp <= 0 || fabs(rz) < 1e-300)
        {
            st->done[0] = 1;
            st->allDone = 1;
        }
        else
        {
            st->alpha[0] = rz / pAp;
        }
    }
}

/// x += alpha p; r -= alpha Ap; residual test; z = D^-1 r; beta (Matrix.cpp:195-217).
template <class T = double>
__global__ void __launch_bounds__(TPB, kSolverMinBlocks) k_cg_update(int n, const T* __restrict__ diag, const T* __restrict__ p,
                                                   const T* __restrict__ Ap, T* __restrict__ x, T* __restrict__ r,
                                                   double* partials, SolveState* st)
{
    if (st->allDone) return;
    const T alpha = static_cast<T>(st->alpha[0]);
    double mx[2] = {0.0, 0.0};
    double sm[2] = {0.0, 0.0};
    FOR_ROWS(c, n)
    {
        x[c] = x[c] + alpha * p[c];
        const T ri = r[c] - alpha * Ap[c];
        r[c] = ri;
        if (isnan(static_cast<double>(ri))) mx[1] = 1.0;
        mx[0] = smax(mx[0], fabs(static_cast<double>(ri)));
        const T zi = inv_diag_cg(diag[c]) * ri;
        sm[0] += static_cast<double>(ri * zi);
        sm[1] += static_cast<double>(ri) * static_cast<double>(ri);
    }
    block_max<2>(mx);
    __syncthreads();
    block_sum<2>(sm);
    const int G = gridDim.x;
    if (threadIdx.x == 0)
    {
        partials[blockIdx.x] = mx[0];
        partials[G + blockIdx.x] = mx[1];
        partials[2 * G + blockIdx.x] = sm[0];
        partials[3 * G + blockIdx.x] = sm[1];
    }
    if (!last_block(&st->ticket[0])) return;
    double fm[2], fs[2];
    final_max<2>(partials, G, fm);
    __syncthreads();
    final_sum<2>(partials + 2 * G, G, fs);
    if (threadIdx.x == 0)
    {
        st->ticket[0] = 0;
        const int it = st->it[0] + 1;
        st->it[0] = it;
        const double fin = fm[1] > 0 ? NAN : resid_norm(st, fm[0], fs[1]);
        st->fin[0] = fin;
        if (fin / st->bnorm[0] < st->tol)
        {
            st->conv[0] = 1;
            st->done[0] = 1;
        }
        else if (isnan(fin))
        {
            // the reference keeps iterating on NaN until maxIter; the
            // iterate stays NaN, so stop here and report what it reports
            st->it[0] = st->maxIter;
            st->done[0] = 1;
        }
        else
        {
            const double rzNew = fs[0];
            st->beta[0] = rzNew / st->rz[0];
            st->rz[0] = rzNew;
            if (it >= st->maxIter) st->done[0] = 1;
        }
        st->allDone = st->done[0];
    }
}

/// p = z + beta p.
template <class T = double>
__global__ void __launch_bounds__(TPB, kSolverMinBlocks) k_cg_p(int n, const T* __restrict__ diag, const T* __restrict__ r,
                                              T* __restrict__ p, const SolveState* st)
{
    if (st->allDone) return;
    const T beta = static_cast<T>(st->beta[0]);
    FOR_ROWS(c, n) p[c] = inv_diag_cg(diag[c]) * r[c] + beta * p[c];
}

// ------------------------ BiCGStab, 1..3 right-hand sides ------------------
// The components of the momentum equation share their matrix (the reference
// asserts equal diagonals, simpleSolver.cpp:123-144, and every off-diagonal
// term is component-independent), so up to three BiCGStab iterations run in
// lockstep over one matrix read; each component keeps its own scalars and
// stops on its own test exactly where the serial loop would.

template <int W, int NC>
__global__ void __launch_bounds__(TPB, kSolverMinBlocks) k_bi_init(DMat A, const double* __restrict__ val,
                                                 const double* __restrict__ diag, double* __restrict__ invD, V3P b,
                                                 V3P x, V3P r, V3P r0, V3P p, V3P v, double* partials, SolveState* st)
{
    double mx[3 * NC];  // |r|, |b|, nan per comp
    double sm[NC];      // r.r
#pragma unroll
    for (int q = 0; q < 3 * NC; ++q) mx[q] = 0.0;
#pragma unroll
    for (int q = 0; q < NC; ++q) sm[q] = 0.0;
    const double* xs[NC];
#pragma unroll
    for (int q = 0; q < NC; ++q) xs[q] = x.c[q];
    FOR_ROWS(c, A.n)
    {
        invD[c] = inv_diag_bicg(diag[c]);  // invD of Matrix.cpp:229-236
        double y[NC];
        spmv_row<W, NC>(A, val, c, xs, y);
#pragma unroll
        for (int q = 0; q < NC; ++q)
        {
            const double bi = b.c[q][c];
            const double ri = bi - y[q];
            r.c[q][c] = ri;
            r0.c[q][c] = ri;
            p.c[q][c] = 0.0;
            v.c[q][c] = 0.0;
            if (isnan(ri) || isnan(bi)) mx[2 * NC + q] = 1.0;
            mx[q] = smax(mx[q], fabs(ri));
            mx[NC + q] = smax(mx[NC + q], fabs(bi));
            sm[q] += ri * ri;
        }
    }
    block_max<3 * NC>(mx);
    __syncthreads();
    block_sum<NC>(sm);
    const int G = gridDim.x;
    if (threadIdx.x == 0)
    {
#pragma unroll
        for (int q = 0; q < 3 * NC; ++q) partials[q * G + blockIdx.x] = mx[q];
#pragma unroll
        for (int q = 0; q < NC; ++q) partials[(3 * NC + q) * G + blockIdx.x] = sm[q];
    }
    if (!last_block(&st->ticket[0])) return;
    double fm[3 * NC], fs[NC];
    final_max<3 * NC>(partials, G, fm);
    __syncthreads();
    final_sum<NC>(partials + 3 * NC * G, G, fs);
    if (threadIdx.x == 0)
    {
        st->ticket[0] = 0;
        int all = 1;
        for (int q = 0; q < NC; ++q)
        {
            const double init = fm[2 * NC + q] > 0 ? NAN : fm[q];
            const double bn = smax(fm[NC + q], 1e-300);
            st->init[q] = init;
            st->bnorm[q] = bn;
            st->it[q] = 0;
            st->conv[q] = 0;
            st->done[q] = 0;
            st->special[q] = 0;
            st->fin[q] = 0.0;
            st->rho[q] = 1.0;
            st->alpha[q] = 1.0;
            st->omega[q] = 1.0;
            st->rz[q] = fs[q];  // rhoNew of the first iteration: r0.r = r.r
            if (init / bn < st->tol)
            {
                st->conv[q] = 1;
                st->done[q] = 1;
                st->fin[q] = init;
            }
            else if (st->maxIter <= 0 || fabs(fs[q]) < 1e-300)
            {
                st->done[q] = 1;
            }
            all &= st->done[q];
        }
        st->allDone = all;
    }
}

/// p = r + beta (p - omega v); z = p D^-1   (Matrix.cpp:262-272)
template <int NC>
__global__ void __launch_bounds__(TPB, kSolverMinBlocks) k_bi_p(int n, const double* __restrict__ invD, V3P r, V3P p, V3P v,
                                              V3P z, const SolveState* st)
{
    if (st->allDone) return;
    double beta[NC], om[NC];
    int dn[NC];
#pragma unroll
    for (int q = 0; q < NC; ++q)
    {
        dn[q] = st->done[q];
        beta[q] = (st->rz[q] / st->rho[q]) * (st->alpha[q] / st->omega[q]);
        om[q] = st->omega[q];
    }
    FOR_ROWS(c, n)
    {
        // every load of the row before its first store: the component
        // arrays are not restrict-qualified, so a store would otherwise
        // hold back the next component's loads
        const double id = invD[c];
        double rv[NC], pv[NC], vv[NC];
#pragma unroll
        for (int q = 0; q < NC; ++q)
            if (!dn[q])
            {
                rv[q] = r.c[q][c];
                pv[q] = p.c[q][c];
                vv[q] = v.c[q][c];
            }
#pragma unroll
        for (int q = 0; q < NC; ++q)
        {
            if (dn[q]) continue;
            const double pi = rv[q] + beta[q] * (pv[q] - om[q] * vv[q]);
            p.c[q][c] = pi;
            z.c[q][c] = pi * id;
        }
    }
}

/// v = A z; r0.v; alpha (Matrix.cpp:273-276)
template <int W, int NC>
__global__ void __launch_bounds__(TPB, kSolverMinBlocks) k_bi_spmv1(DMat A, const double* __restrict__ val, V3P z, V3P v, V3P r0,
                                                  double* partials, SolveState* st)
{
    pdl_entry();
    if (st->allDone) return;
    double sm[NC];
#pragma unroll
    for (int q = 0; q < NC; ++q) sm[q] = 0.0;
    const double* xs[NC];
#pragma unroll
    for (int q = 0; q < NC; ++q) xs[q] = z.c[q];
    FOR_ROWS(c, A.n)
    {
        double r0v[NC];
#pragma unroll
        for (int q = 0; q < NC; ++q) r0v[q] = r0.c[q][c];
        double y[NC];
        spmv_row<W, NC>(A, val, c, xs, y);
#pragma unroll
        for (int q = 0; q < NC; ++q)
        {
            v.c[q][c] = y[q];
            sm[q] += r0v[q] * y[q];
        }
    }
    block_sum<NC>(sm);
    const int G = gridDim.x;
    if (threadIdx.x == 0)
#pragma unroll
        for (int q = 0; q < NC; ++q) partials[q * G + blockIdx.x] = sm[q];
    if (!last_block(&st->ticket[0])) return;
    double fs[NC];
    final_sum<NC>(partials, G, fs);
    if (threadIdx.x == 0)
    {
        st->ticket[0] = 0;
        int all = 1;
        for (int q = 0; q < NC; ++q)
        {
            if (!st->done[q])
            {
                st->rho[q] = st->rz[q];
                const double denom = fs[q];
                if (fabs(denom) < 1e-300) st->done[q] = 1;
                else st->alpha[q] = st->rho[q] / denom;
            }
            all &= st->done[q];
        }
        st->allDone = all;
    }
}

/// The end of the second BiCGStab product: block sums of t.t (sm[q]) and
/// t.s (sm[NC + q]) into partials; the last block sets omega, or takes the
/// tDenom breakdown exit (Matrix.cpp:291-300).
template <int NC>
__device__ __forceinline__ void omega_epilogue(double (&sm)[2 * NC], double* partials, SolveState* st)
{
    block_sum<2 * NC>(sm);
    const int G = gridDim.x;
    if (threadIdx.x == 0)
#pragma unroll
        for (int q = 0; q < 2 * NC; ++q) partials[q * G + blockIdx.x] = sm[q];
    if (!last_block(&st->ticket[0])) return;
    double fs[2 * NC];
    final_sum<2 * NC>(partials, G, fs);
    if (threadIdx.x == 0)
    {
        st->ticket[0] = 0;
        int all = 1;
        for (int q = 0; q < NC; ++q)
        {
            if (!st->done[q])
            {
                const double tDenom = fs[q];
                if (tDenom < 1e-300)
                {
                    // r = s and the iteration counts; k_bi_x applies this
                    // iteration's x += alpha z and reports |s|inf
                    st->special[q] = 1;
                    st->it[q] = st->it[q] + 1;
                    st->done[q] = 1;
                }
                else
                {
                    st->omega[q] = fs[NC + q] / tDenom;
                }
            }
            all &= st->done[q];
        }
        st->allDone = all;
    }
}

/// t = A sh with sh = (r - alpha v) D^-1 formed per column as the row is
/// read; t.t and t.s; omega, or the tDenom breakdown exit (Matrix.cpp:
/// 277-300).  s and sh are never stored: every reader forms them from r, v
/// and invD with the same two operations, so each value is the reference's,
/// and the separate s pass and its two stores disappear.  The |s|inf that
/// the breakdown exit reports is taken by k_bi_x, in that case only.
template <int W, int NC>
__global__ void __launch_bounds__(TPB, kSolverMinBlocks) k_bi_spmv2(DMat A, const double* __restrict__ val,
                                                  const double* __restrict__ invD, V3P r, V3P v, V3P t,
                                                  double* partials, SolveState* st)
{
    if (st->allDone) return;
    double al[NC];
    double sm[2 * NC];
#pragma unroll
    for (int q = 0; q < NC; ++q)
    {
        al[q] = st->alpha[q];
        sm[q] = sm[NC + q] = 0.0;
    }
    FOR_ROWS(c, A.n)
    {
        double y[NC];
        spmv_row_gather<W, NC>(A, val, c, y, [&](int col, double (&xv)[NC]) {
            const double id = __ldg(invD + col);
#pragma unroll
            for (int q = 0; q < NC; ++q) xv[q] = (__ldg(r.c[q] + col) - al[q] * __ldg(v.c[q] + col)) * id;
        });
#pragma unroll
        for (int q = 0; q < NC; ++q)
        {
            const double si = r.c[q][c] - al[q] * v.c[q][c];
            t.c[q][c] = y[q];
            sm[q] += y[q] * y[q];
            sm[NC + q] += y[q] * si;
        }
    }
    omega_epilogue<NC>(sm, partials, st);
}

/// The end of the BiCGStab update: block reductions of |r|inf (mx[q]), the
/// NaN flags (mx[NC + q]) and r0.r (sm[q]); the last block applies the
/// stopping test (Matrix.cpp:301-315), or finishes a component that broke
/// down in the second product with |s|inf as its final residual.
template <int NC>
__device__ __forceinline__ void update_epilogue(double (&mx)[2 * NC], double (&sm)[NC], double* partials,
                                                SolveState* st)
{
    block_max<2 * NC>(mx);
    __syncthreads();
    block_sum<NC>(sm);
    const int G = gridDim.x;
    if (threadIdx.x == 0)
    {
#pragma unroll
        for (int q = 0; q < 2 * NC; ++q) partials[q * G + blockIdx.x] = mx[q];
#pragma unroll
        for (int q = 0; q < NC; ++q) partials[(2 * NC + q) * G + blockIdx.x] = sm[q];
    }
    if (!last_block(&st->ticket[0])) return;
    double fm[2 * NC], fs[NC];
    final_max<2 * NC>(partials, G, fm);
    __syncthreads();
    final_sum<NC>(partials + 2 * NC * G, G, fs);
    if (threadIdx.x == 0)
    {
        st->ticket[0] = 0;
        int all = 1;
        for (int q = 0; q < NC; ++q)
        {
            if (st->special[q])
            {
                st->fin[q] = fm[NC + q] > 0 ? NAN : fm[q];
                st->conv[q] = st->fin[q] / st->bnorm[q] < st->tol;
            }
            else if (!st->done[q])
            {
                const int it = st->it[q] + 1;
                st->it[q] = it;
                const double fin = fm[NC + q] > 0 ? NAN : fm[q];
                st->fin[q] = fin;
                if (fin / st->bnorm[q] < st->tol)
                {
                    st->conv[q] = 1;
                    st->done[q] = 1;
                }
                else if (isnan(fin))
                {
                    st->it[q] = st->maxIter;
                    st->done[q] = 1;
                }
                else
                {
                    st->rz[q] = fs[q];
                    if (it >= st->maxIter || fabs(fs[q]) < 1e-300) st->done[q] = 1;
                }
            }
            all &= st->done[q];
        }
        for (int q = 0; q < 3; ++q) st->special[q] = 0;
        st->allDone = all;
    }
}

/// x = (x + alpha z) + omega sh; r = s - omega t; |r|inf test; next r0.r
/// (Matrix.cpp:280-282, 301-315, 263-264), with s = r - alpha v and sh = s
/// invD formed as in k_bi_spmv2.  A component that broke down in k_bi_spmv2
/// takes only its x + alpha z, and its |s|inf becomes the final residual.
template <int NC>
__global__ void __launch_bounds__(TPB, kSolverMinBlocks) k_bi_x(int n, const double* __restrict__ invD, V3P x, V3P z,
                                              V3P v, V3P t, V3P r, V3P r0, double* partials, SolveState* st)
{
    if (st->allDone && !(st->special[0] | st->special[1] | st->special[2])) return;
    double om[NC], al[NC];
    int dn[NC], sp[NC];
    double mx[2 * NC], sm[NC];
#pragma unroll
    for (int q = 0; q < NC; ++q)
    {
        dn[q] = st->done[q];
        sp[q] = st->special[q];
        om[q] = st->omega[q];
        al[q] = st->alpha[q];
        mx[q] = mx[NC + q] = 0.0;
        sm[q] = 0.0;
    }
    FOR_ROWS(c, n)
    {
        const double id = invD[c];
        // one component at a time: its loads, then its two stores
#pragma unroll
        for (int q = 0; q < NC; ++q)
        {
            if (dn[q])
            {
                if (sp[q])
                {
                    x.c[q][c] = x.c[q][c] + al[q] * z.c[q][c];
                    const double si = r.c[q][c] - al[q] * v.c[q][c];
                    if (isnan(si)) mx[NC + q] = 1.0;
                    mx[q] = smax(mx[q], fabs(si));
                }
                continue;
            }
            const double xv = x.c[q][c], zv = z.c[q][c], rv = r.c[q][c];
            const double vv = v.c[q][c], tv = t.c[q][c], r0v = r0.c[q][c];
            const double si = rv - al[q] * vv;
            x.c[q][c] = (xv + al[q] * zv) + om[q] * (si * id);
            const double ri = si - om[q] * tv;
            r.c[q][c] = ri;
            if (isnan(ri)) mx[NC + q] = 1.0;
            mx[q] = smax(mx[q], fabs(ri));
            sm[q] += r0v * ri;
        }
    }
    update_epilogue<NC>(mx, sm, partials, st);
}


// ------------- BiCGStab with the AMG V-cycle as right preconditioner --------
// The reference's iteration (Matrix.cpp:262-315) with M = the V-cycle in
// place of D^-1: z = M p and sh = M s are applied between these kernels by
// amgCycle3, so p and s are stored here for it to read.

/// p = r + beta (p - omega v)  (Matrix.cpp:262-270)
template <int NC>
__global__ void __launch_bounds__(TPB, kSolverMinBlocks) k_bia_p(int n, V3P r, V3P p, V3P v, const SolveState* st)
{
    pdl_entry();
    if (st->allDone) return;
    double beta[NC], om[NC];
    int dn[NC];
#pragma unroll
    for (int q = 0; q < NC; ++q)
    {
        dn[q] = st->done[q];
        beta[q] = (st->rz[q] / st->rho[q]) * (st->alpha[q] / st->omega[q]);
        om[q] = st->omega[q];
    }
    FOR_ROWS(c, n)
    {
        double rv[NC], pv[NC], vv[NC];
#pragma unroll
        for (int q = 0; q < NC; ++q)
            if (!dn[q])
            {
                rv[q] = r.c[q][c];
                pv[q] = p.c[q][c];
                vv[q] = v.c[q][c];
            }
#pragma unroll
        for (int q = 0; q < NC; ++q)
            if (!dn[q]) p.c[q][c] = rv[q] + beta[q] * (pv[q] - om[q] * vv[q]);
    }
}

/// s = r - alpha v  (Matrix.cpp:277)
template <int NC>
__global__ void __launch_bounds__(TPB, kSolverMinBlocks) k_bia_s(int n, V3P r, V3P v, V3P s, const SolveState* st)
{
    pdl_entry();
    if (st->allDone) return;
    double al[NC];
    int dn[NC];
#pragma unroll
    for (int q = 0; q < NC; ++q)
    {
        dn[q] = st->done[q];
        al[q] = st->alpha[q];
    }
    FOR_ROWS(c, n)
    {
        double rv[NC], vv[NC];
#pragma unroll
        for (int q = 0; q < NC; ++q)
            if (!dn[q])
            {
                rv[q] = r.c[q][c];
                vv[q] = v.c[q][c];
            }
#pragma unroll
        for (int q = 0; q < NC; ++q)
            if (!dn[q]) s.c[q][c] = rv[q] - al[q] * vv[q];
    }
}

/// t = A sh; t.t and t.s; omega or the breakdown exit (Matrix.cpp:278-300)
template <int W, int NC>
__global__ void __launch_bounds__(TPB, kSolverMinBlocks) k_bia_spmv2(DMat A, const double* __restrict__ val, V3P sh,
                                                                     V3P s, V3P t, double* partials, SolveState* st)
{
    pdl_entry();
    if (st->allDone) return;
    double sm[2 * NC];
#pragma unroll
    for (int q = 0; q < 2 * NC; ++q) sm[q] = 0.0;
    const double* xs[NC];
#pragma unroll
    for (int q = 0; q < NC; ++q) xs[q] = sh.c[q];
    FOR_ROWS(c, A.n)
    {
        double y[NC];
        spmv_row<W, NC>(A, val, c, xs, y);
#pragma unroll
        for (int q = 0; q < NC; ++q)
        {
            const double si = s.c[q][c];
            t.c[q][c] = y[q];
            sm[q] += y[q] * y[q];
            sm[NC + q] += y[q] * si;
        }
    }
    omega_epilogue<NC>(sm, partials, st);
}

/// x = (x + alpha z) + omega sh; r = s - omega t; |r|inf test; next r0.r
/// (Matrix.cpp:280-282, 301-315, 263-264); a component that broke down in
/// k_bia_spmv2 takes x + alpha z and |s|inf as its final residual
template <int NC>
__global__ void __launch_bounds__(TPB, kSolverMinBlocks) k_bia_x(int n, V3P x, V3P z, V3P s, V3P sh, V3P t, V3P r,
                                                                 V3P r0, double* partials, SolveState* st)
{
    pdl_entry();
    if (st->allDone && !(st->special[0] | st->special[1] | st->special[2])) return;
    double om[NC], al[NC];
    int dn[NC], sp[NC];
    double mx[2 * NC], sm[NC];
#pragma unroll
    for (int q = 0; q < NC; ++q)
    {
        dn[q] = st->done[q];
        sp[q] = st->special[q];
        om[q] = st->omega[q];
        al[q] = st->alpha[q];
        mx[q] = mx[NC + q] = 0.0;
        sm[q] = 0.0;
    }
    FOR_ROWS(c, n)
    {
#pragma unroll
        for (int q = 0; q < NC; ++q)
        {
            if (dn[q])
            {
                if (sp[q])
                {
                    x.c[q][c] = x.c[q][c] + al[q] * z.c[q][c];
                    const double si = s.c[q][c];
                    if (isnan(si)) mx[NC + q] = 1.0;
                    mx[q] = smax(mx[q], fabs(si));
                }
                continue;
            }
            const double xv = x.c[q][c], zv = z.c[q][c], si = s.c[q][c];
            const double hv = sh.c[q][c], tv = t.c[q][c], r0v = r0.c[q][c];
            x.c[q][c] = (xv + al[q] * zv) + om[q] * hv;
            const double ri = si - om[q] * tv;
            r.c[q][c] = ri;
            if (isnan(ri)) mx[NC + q] = 1.0;
            mx[q] = smax(mx[q], fabs(ri));
            sm[q] += r0v * ri;
        }
    }
    update_epilogue<NC>(mx, sm, partials, st);
}

}  // namespace cfg
