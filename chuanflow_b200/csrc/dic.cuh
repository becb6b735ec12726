// Multicolour DIC preconditioner for the pressure PCG (no reference
// counterpart: the reference's "DICG" is Jacobi-preconditioned CG,
// src/common/include/cf/common/Matrix.h:65-72).  OpenFOAM's DIC keeps the
// matrix's off-diagonals and modifies only the diagonal, eliminating in
// face (owner < neighbour) order, which is sequential.  Here the cells are
// coloured so that no two neighbours share a colour, and "lower" means "of
// a smaller colour": every colour is then one parallel phase.
//   colours: greedy first-fit over cells in ascending order;
//   factor:  colour by colour, rD_i = ((a_ii - a_ij1^2/rD_j1) - ...) over the
//            lower neighbours in ascending column order, stored as 1/rD_i;
//   apply:   forward z_i = rDinv_i (r_i - sum_lower a_ij z_j) colour by
//            colour, then backward z_i -= rDinv_i sum_upper a_ij z_j over the
//            colours in reverse, all but the last.
// Each colour's lower and upper entries sit in their own SELL-32 arrays over
// that colour's rows, so a phase reads only its own part of the matrix.
#pragma once

#include "kernels.cuh"
#include "solvers.cuh"

namespace cfg
{

/// the colour layouts' values from the main matrix (T = float also rounds
/// them to single precision)
template <class T>
__global__ void __launch_bounds__(TPB, kSolverMinBlocks) k_dic_gather(int n, const int* __restrict__ src, const double* __restrict__ val,
                                                    T* __restrict__ out)
{
    ROW_LOOP(e, n) out[e] = src[e] >= 0 ? static_cast<T>(val[src[e]]) : T(0);
}

/// One row's entries of a colour slice (lane `lane`, entries e0 + 32k below
/// e1): columns and values loaded for all W slots first, then the gathered
/// x_j, so a row costs one index latency and one gather latency however
/// many entries it has.  Pads (column -1) come after a row's last entry.
/// W = 0 walks the list entry by entry.
template <int W, class T>
struct DicRow
{
    int col[W > 0 ? W : 1];
    T val[W > 0 ? W : 1];
    T x[W > 0 ? W : 1];
    __device__ __forceinline__ void load(const int* __restrict__ cols, const T* __restrict__ vals, int e0, int e1,
                                         const T* __restrict__ xs)
    {
#pragma unroll
        for (int k = 0; k < W; ++k)
        {
            const int e = e0 + 32 * k;
            col[k] = e < e1 ? __ldg(cols + e) : -1;
            val[k] = e < e1 ? __ldg(vals + e) : T(0);
        }
#pragma unroll
        for (int k = 0; k < W; ++k) x[k] = col[k] >= 0 ? xs[col[k]] : T(0);
    }
};

/// rD_i = a_ii - sum a_ij^2 / rD_j over the lower entries, one colour
template <int W, class T>
__global__ void __launch_bounds__(TPB, kSolverMinBlocks) k_dic_factor(DDicT<T> D, DicPhase ph, const T* __restrict__ diag)
{
    FOR_ROWS(t, ph.cnt)
    {
        const int i = D.rows[ph.off + t];
        const int sl = ph.slice0 + (t >> 5), lane = t & 31;
        T d = diag[i];
        const int e0 = D.lStart[sl] + lane, e1 = D.lStart[sl + 1];
        if constexpr (W > 0)
        {
            DicRow<W, T> rw;
            rw.load(D.lCol, D.lVal, e0, e1, D.rD);
#pragma unroll
            for (int k = 0; k < W; ++k)
                if (rw.col[k] >= 0) d = d - rw.val[k] * rw.val[k] / rw.x[k];
        }
        else
        {
            for (int e = e0; e < e1; e += 32)
            {
                const int j = D.lCol[e];
                if (j < 0) break;
                const T a = D.lVal[e];
                d = d - a * a / D.rD[j];
            }
        }
        D.rD[i] = d;
        D.rDinv[i] = T(1) / d;
    }
}

/// forward phase of one colour: z_i = rDinv_i (r_i - sum_lower a_ij z_j);
/// the last colour's rows also contribute their r_i z_i partials
template <int W, class T>
__global__ void __launch_bounds__(TPB, kSolverMinBlocks) k_dic_fwd(DDicT<T> D, DicPhase ph, const T* __restrict__ r, T* z, int last,
                                                 double* partials, SolveState* st)
{
    if (st->allDone) return;
    double sm[1] = {0.0};
    FOR_ROWS(t, ph.cnt)
    {
        const int i = D.rows[ph.off + t];
        const int sl = ph.slice0 + (t >> 5), lane = t & 31;
        T s = T(0);
        const int e0 = D.lStart[sl] + lane, e1 = D.lStart[sl + 1];
        if constexpr (W > 0)
        {
            DicRow<W, T> rw;
            rw.load(D.lCol, D.lVal, e0, e1, z);
#pragma unroll
            for (int k = 0; k < W; ++k)
                if (rw.col[k] >= 0) s += rw.val[k] * rw.x[k];
        }
        else
        {
            for (int e = e0; e < e1; e += 32)
            {
                const int j = D.lCol[e];
                if (j < 0) break;
                s += D.lVal[e] * z[j];
            }
        }
        const T ri = r[i];
        const T zi = D.rDinv[i] * (ri - s);
        z[i] = zi;
        sm[0] += static_cast<double>(ri * zi);
    }
    if (!last) return;
    block_sum<1>(sm);
    if (threadIdx.x == 0) partials[ph.partialOff + blockIdx.x] = sm[0];
}

/// backward phase of one colour: z_i -= rDinv_i sum_upper a_ij z_j, with
/// the r_i z_i partials; `final` (the phase that runs last) also reduces
/// all colours' partials into r.z and advances beta
template <int W, class T>
__global__ void __launch_bounds__(TPB, kSolverMinBlocks) k_dic_bwd(DDicT<T> D, DicPhase ph, const T* __restrict__ r, T* z, int final,
                                                 int nPartials, double* partials, SolveState* st)
{
    if (st->allDone) return;
    double sm[1] = {0.0};
    FOR_ROWS(t, ph.cnt)
    {
        const int i = D.rows[ph.off + t];
        const int sl = ph.slice0 + (t >> 5), lane = t & 31;
        T s = T(0);
        const int e0 = D.uStart[sl] + lane, e1 = D.uStart[sl + 1];
        if constexpr (W > 0)
        {
            DicRow<W, T> rw;
            rw.load(D.uCol, D.uVal, e0, e1, z);
#pragma unroll
            for (int k = 0; k < W; ++k)
                if (rw.col[k] >= 0) s += rw.val[k] * rw.x[k];
        }
        else
        {
            for (int e = e0; e < e1; e += 32)
            {
                const int j = D.uCol[e];
                if (j < 0) break;
                s += D.uVal[e] * z[j];
            }
        }
        const T zi = z[i] - D.rDinv[i] * s;
        z[i] = zi;
        sm[0] += static_cast<double>(r[i] * zi);
    }
    block_sum<1>(sm);
    if (threadIdx.x == 0) partials[ph.partialOff + blockIdx.x] = sm[0];
    if (!final) return;
    if (!last_block(&st->ticket[0])) return;
    double fs[1];
    final_sum<1>(partials, nPartials, fs);
    if (threadIdx.x == 0)
    {
        st->ticket[0] = 0;
        const double rzNew = fs[0];
        // the first application (it == 0) sets p = z: beta 0 with p = 0
        st->beta[0] = st->it[0] == 0 ? 0.0 : rzNew / st->rz[0];
        st->rz[0] = rzNew;
    }
}

/// x += alpha p; r -= alpha Ap; residual test (Matrix.cpp:195-208), without z
template <class T = double>
__global__ void __launch_bounds__(TPB, kSolverMinBlocks) k_cg_update_nz(int n, const T* __restrict__ p, const T* __restrict__ Ap,
                                                      T* __restrict__ x, T* __restrict__ r, double* partials,
                                                      SolveState* st)
{
    if (st->allDone) return;
    const T alpha = static_cast<T>(st->alpha[0]);
    double mx[2] = {0.0, 0.0};
    double sm[1] = {0.0};
    FOR_ROWS(c, n)
    {
        x[c] = x[c] + alpha * p[c];
        const T ri = r[c] - alpha * Ap[c];
        r[c] = ri;
        if (isnan(static_cast<double>(ri))) mx[1] = 1.0;
        mx[0] = smax(mx[0], fabs(static_cast<double>(ri)));
        sm[0] += static_cast<double>(ri) * static_cast<double>(ri);
    }
    block_max<2>(mx);
    __syncthreads();
    block_sum<1>(sm);
    const int G = gridDim.x;
    if (threadIdx.x == 0)
    {
        partials[blockIdx.x] = mx[0];
        partials[G + blockIdx.x] = mx[1];
        partials[2 * G + blockIdx.x] = sm[0];
    }
    if (!last_block(&st->ticket[0])) return;
    double fm[2], fs[1];
    final_max<2>(partials, G, fm);
    __syncthreads();
    final_sum<1>(partials + 2 * G, G, fs);
    if (threadIdx.x == 0)
    {
        st->ticket[0] = 0;
        const int it = st->it[0] + 1;
        st->it[0] = it;
        const double fin = fm[1] > 0 ? NAN : resid_norm(st, fm[0], fs[0]);
        st->fin[0] = fin;
        if (fin / st->bnorm[0] < st->tol)
        {
            st->conv[0] = 1;
            st->done[0] = 1;
        }
        else if (isnan(fin))
        {
            st->it[0] = st->maxIter;
            st->done[0] = 1;
        }
        else if (it >= st->maxIter)
        {
            st->done[0] = 1;
        }
        st->allDone = st->done[0];
    }
}

/// p = z + beta p
template <class T = double>
__global__ void __launch_bounds__(TPB, kSolverMinBlocks) k_cg_pz(int n, const T* __restrict__ z, T* __restrict__ p, const SolveState* st)
{
    if (st->allDone) return;
    const T beta = static_cast<T>(st->beta[0]);
    FOR_ROWS(c, n) p[c] = z[c] + beta * p[c];
}

}  // namespace cfg
