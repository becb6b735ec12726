// The SIMPLE outer iteration on the device (src/3d/src/solvers/simpleSolver.cpp:33-394)
// and the host driver that sequences its kernels.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <type_traits>

#include "ctx.h"
#include "kernels.cuh"
#include "solvers.cuh"
#include "dic.cuh"

namespace cfg
{

// scalar slots of one outer iteration (device array scal_)
enum Slot
{
    S_CONT = 0,     // continuityError of the predictor flux
    S_CONT_AFTER,   // continuityError after correctFluxes
    S_PSTEP,        // max |pFull - p|
    S_PSCALE,       // max |p|
    S_AP,           // the pressure relaxation used
    S_PDELTA,       // max |aP (pFull - p)|
    S_UMAX,
    S_DUMAX,
    S_NONFINITE,
    S_NET,          // adjustPhi sums
    S_FREE,
    S_UINNER,       // device-side loops: momentum inner iterations, unconverged solves
    S_UUNCONV,
    S_TINNER,       // device-side loops: RANS model inner iterations, unconverged solves
    S_TUNCONV,
    S_PINNER,       // device-side loops: pressure inner iterations, unconverged solves
    S_PUNCONV,
    S_COUNT
};

// ---------------------------------------------------------------------------
// momentum assembly: fvm::div (divScheme.cpp:11-62) + fvm::laplacian with
// the harmonic face viscosity (laplacianScheme.cpp:146-215), sign -1, plus
// the deferred pressure-gradient source (simpleSolver.cpp:99-112).  One row
// per thread: the diagonal as the reference's face loops add into it (all
// convection terms in face order, then all diffusion terms), the row's
// entries in CSR column order, and the three base right-hand sides.
// ---------------------------------------------------------------------------

struct MomArgs
{
    const double* phi;
    const double* gamma;
    BcTab ub;
    double alpha;  // 0 upwind (and linear-upwind), 1 linear, blendCoeff for blend
    double force[3];
    CV3P gPn;
    int linUpwind;  // add the linear-upwind deferred correction from gUc
    CGrad3 gUc;     // grad of each U component, when linUpwind
    double* mVal;
    double* uDiag;
    V3P base;
    double dt;  // > 0: fvm::ddt(U, uOld, dt) first (divScheme.cpp:80-93)
    CV3P uOld;
};

__device__ __forceinline__ void div_weights(double p, double alpha, double ow, double& wPo, double& wNo)
{
    wPo = 0.0;
    wNo = 0.0;
    if (p >= 0) wPo = 1.0;
    else wNo = 1.0;
    if (alpha > 0)
    {
        wPo = alpha * ow + (1.0 - alpha) * wPo;
        wNo = alpha * (1.0 - ow) + (1.0 - alpha) * wNo;
    }
}

__global__ void __launch_bounds__(TPB) k_assemble_U(DMesh m, MomArgs a)
{
    ROW_LOOP(c, m.nC)
    {
        const int sl = c >> 5, lane = c & 31;
        const int e0 = m.cfStart[sl] + lane, e1 = m.cfStart[sl + 1];
        double diag = 0.0;
        double r0 = 0.0, r1 = 0.0, r2 = 0.0;
        if (a.dt > 0)
        {
            // the implicit Euler term, assembled before every face term
            const double at = m.V[c] / a.dt;
            diag = at;
            r0 = at * a.uOld.c[0][c];
            r1 = at * a.uOld.c[1][c];
            r2 = at * a.uOld.c[2][c];
        }
        for (int e = e0; e < e1; e += 32)  // convection
        {
            const int code = m.cfCode[e];
            if (code < 0) break;
            const int f = code >> 1, side = code & 1;
            const double p = a.phi[f];
            if (f < m.nI)
            {
                double wPo, wNo;
                div_weights(p, a.alpha, m.ow[f], wPo, wNo);
                diag += side ? -(p * wNo) : p * wPo;
            }
            else
            {
                const int b = m.cfOther[e];
                diag += p * a.ub.c[0][b];
                r0 += (-p) * a.ub.k[0][b];
                r1 += (-p) * a.ub.k[1][b];
                r2 += (-p) * a.ub.k[2][b];
            }
        }
        for (int e = e0; e < e1; e += 32)  // diffusion
        {
            const int code = m.cfCode[e];
            if (code < 0) break;
            const int f = code >> 1;
            const double coef = a.gamma[f] * m.oc[f];
            if (f < m.nI)
            {
                diag += coef;
            }
            else
            {
                const int b = m.cfOther[e];
                diag += (-coef) * (a.ub.c[0][b] - 1.0);
                r0 += coef * a.ub.k[0][b];
                r1 += coef * a.ub.k[1][b];
                r2 += coef * a.ub.k[2][b];
            }
        }
        const double v = m.V[c];
        r0 += ((a.force[0] + 0.0) - a.gPn.c[0][c]) * v;
        r1 += ((a.force[1] + 0.0) - a.gPn.c[1][c]) * v;
        r2 += ((a.force[2] + 0.0) - a.gPn.c[2][c]) * v;
        if (a.linUpwind)
        {
            // linear-upwind deferred correction: -phi_f (grad U)_u.(Cf - C_u)
            // on the owner row, + on the neighbour row, in face order
            double s0 = 0.0, s1 = 0.0, s2 = 0.0;
            for (int e = e0; e < e1; e += 32)
            {
                const int code = m.cfCode[e];
                if (code < 0) break;
                const int f = code >> 1, side = code & 1;
                if (f >= m.nI) continue;
                const double p = a.phi[f];
                const int u = p >= 0 ? m.own[f] : m.nbr[f];
                const double dx = m.fcx[f] - m.cx[u], dy = m.fcy[f] - m.cy[u], dz = m.fcz[f] - m.cz[u];
                const double k0 = p * (a.gUc.g[0].c[0][u] * dx + a.gUc.g[0].c[1][u] * dy + a.gUc.g[0].c[2][u] * dz);
                const double k1 = p * (a.gUc.g[1].c[0][u] * dx + a.gUc.g[1].c[1][u] * dy + a.gUc.g[1].c[2][u] * dz);
                const double k2 = p * (a.gUc.g[2].c[0][u] * dx + a.gUc.g[2].c[1][u] * dy + a.gUc.g[2].c[2][u] * dz);
                if (side)
                {
                    s0 = s0 + k0;
                    s1 = s1 + k1;
                    s2 = s2 + k2;
                }
                else
                {
                    s0 = s0 - k0;
                    s1 = s1 - k1;
                    s2 = s2 - k2;
                }
            }
            r0 += s0;
            r1 += s1;
            r2 += s2;
        }
        a.uDiag[c] = diag;
        a.base.c[0][c] = r0;
        a.base.c[1][c] = r1;
        a.base.c[2][c] = r2;
        const int me1 = m.mStart[sl + 1];
        for (int e = m.mStart[sl] + lane; e < me1; e += 32)
        {
            const int code = m.mCode[e];
            if (code == -1) break;
            double val;
            if (code == -2)
            {
                val = diag;
            }
            else
            {
                const int f = code >> 1, side = code & 1;
                const double p = a.phi[f];
                double wPo, wNo;
                div_weights(p, a.alpha, m.ow[f], wPo, wNo);
                const double conv = side ? -(p * wPo) : p * wNo;
                val = conv + (-(a.gamma[f] * m.oc[f]));
            }
            a.mVal[e] = val;
        }
    }
}

/// Pressure equation: fvm::laplacianFace(rAUf) sign -1 plus -div(phi)
/// (simpleSolver.cpp:265-273), and continuityError of the same flux
/// (pressureCorrection.cpp:90-125).
__global__ void __launch_bounds__(TPB) k_assemble_p(DMesh m, const double* __restrict__ phi,
                                                    const double* __restrict__ rAUf, const double* __restrict__ pc,
                                                    const double* __restrict__ pk, double* pVal, double* pDiag,
                                                    double* pBase, double* scal, int refCell, double refValue)
{
    double cmax = 0.0;
    ROW_LOOP(c, m.nC)
    {
        const int sl = c >> 5, lane = c & 31;
        const int e0 = m.cfStart[sl] + lane, e1 = m.cfStart[sl + 1];
        double dv = 0.0;
        for (int e = e0; e < e1; e += 32)
        {
            const int code = m.cfCode[e];
            if (code < 0) break;
            const double ph = phi[code >> 1];
            dv = (code & 1) ? dv - ph : dv + ph;
        }
        cmax = smax(cmax, fabs(dv) / smax(m.lscale[c], 1e-300));
        double diag = 0.0, r = 0.0;
        for (int e = e0; e < e1; e += 32)
        {
            const int code = m.cfCode[e];
            if (code < 0) break;
            const int f = code >> 1;
            const double coef = rAUf[f] * m.oc[f];
            if (f < m.nI)
            {
                diag += coef;
            }
            else
            {
                const int b = m.cfOther[e];
                diag += (-coef) * (pc[b] - 1.0);
                r += coef * pk[b];
            }
        }
        r += -dv;
        if (c == refCell)
        {
            r += diag * refValue;
            diag += diag;
        }
        pDiag[c] = diag;
        pBase[c] = r;
        const int me1 = m.mStart[sl + 1];
        for (int e = m.mStart[sl] + lane; e < me1; e += 32)
        {
            const int code = m.mCode[e];
            if (code == -1) break;
            pVal[e] = code == -2 ? diag : -(rAUf[code >> 1] * m.oc[code >> 1]);
        }
    }
    double v[1] = {cmax};
    block_max<1>(v);
    if (threadIdx.x == 0) atomic_max_nonneg(scal + S_CONT, v[0]);
}

/// continuityError alone (the corrected flux).
__global__ void __launch_bounds__(TPB) k_continuity(DMesh m, const double* __restrict__ phi, double* scal, int slot)
{
    double cmax = 0.0;
    ROW_LOOP(c, m.nC)
    {
        const int sl = c >> 5, lane = c & 31;
        double dv = 0.0;
        const int e1 = m.cfStart[sl + 1];
        for (int e = m.cfStart[sl] + lane; e < e1; e += 32)
        {
            const int code = m.cfCode[e];
            if (code < 0) break;
            const double ph = phi[code >> 1];
            dv = (code & 1) ? dv - ph : dv + ph;
        }
        cmax = smax(cmax, fabs(dv) / smax(m.lscale[c], 1e-300));
    }
    double v[1] = {cmax};
    block_max<1>(v);
    if (threadIdx.x == 0) atomic_max_nonneg(scal + slot, v[0]);
}

/// fvc::divPhi (interpolate.cpp:419-432)
__global__ void __launch_bounds__(TPB) k_divphi(DMesh m, const double* __restrict__ phi, double* out)
{
    ROW_LOOP(c, m.nC)
    {
        const int sl = c >> 5, lane = c & 31;
        double dv = 0.0;
        const int e1 = m.cfStart[sl + 1];
        for (int e = m.cfStart[sl] + lane; e < e1; e += 32)
        {
            const int code = m.cfCode[e];
            if (code < 0) break;
            const double ph = phi[code >> 1];
            dv = (code & 1) ? dv - ph : dv + ph;
        }
        out[c] = dv;
    }
}


/// rAU = V / aDiag and the pressure-free blend Hfree (simpleSolver.cpp:123-172).
__global__ void __launch_bounds__(TPB) k_hfree(DMesh m, const double* __restrict__ uDiag, CV3P U, CV3P x,
                                               double relaxU, V3P Hf, double* rAUr)
{
    ROW_LOOP(c, m.nC)
    {
        rAUr[c] = m.V[c] / smax(uDiag[c], 1e-300);
#pragma unroll
        for (int q = 0; q < 3; ++q) Hf.c[q][c] = (1.0 - relaxU) * U.c[q][c] + relaxU * x.c[q][c];
    }
}

/// phi from a cell vector field: updatePhiInternal (pressureCorrection.cpp:10-25)
/// and correctBoundaryFlux (volFields.cpp:294-306) under a linearisation table.
__global__ void __launch_bounds__(TPB) k_flux(DMesh m, CV3P H, BcTab hb, const int* __restrict__ emptyFace,
                                              double* phi)
{
    ROW_LOOP(f, m.nF)
    {
        const int o = m.own[f];
        double ux, uy, uz;
        if (f < m.nI)
        {
            const int n = m.nbr[f];
            const double w = m.ow[f], w1 = 1.0 - w;
            ux = H.c[0][o] * w + H.c[0][n] * w1;
            uy = H.c[1][o] * w + H.c[1][n] * w1;
            uz = H.c[2][o] * w + H.c[2][n] * w1;
        }
        else
        {
            const int b = f - m.nI;
            if (emptyFace && emptyFace[b])
            {
                phi[f] = 0.0;
                continue;
            }
            ux = hb.c[0][b] * H.c[0][o] + hb.k[0][b];
            uy = hb.c[1][b] * H.c[1][o] + hb.k[1][b];
            uz = hb.c[2][b] * H.c[2][o] + hb.k[2][b];
        }
        phi[f] = ux * m.sfx[f] + uy * m.sfy[f] + uz * m.sfz[f];
    }
}

/// internal phi only (updatePhiInternal), used for the initial flux
__global__ void __launch_bounds__(TPB) k_flux_internal(DMesh m, CV3P U, double* phi)
{
    ROW_LOOP(f, m.nI)
    {
        const int o = m.own[f], n = m.nbr[f];
        const double w = m.ow[f], w1 = 1.0 - w;
        const double ux = U.c[0][o] * w + U.c[0][n] * w1;
        const double uy = U.c[1][o] * w + U.c[1][n] * w1;
        const double uz = U.c[2][o] * w + U.c[2][n] * w1;
        phi[f] = ux * m.sfx[f] + uy * m.sfy[f] + uz * m.sfz[f];
    }
}

/// adjustPhi sums (simpleSolver.cpp:220-232), serial in the reference's
/// order: patch by patch, face by face.
__global__ void k_adjust_sums(const double* phi, const int* pStart, const int* pSize, const int* pFree, int nPatch,
                              double* scal)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    double netSum = 0, freeSum = 0;
    for (int pi = 0; pi < nPatch; ++pi)
    {
        double s = 0;
        for (int f = pStart[pi]; f < pStart[pi] + pSize[pi]; ++f) s += phi[f];
        netSum += s;
        if (pFree[pi]) freeSum += s;
    }
    scal[S_NET] = netSum;
    scal[S_FREE] = freeSum;
}

__global__ void __launch_bounds__(TPB) k_adjust_scale(int nB, int nI, const int* __restrict__ freeFace,
                                                      double* phi, const double* scal)
{
    const double freeSum = scal[S_FREE], netSum = scal[S_NET];
    if (!(fabs(freeSum) > 1e-30)) return;
    const double scale = (freeSum - netSum) / freeSum;
    ROW_LOOP(b, nB)
    if (freeFace[b]) phi[nI + b] *= scale;
}

/// interpolateToFaces (pressureCorrection.cpp:27-35)
__global__ void __launch_bounds__(TPB) k_face_interp(DMesh m, const double* __restrict__ cell, double* face)
{
    ROW_LOOP(f, m.nF)
    {
        const int o = m.own[f];
        face[f] = f < m.nI ? m.ow[f] * cell[o] + (1.0 - m.ow[f]) * cell[m.nbr[f]] : cell[o];
    }
}

/// correctFluxes (pressureCorrection.cpp:37-88)
__global__ void __launch_bounds__(TPB) k_correct_flux(DMesh m, const double* __restrict__ pF, CV3P gP,
                                                      const double* __restrict__ rAUf, const double* __restrict__ pc,
                                                      const double* __restrict__ pk, int corrected, double* phi)
{
    ROW_LOOP(f, m.nF)
    {
        const double d2 = m.dd2[f];
        if (d2 <= 0) continue;
        const double rf = rAUf[f];
        const double coef = rf * m.sfd[f] / d2;
        const int o = m.own[f];
        double corr = 0;
        if (corrected)
        {
            double gx, gy, gz;
            if (f < m.nI)
            {
                const int n = m.nbr[f];
                const double w = m.ow[f], w1 = 1.0 - w;
                gx = gP.c[0][o] * w + gP.c[0][n] * w1;
                gy = gP.c[1][o] * w + gP.c[1][n] * w1;
                gz = gP.c[2][o] * w + gP.c[2][n] * w1;
            }
            else
            {
                gx = gP.c[0][o];
                gy = gP.c[1][o];
                gz = gP.c[2][o];
            }
            corr = rf * (m.cvx[f] * gx + m.cvy[f] * gy + m.cvz[f] * gz);
        }
        if (f < m.nI)
        {
            const double dp = pF[m.nbr[f]] - pF[o];
            phi[f] = phi[f] - (coef * dp + corr);
        }
        else
        {
            const int b = f - m.nI;
            phi[f] = phi[f] - (coef * ((pc[b] - 1.0) * pF[o] + pk[b]) + corr);
        }
    }
}

/// max |pFull - p| and max |p| (simpleSolver.cpp:303-309)
__global__ void __launch_bounds__(TPB) k_pstep(int n, const double* __restrict__ pF, const double* __restrict__ p,
                                               double* scal)
{
    double v[2] = {0.0, 0.0};
    ROW_LOOP(c, n)
    {
        v[0] = smax(v[0], fabs(pF[c] - p[c]));
        v[1] = smax(v[1], fabs(p[c]));
    }
    block_max<2>(v);
    if (threadIdx.x == 0)
    {
        atomic_max_nonneg(scal + S_PSTEP, v[0]);
        atomic_max_nonneg(scal + S_PSCALE, v[1]);
    }
}

/// aP, the pressure relaxation and the velocity correction, and the
/// residual maxima (simpleSolver.cpp:310-348)
__global__ void __launch_bounds__(TPB) k_update(int n, const double* __restrict__ pF, double* p, V3P U, CV3P Hf,
                                                CV3P gPF, CV3P gPn, const double* __restrict__ rAUr, double relaxP,
                                                double pRelaxStart, double* scal)
{
    const double pStep = scal[S_PSTEP], pScale = scal[S_PSCALE];
    const double aP = pRelaxStart > 0 ? smin(relaxP, smax(pRelaxStart, 0.15 * pScale / smax(pStep, 1e-300))) : relaxP;
    double v[3] = {0.0, 0.0, 0.0};
    int bad = 0;
    ROW_LOOP(c, n)
    {
        const double po = p[c];
        const double dp = aP * (pF[c] - po);
        v[0] = smax(v[0], fabs(dp));
        const double pn = po + dp;
        p[c] = pn;
        const double s = aP * rAUr[c];
        double un[3], du[3];
#pragma unroll
        for (int q = 0; q < 3; ++q)
        {
            un[q] = Hf.c[q][c] - (gPF.c[q][c] - gPn.c[q][c]) * s;
            du[q] = un[q] - U.c[q][c];
            U.c[q][c] = un[q];
        }
        v[1] = smax(v[1], sqrt(un[0] * un[0] + un[1] * un[1] + un[2] * un[2]));
        v[2] = smax(v[2], sqrt(du[0] * du[0] + du[1] * du[1] + du[2] * du[2]));
        if (!isfinite(un[0]) || !isfinite(un[1]) || !isfinite(un[2]) || !isfinite(pn)) bad = 1;
    }
    block_max<3>(v);
    bad = __syncthreads_or(bad);
    if (threadIdx.x == 0)
    {
        atomic_max_nonneg(scal + S_PDELTA, v[0]);
        atomic_max_nonneg(scal + S_UMAX, v[1]);
        atomic_max_nonneg(scal + S_DUMAX, v[2]);
        if (bad) atomic_max_nonneg(scal + S_NONFINITE, 1.0);
        if (blockIdx.x == 0) scal[S_AP] = aP;
    }
}

__global__ void __launch_bounds__(TPB) k_axpby_rhs(int n, CV3P base, V3P rhs, int nc)
{
    ROW_LOOP(c, n)
    for (int q = 0; q < nc; ++q) rhs.c[q][c] = base.c[q][c];
}

/// h = rhs - (A x - diag x) (fvMatrix::explicitOperator, fvMatrix.cpp:131-146)
__global__ void __launch_bounds__(TPB) k_explicit_op(DMat A, const double* __restrict__ val,
                                                     const double* __restrict__ diag, const double* __restrict__ rhs,
                                                     const double* __restrict__ x, double* h)
{
    const double* xs[1] = {x};
    ROW_LOOP(c, A.n)
    {
        double y[1];
        spmv_row<0, 1>(A, val, c, xs, y);
        h[c] = rhs[c] - (y[0] - diag[c] * x[c]);
    }
}

/// Keeps the stream busy for about `us` microseconds (a fixed number of
/// sleeps; it waits on nothing).
__global__ void k_hold(int us)
{
    for (int i = 0; i < us; ++i) __nanosleep(1000);
}
/// the hold before an event-timed chunk: longer than the host takes to
/// enqueue one timed iteration (four kernels and five events)
constexpr int kHoldUs = 200;

__global__ void __launch_bounds__(TPB) k_fill(int n, double v, double* a)
{
    ROW_LOOP(i, n) a[i] = v;
}

__global__ void __launch_bounds__(TPB) k_to_float(int n, const double* __restrict__ a, float* __restrict__ b)
{
    ROW_LOOP(i, n) b[i] = static_cast<float>(a[i]);
}

/// x += e, e in single precision
__global__ void __launch_bounds__(TPB) k_add_f32(int n, const float* __restrict__ e, double* __restrict__ x)
{
    ROW_LOOP(i, n) x[i] = x[i] + static_cast<double>(e[i]);
}

/// PISO's pressure-free response (pisoSolver.cpp:118-139): rAU = V/aDiag and
/// HbyA = rAU (H(U) + V grad p^n) / V with H(U) = rhs - (A U - aDiag U), the
/// explicit operator of the momentum equation (fvMatrix.cpp:131-146)
template <int W>
__global__ void __launch_bounds__(TPB) k_piso_hbya(DMat A, const double* __restrict__ val,
                                                   const double* __restrict__ diag, CV3P rhs, CV3P U, CV3P gPn,
                                                   const double* __restrict__ V, double* __restrict__ rAU, V3P H)
{
    const double* xs[3] = {U.c[0], U.c[1], U.c[2]};
    ROW_LOOP(c, A.n)
    {
        double y[3];
        spmv_row<W, 3>(A, val, c, xs, y);
        const double d = diag[c], v = V[c];
        const double r = v / smax(d, 1e-300);
        rAU[c] = r;
#pragma unroll
        for (int q = 0; q < 3; ++q)
        {
            const double h = rhs.c[q][c] - (y[q] - d * U.c[q][c]);
            H.c[q][c] = r * (h + v * gPn.c[q][c]) / v;
        }
    }
}

/// U = HbyA - rAU grad p (pisoSolver.cpp:202-206)
__global__ void __launch_bounds__(TPB) k_piso_update(int n, CV3P H, const double* __restrict__ rAU, CV3P gP, V3P U)
{
    ROW_LOOP(c, n)
    {
#pragma unroll
        for (int q = 0; q < 3; ++q) U.c[q][c] = H.c[q][c] - rAU[c] * gP.c[q][c];
    }
}

// ===========================================================================
// host side
// ===========================================================================

namespace
{
inline double hdot(const Vec& a, const Vec& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
}

Ctx::Ctx(const Mesh& mesh, int device, cudaStream_t stream, int order)
    : mesh_(mesh), device_(device), stream_(stream), order_(order)
{
    if (mesh_.nCells >= (1LL << 30) || mesh_.nFaces() >= (1LL << 30))
        fail(CFG_EINVAL, "mesh too large for 32-bit device indices");
    CFG_CUDA(cudaSetDevice(device_));
    if (!stream_)
    {
        CFG_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
        ownStream_ = true;
    }
    if (const char* g = std::getenv("CHUANFLOW_GRAPHS")) useGraphs_ = std::strcmp(g, "0") != 0;
    const size_t nP = mesh_.patches.size();
    uType_.assign(nP, CFG_BC_ZERO_GRADIENT);
    pType_.assign(nP, CFG_BC_ZERO_GRADIENT);
    uVal_.assign(nP, Vec{});
    pVal_.assign(nP, 0.0);
    for (int i = 0; i < 16; ++i) CFG_CUDA(cudaEventCreate(&tm_.ev[i]));
    buildDevice();
}

Ctx::~Ctx()
{
    cudaSetDevice(device_);
    cudaStreamSynchronize(stream_);
    for (void* p : allocs_) cudaFree(p);
    if (stHost_) cudaFreeHost(stHost_);
    if (scalHost_) cudaFreeHost(scalHost_);
    for (int i = 0; i < 16; ++i) cudaEventDestroy(tm_.ev[i]);
    for (auto& e : kev_) cudaEventDestroy(e);
    for (auto& g : graphs_) cudaGraphExecDestroy(g.second);
    if (bodyStream_) cudaStreamDestroy(bodyStream_);
    if (ownStream_) cudaStreamDestroy(stream_);
}

void Ctx::buildDevice()
{
    const Mesh& M = mesh_;
    const int nC = static_cast<int>(M.nCells), nF = static_cast<int>(M.nFaces()), nI = static_cast<int>(M.nInternal());
    const int nB = nF - nI;
    nSlices_ = (nC + 31) / 32;
    DMesh& d = dm_;
    d.nC = nC;
    d.nF = nF;
    d.nI = nI;
    d.nB = nB;
    d.nRowsPad = nSlices_ * 32;
    int sms = 0;
    CFG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device_));
    G_ = std::max(1, std::min((nC + TPB - 1) / TPB, sms * 8));
    sms_ = sms;
    if (const char* e = std::getenv("CHUANFLOW_ROW_BLOCKS_PER_SM")) rowBlocksPerSM_ = std::max(0, std::atoi(e));
    if (const char* e = std::getenv("CHUANFLOW_PDL")) pdl_ = std::atoi(e) != 0;
    GS_ = rowGrid(nC);
    initRowBlocks_ = rowBlocksPerSM_;
    initGS_ = GS_;
    GF_ = std::max(1, std::min((nF + TPB - 1) / TPB, sms * 8));

    // ---- per-face geometry derived on the host in the reference's order ----
    std::vector<int> own(nF), nbr(std::max(nI, 1));
    std::vector<double> sfx(nF), sfy(nF), sfz(nF), oc(nF), sfd(nF), dd2(nF), cvx(nF), cvy(nF), cvz(nF);
    std::vector<double> wq(std::max(nI, 1)), skx(std::max(nI, 1)), sky(std::max(nI, 1)), skz(std::max(nI, 1));
    std::vector<double> fcx(nF), fcy(nF), fcz(nF), cx(nC), cy(nC), cz(nC), lscale(nC, 0.0);
    const std::vector<double> ow = M.ownerWeights();
    const std::vector<Vec> skew = M.skewVectors(ow);
    for (int f = 0; f < nF; ++f)
    {
        own[f] = static_cast<int>(M.owner[f]);
        const Vec& s = M.Sf[f];
        const Vec& dv = M.d[f];
        sfx[f] = s.x;
        sfy[f] = s.y;
        sfz[f] = s.z;
        const double d2 = hdot(dv, dv);
        dd2[f] = d2;
        sfd[f] = hdot(s, dv);
        oc[f] = hdot(s, dv) / d2;  // orthoCoeff (laplacianScheme.cpp:122-129)
        const double dm = std::sqrt(hdot(dv, dv));
        const Vec dh{dv.x / dm, dv.y / dm, dv.z / dm};
        const double sdh = hdot(s, dh);
        cvx[f] = s.x - dh.x * sdh;
        cvy[f] = s.y - dh.y * sdh;
        cvz[f] = s.z - dh.z * sdh;
        fcx[f] = M.Cf[f].x;
        fcy[f] = M.Cf[f].y;
        fcz[f] = M.Cf[f].z;
        const double a = M.magSf[f];
        const int o = own[f];
        lscale[o] = lscale[o] < a ? a : lscale[o];
        if (f < nI)
        {
            const int n = static_cast<int>(M.neighbour[f]);
            nbr[f] = n;
            lscale[n] = lscale[n] < a ? a : lscale[n];
            // volScalarField::faceValue weight (volFields.cpp:104-109)
            const Vec t = M.Cf[f] - M.C[o];
            const double x = d2 > 0 ? hdot(t, dv) / d2 : 0.0;
            const double mx0 = (0.0 < x) ? x : 0.0;
            wq[f] = d2 > 0 ? ((mx0 < 1.0) ? mx0 : 1.0) : 0.5;
            skx[f] = skew[f].x;
            sky[f] = skew[f].y;
            skz[f] = skew[f].z;
        }
    }
    for (int c = 0; c < nC; ++c)
    {
        cx[c] = M.C[c].x;
        cy[c] = M.C[c].y;
        cz[c] = M.C[c].z;
    }

    // ---- device numbering: slot i holds original cell perm_[i] ----
    {
        const std::vector<int64_t> o = cellOrder(M, order_);
        perm_.assign(o.begin(), o.end());
        inv_.assign(static_cast<size_t>(nC), 0);
        for (int i = 0; i < nC; ++i) inv_[perm_[i]] = i;
        identityOrder_ = true;
        for (int i = 0; i < nC && identityOrder_; ++i) identityOrder_ = perm_[i] == i;
        ioStage_ = alloc<double>(3 * static_cast<size_t>(nC));
        dPerm_ = identityOrder_ ? nullptr : upload(perm_);
    }
    const std::vector<int>& perm = perm_;
    const std::vector<int>& inv = inv_;

    // ---- cell -> face lists (ascending faces) and matrix rows ----
    std::vector<int> cnt(nC, 0), rowCnt(nC, 1);
    for (int f = 0; f < nF; ++f)
    {
        ++cnt[own[f]];
        if (f < nI)
        {
            ++cnt[nbr[f]];
            ++rowCnt[own[f]];
            ++rowCnt[nbr[f]];
        }
    }
    std::vector<int> cStart(nC + 1, 0);
    for (int c = 0; c < nC; ++c) cStart[c + 1] = cStart[c] + cnt[c];
    std::vector<int> listF(cStart[nC]), fill(nC, 0);
    for (int f = 0; f < nF; ++f)
    {
        const int o = own[f];
        listF[cStart[o] + fill[o]++] = f << 1;
        if (f < nI)
        {
            const int n = nbr[f];
            listF[cStart[n] + fill[n]++] = (f << 1) | 1;
        }
    }
    // slices of 32 device slots; widths from the cells they hold
    std::vector<int> cfStart(nSlices_ + 1, 0), mStart(nSlices_ + 1, 0);
    for (int s = 0; s < nSlices_; ++s)
    {
        int w = 0, wm = 0;
        for (int l = 0; l < 32; ++l)
        {
            const int i = 32 * s + l;
            if (i >= nC) break;
            w = std::max(w, cnt[perm[i]]);
            wm = std::max(wm, rowCnt[perm[i]]);
        }
        cfStart[s + 1] = cfStart[s] + 32 * w;
        mStart[s + 1] = mStart[s] + 32 * wm;
        maxW_ = std::max(maxW_, wm);
    }
    std::vector<int> cfCode(cfStart[nSlices_], -1), cfOther(cfStart[nSlices_], 0);
    std::vector<int> mCol(mStart[nSlices_], -1), mCode(mStart[nSlices_], -1);
    std::vector<std::pair<int, int>> row;  // (original col, code)
    for (int i = 0; i < nC; ++i)
    {
        const int c = perm[i];
        const int s = i >> 5, l = i & 31;
        row.clear();
        row.push_back({c, -2});
        for (int k = 0; k < cnt[c]; ++k)
        {
            const int code = listF[cStart[c] + k];
            const int f = code >> 1;
            const int e = cfStart[s] + 32 * k + l;
            cfCode[e] = code;
            if (f < nI)
            {
                const int other = (code & 1) ? own[f] : nbr[f];
                cfOther[e] = inv[other];
                row.push_back({other, code});
            }
            else
            {
                cfOther[e] = f - nI;
            }
        }
        // CSR column order of the original numbering (Matrix.cpp:72-76);
        // entries with equal columns (two faces between the same cells) stay
        // separate, in face order
        std::stable_sort(row.begin(), row.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
        for (size_t k = 0; k < row.size(); ++k)
        {
            const int e = mStart[s] + 32 * static_cast<int>(k) + l;
            mCol[e] = inv[row[k].first];
            mCode[e] = row[k].second;
        }
    }

    // ---- multicolour DIC layouts (dic.cuh) ----
    {
        int nCol = 0;
        const std::vector<int> colourOrig = greedyColours(cellGraph(M), &nCol);
        std::vector<int> colour(nC);
        for (int i = 0; i < nC; ++i) colour[i] = colourOrig[perm[i]];
        nColours_ = nCol;
        std::vector<int> rows;
        std::vector<int> lStart{0}, uStart{0}, lCol, lSrc, uCol, uSrc;
        dicPhase_.clear();
        int slice = 0, pOff = 0;
        for (int col = 0; col < nCol; ++col)
        {
            DicPhase ph{static_cast<int>(rows.size()), 0, slice, pOff};
            for (int c = 0; c < nC; ++c)
                if (colour[c] == col) rows.push_back(c);
            ph.cnt = static_cast<int>(rows.size()) - ph.off;
            const int nSl = (ph.cnt + 31) / 32;
            for (int sl = 0; sl < nSl; ++sl)
            {
                std::vector<std::vector<std::pair<int, int>>> lo(32), up(32);
                int wl = 0, wu = 0;
                for (int l = 0; l < 32; ++l)
                {
                    const int t = 32 * sl + l;
                    if (t >= ph.cnt) break;
                    const int c = rows[ph.off + t];
                    const int s0 = c >> 5, l0 = c & 31;
                    for (int k = 0;; ++k)
                    {
                        const int e = mStart[s0] + 32 * k + l0;
                        if (e >= mStart[s0 + 1] || mCol[e] < 0) break;
                        const int j = mCol[e];
                        if (j == c) continue;
                        (colour[j] < col ? lo : up)[l].push_back({j, e});
                    }
                    wl = std::max(wl, static_cast<int>(lo[l].size()));
                    wu = std::max(wu, static_cast<int>(up[l].size()));
                }
                const size_t lb = lCol.size(), ub = uCol.size();
                lCol.resize(lb + 32 * wl, -1);
                lSrc.resize(lb + 32 * wl, -1);
                uCol.resize(ub + 32 * wu, -1);
                uSrc.resize(ub + 32 * wu, -1);
                for (int l = 0; l < 32; ++l)
                {
                    for (size_t k = 0; k < lo[l].size(); ++k)
                    {
                        lCol[lb + 32 * k + l] = lo[l][k].first;
                        lSrc[lb + 32 * k + l] = lo[l][k].second;
                    }
                    for (size_t k = 0; k < up[l].size(); ++k)
                    {
                        uCol[ub + 32 * k + l] = up[l][k].first;
                        uSrc[ub + 32 * k + l] = up[l][k].second;
                    }
                }
                lStart.push_back(static_cast<int>(lCol.size()));
                uStart.push_back(static_cast<int>(uCol.size()));
            }
            slice += nSl;
            pOff += rowGrid(ph.cnt);
            dicPhase_.push_back(ph);
        }
        dicPartials_ = pOff + 1;
        initDicPartials_ = dicPartials_;
        dic_.nColours = nCol;
        dic_.rows = upload(rows);
        dic_.lStart = upload(lStart);
        dic_.lCol = upload(lCol);
        dic_.lSrc = upload(lSrc);
        dic_.uStart = upload(uStart);
        dic_.uCol = upload(uCol);
        dic_.uSrc = upload(uSrc);
        dic_.lVal = alloc<double>(lCol.size());
        dic_.uVal = alloc<double>(uCol.size());
        dic_.rD = alloc<double>(nC);
        dic_.rDinv = alloc<double>(nC);
        nLo_ = static_cast<int>(lCol.size());
        nUp_ = static_cast<int>(uCol.size());
    }

    {
        std::vector<int> ownN(nF), nbrN(std::max(nI, 1));
        for (int f = 0; f < nF; ++f) ownN[f] = inv[own[f]];
        for (int f = 0; f < nI; ++f) nbrN[f] = inv[nbr[f]];
        d.own = upload(ownN);
        d.nbr = upload(nbrN);
    }
    d.sfx = upload(sfx);
    d.sfy = upload(sfy);
    d.sfz = upload(sfz);
    {
        std::vector<double> owv(ow.begin(), ow.end());
        d.ow = upload(owv);
    }
    d.wq = upload(wq);
    d.skx = upload(skx);
    d.sky = upload(sky);
    d.skz = upload(skz);
    d.oc = upload(oc);
    d.sfd = upload(sfd);
    d.dd2 = upload(dd2);
    d.cvx = upload(cvx);
    d.cvy = upload(cvy);
    d.cvz = upload(cvz);
    auto permuted = [&](const std::vector<double>& a) {
        std::vector<double> b(static_cast<size_t>(nC));
        for (int i = 0; i < nC; ++i) b[i] = a[perm[i]];
        return b;
    };
    d.V = upload(permuted(M.V));
    d.lscale = upload(permuted(lscale));
    d.cx = upload(permuted(cx));
    d.cy = upload(permuted(cy));
    d.cz = upload(permuted(cz));
    d.fcx = upload(fcx);
    d.fcy = upload(fcy);
    d.fcz = upload(fcz);
    d.cfStart = upload(cfStart);
    d.cfCode = upload(cfCode);
    d.cfOther = upload(cfOther);
    d.mStart = upload(mStart);
    nSlicesEntries_ = mStart[nSlices_];
    d.mCol = upload(mCol);
    d.mCode = upload(mCode);

    const size_t nE = static_cast<size_t>(mStart[nSlices_]);
    auto v3 = [&](V3P& v, size_t n) {
        for (int q = 0; q < 3; ++q) v.c[q] = alloc<double>(n);
    };
    for (int q = 0; q < 3; ++q)
    {
        uc_[q] = alloc<double>(nB);
        uk_[q] = alloc<double>(nB);
        hc_[q] = alloc<double>(nB);
        hk_[q] = alloc<double>(nB);
    }
    pc_ = alloc<double>(nB);
    pk_ = alloc<double>(nB);
    v3(U_, nC);
    v3(gPn_, nC);
    v3(gPF_, nC);
    v3(Hf_, nC);
    v3(gA_, nC);
    v3(gB_, nC);
    v3(uBase_, nC);
    v3(uRhs_, nC);
    v3(ux_, nC);
    p_ = alloc<double>(nC);
    phi_ = alloc<double>(nF);
    rAUr_ = alloc<double>(nC);
    rAUf_ = alloc<double>(nF);
    uDiag_ = alloc<double>(nC);
    pDiag_ = alloc<double>(nC);
    pBase_ = alloc<double>(nC);
    pRhs_ = alloc<double>(nC);
    px_ = alloc<double>(nC);
    mVal_ = alloc<double>(nE);
    pVal_d_ = alloc<double>(nE);
    cr_ = alloc<double>(nC);
    cp_ = alloc<double>(nC);
    cAp_ = alloc<double>(nC);
    cz_ = alloc<double>(nC);
    v3(br_, nC);
    v3(br0_, nC);
    v3(bp_, nC);
    v3(bv_, nC);
    v3(bs_, nC);
    v3(bsh_, nC);
    v3(bt_, nC);
    v3(bz_, nC);
    bInvD_ = alloc<double>(nC);
    gU_ = alloc<double>(nF);
    fScratch_ = alloc<double>(nF);
    bScratch_ = alloc<double>(2 * static_cast<size_t>(nB));
    {
        std::vector<int> ps, pz;
        for (const auto& p : M.patches)
        {
            ps.push_back(static_cast<int>(p.start));
            pz.push_back(static_cast<int>(p.size));
        }
        dpStart_ = upload(ps);
        dpSize_ = upload(pz);
        dpFree_ = alloc<int>(ps.size());
        dFreeFace_ = alloc<int>(nB);
        dEmptyFace_ = alloc<int>(nB);
    }
    partials_ = alloc<double>(static_cast<size_t>(16) * std::max(std::max(std::max(G_, GF_), GS_), dicPartials_));
    st_ = alloc<SolveState>(1);
    scal_ = alloc<double>(S_COUNT);
    loopCount_ = alloc<int>(1);
    CFG_CUDA(cudaStreamCreateWithFlags(&bodyStream_, cudaStreamNonBlocking));
    CFG_CUDA(cudaMallocHost(&stHost_, sizeof(SolveState)));
    CFG_CUDA(cudaMallocHost(&scalHost_, sizeof(double) * S_COUNT));
    CFG_CUDA(cudaStreamSynchronize(stream_));
}

void Ctx::setPatchBC(char field, int patch, int type, const double* value)
{
    if (patch < 0 || patch >= static_cast<int>(mesh_.patches.size())) fail(CFG_EINVAL, "patch index out of range");
    if (type < CFG_BC_FIXED_VALUE || type > CFG_BC_EMPTY) fail(CFG_EINVAL, "unknown boundary-condition type");
    if (field == 'U')
    {
        uType_[patch] = type;
        uVal_[patch] = value ? Vec{value[0], value[1], value[2]} : Vec{};
    }
    else if (field == 'p')
    {
        pType_[patch] = type;
        pVal_[patch] = value ? value[0] : 0.0;
    }
    else
    {
        fail(CFG_EINVAL, "field must be 'U' or 'p'");
    }
    bcDirty_ = true;
}

void Ctx::setFaceValuesU(int64_t n, const int64_t* faces, const double* values)
{
    for (int64_t i = 0; i < n; ++i)
    {
        const int64_t f = faces[i];
        if (f < mesh_.nInternal() || f >= mesh_.nFaces())
            fail(CFG_EINVAL, "volVectorField::setFaceValue: internal face " + std::to_string(f));
        uFace_[f] = Vec{values[3 * i], values[3 * i + 1], values[3 * i + 2]};
    }
    bcDirty_ = true;
}

void Ctx::clearFaceValuesU()
{
    uFace_.clear();
    bcDirty_ = true;
}

namespace
{
// volVectorField::linearise for one face and component (volFields.cpp:246-283)
void linVector(const Mesh& M, int type, const Vec& patchVal, const Vec* faceVal, int64_t f, int comp, double& c,
               double& k)
{
    const Vec value = faceVal ? *faceVal : patchVal;
    auto cmp = [](const Vec& v, int q) { return q == 0 ? v.x : (q == 1 ? v.y : v.z); };
    switch (type)
    {
    case CFG_BC_FIXED_VALUE:
        c = 0;
        k = cmp(value, comp);
        return;
    case CFG_BC_FIXED_GRADIENT:
    {
        const Vec& sf = M.Sf[f];
        const double a = std::sqrt(hdot(sf, sf));
        const Vec n{sf.x / a, sf.y / a, sf.z / a};
        c = 1;
        k = cmp(patchVal, comp) * hdot(M.d[f], n);
        return;
    }
    case CFG_BC_ZERO_GRADIENT:
    case CFG_BC_OUTLET:
        c = 1;
        k = 0;
        return;
    case CFG_BC_SYMMETRY:
    case CFG_BC_WALL:
    {
        const Vec& sf = M.Sf[f];
        const double a = std::sqrt(hdot(sf, sf));
        const double ax = std::abs(sf.x / a), ay = std::abs(sf.y / a), az = std::abs(sf.z / a);
        int axis;
        double big;
        if (ax >= ay && ax >= az) { axis = 0; big = ax; }
        else if (ay >= az) { axis = 1; big = ay; }
        else { axis = 2; big = az; }
        if (big < 1.0 - 1e-6) fail(CFG_ESETUP, "fields: symmetry normal not axis aligned");
        c = (comp == axis) ? 0.0 : 1.0;
        k = 0;
        return;
    }
    default:
        fail(CFG_ESETUP, "volVectorField: unknown patch bc type");
    }
}

// volScalarField::linearise (volFields.cpp:117-147)
void linScalar(const Mesh& M, int type, double value, int64_t f, double& c, double& k)
{
    switch (type)
    {
    case CFG_BC_FIXED_VALUE:
        c = 0;
        k = value;
        return;
    case CFG_BC_FIXED_GRADIENT:
    {
        const Vec& sf = M.Sf[f];
        const double a = std::sqrt(hdot(sf, sf));
        const Vec n{sf.x / a, sf.y / a, sf.z / a};
        c = 1;
        k = value * hdot(M.d[f], n);
        return;
    }
    case CFG_BC_ZERO_GRADIENT:
    case CFG_BC_SYMMETRY:
    case CFG_BC_OUTLET:
        c = 1;
        k = 0;
        return;
    default:
        fail(CFG_ESETUP, "volScalarField: unknown patch bc type");
    }
}
}  // namespace

void Ctx::refreshBc()
{
    if (!bcDirty_) return;
    const Mesh& M = mesh_;
    const int64_t nI = M.nInternal(), nB = M.nBoundary();
    std::vector<double> uc[3], uk[3], hc[3], hk[3], pc(nB), pk(nB);
    for (int q = 0; q < 3; ++q)
    {
        uc[q].resize(nB);
        uk[q].resize(nB);
        hc[q].resize(nB);
        hk[q].resize(nB);
    }
    nFreeUFaces_ = 0;
    for (int64_t b = 0; b < nB; ++b)
    {
        const int64_t f = nI + b;
        const int pi = static_cast<int>(M.facePatch[f]);
        auto it = uFace_.find(f);
        const Vec* fv = it == uFace_.end() ? nullptr : &it->second;
        const int ut = uType_[pi];
        // constrainHbyA (simpleSolver.cpp:175-187): fixedValue where U is,
        // zeroGradient elsewhere, with U's per-face values adopted
        const bool fixed = ut == CFG_BC_FIXED_VALUE;
        for (int q = 0; q < 3; ++q)
        {
            if (ut == CFG_BC_EMPTY)
            {
                uc[q][b] = 0;
                uk[q][b] = 0;
            }
            else
            {
                linVector(M, ut, uVal_[pi], fv, f, q, uc[q][b], uk[q][b]);
            }
            linVector(M, fixed ? CFG_BC_FIXED_VALUE : CFG_BC_ZERO_GRADIENT, fixed ? uVal_[pi] : Vec{}, fv, f, q,
                      hc[q][b], hk[q][b]);
        }
        const int pt = pType_[pi];
        if (pt == CFG_BC_FIXED_VALUE || pt == CFG_BC_FIXED_GRADIENT || pt == CFG_BC_ZERO_GRADIENT ||
            pt == CFG_BC_SYMMETRY || pt == CFG_BC_OUTLET)
            linScalar(M, pt, pVal_[pi], f, pc[b], pk[b]);
        else
            pc[b] = pk[b] = NAN;  // rejected when the pressure equation is built
        if (!fixed) ++nFreeUFaces_;
    }
    for (int q = 0; q < 3; ++q)
    {
        CFG_CUDA(cudaMemcpyAsync(uc_[q], uc[q].data(), nB * sizeof(double), cudaMemcpyHostToDevice, stream_));
        CFG_CUDA(cudaMemcpyAsync(uk_[q], uk[q].data(), nB * sizeof(double), cudaMemcpyHostToDevice, stream_));
        CFG_CUDA(cudaMemcpyAsync(hc_[q], hc[q].data(), nB * sizeof(double), cudaMemcpyHostToDevice, stream_));
        CFG_CUDA(cudaMemcpyAsync(hk_[q], hk[q].data(), nB * sizeof(double), cudaMemcpyHostToDevice, stream_));
    }
    {
        std::vector<int> pfree(M.patches.size()), ffree(nB), fempty(nB);
        needReference_ = true;
        for (size_t pi = 0; pi < M.patches.size(); ++pi)
        {
            pfree[pi] = uType_[pi] != CFG_BC_FIXED_VALUE;
            if (pType_[pi] == CFG_BC_FIXED_VALUE) needReference_ = false;
        }
        for (int64_t b = 0; b < nB; ++b)
        {
            const int pi = static_cast<int>(M.facePatch[nI + b]);
            ffree[b] = pfree[pi];
            fempty[b] = uType_[pi] == CFG_BC_EMPTY;
        }
        if (!pfree.empty())
            CFG_CUDA(cudaMemcpyAsync(dpFree_, pfree.data(), pfree.size() * sizeof(int), cudaMemcpyHostToDevice, stream_));
        CFG_CUDA(cudaMemcpyAsync(dFreeFace_, ffree.data(), nB * sizeof(int), cudaMemcpyHostToDevice, stream_));
        CFG_CUDA(cudaMemcpyAsync(dEmptyFace_, fempty.data(), nB * sizeof(int), cudaMemcpyHostToDevice, stream_));
        CFG_CUDA(cudaStreamSynchronize(stream_));
    }
    CFG_CUDA(cudaMemcpyAsync(pc_, pc.data(), nB * sizeof(double), cudaMemcpyHostToDevice, stream_));
    CFG_CUDA(cudaMemcpyAsync(pk_, pk.data(), nB * sizeof(double), cudaMemcpyHostToDevice, stream_));
    CFG_CUDA(cudaStreamSynchronize(stream_));
    bcDirty_ = false;
}

/// With linear-upwind convection, the gradient of the three U components
/// (the iterate the momentum equation is assembled from; internal faces by
/// the bounded owner weight, as makeFaceValueFn) into gA_, gB_, Hf_, which
/// the momentum solve only overwrites after assembly; returns 1 then.
int Ctx::linUpwindGrad(const BcTab& ub, int gradScheme)
{
    if (schemes_.div != CFG_DIV_LINEAR_UPWIND) return 0;
    const double* xs[3] = {U_.c[0], U_.c[1], U_.c[2]};
    V3P g[3] = {gA_, gB_, Hf_};
    gradCells(xs, 3, ub, gradScheme, false, g);
    return 1;
}

void Ctx::launchCheck(const char* what, int kernels)
{
    launches_ += kernels;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) fail(CFG_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}


/// fvc::grad of NC cell fields into gA_ (NC = 1) or gA_/gB_/... (see callers):
/// scheme linear | corrected | leastSquares; volQuirk selects the
/// volScalarField overload's internal face value for the linear scheme.
void Ctx::gradCells(const double* const* x, int nComp, const BcTab& bc, int scheme, bool volQuirk, V3P* out)
{
    // the kernels come in one- and three-field forms; any other count would
    // leave output pointers unset
    if (nComp != 1 && nComp != 3) fail(CFG_EINVAL, "gradCells: one or three fields per call");
    CV3P xs{{x[0], nComp > 1 ? x[1] : x[0], nComp > 2 ? x[2] : x[0]}};
    Grad3 o{};
    for (int q = 0; q < nComp; ++q) o.g[q] = out[q];
    if (scheme == CFG_GRAD_LEAST_SQUARES)
    {
        // stage 1 into out, stage 2 reads it and writes the scratch set, then copy back
        if (nComp == 1)
        {
            k_grad_ls1<1><<<G_, TPB, 0, stream_>>>(dm_, xs, bc, o);
            launchCheck("grad_ls1");
            Grad3 o2{};
            o2.g[0] = gB_;
            k_grad_ls2<1><<<G_, TPB, 0, stream_>>>(dm_, xs, bc, CGrad3{{cv(out[0])}}, o2);
            launchCheck("grad_ls2");
            for (int q = 0; q < 3; ++q)
                CFG_CUDA(cudaMemcpyAsync(out[0].c[q], gB_.c[q], dm_.nC * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
        }
        else
        {
            // three components: stage 1 into out, stage 2 into the U-equation
            // scratch (solver work vectors are free while gradients run)
            k_grad_ls1<3><<<G_, TPB, 0, stream_>>>(dm_, xs, bc, o);
            launchCheck("grad_ls1");
            Grad3 o2{};
            o2.g[0] = bs_;
            o2.g[1] = bsh_;
            o2.g[2] = bt_;
            k_grad_ls2<3><<<G_, TPB, 0, stream_>>>(dm_, xs, bc, CGrad3{{cv(out[0]), cv(out[1]), cv(out[2])}}, o2);
            launchCheck("grad_ls2");
            for (int q = 0; q < 3; ++q)
                for (int k = 0; k < 3; ++k)
                    CFG_CUDA(cudaMemcpyAsync(out[q].c[k], o2.g[q].c[k], dm_.nC * sizeof(double),
                                             cudaMemcpyDeviceToDevice, stream_));
        }
        return;
    }
    const bool corrected = scheme == CFG_GRAD_CORRECTED;
    if (nComp == 1)
    {
        k_grad_gauss0<1><<<G_, TPB, 0, stream_>>>(dm_, xs, bc, (!corrected && volQuirk) ? 1 : 0, o);
        launchCheck("grad_gauss0");
        if (!corrected) return;
        Grad3 t{};
        t.g[0] = gB_;
        k_grad_gauss_corr<1><<<G_, TPB, 0, stream_>>>(dm_, xs, bc, CGrad3{{cv(out[0])}}, t);
        launchCheck("grad_corr");
        k_grad_gauss_corr<1><<<G_, TPB, 0, stream_>>>(dm_, xs, bc, CGrad3{{cv(gB_)}}, o);
        launchCheck("grad_corr");
    }
    else
    {
        k_grad_gauss0<3><<<G_, TPB, 0, stream_>>>(dm_, xs, bc, 0, o);
        launchCheck("grad_gauss0");
        if (!corrected) return;
        Grad3 t{};
        t.g[0] = bs_;
        t.g[1] = bsh_;
        t.g[2] = bt_;
        k_grad_gauss_corr<3><<<G_, TPB, 0, stream_>>>(dm_, xs, bc, CGrad3{{cv(out[0]), cv(out[1]), cv(out[2])}}, t);
        launchCheck("grad_corr");
        k_grad_gauss_corr<3><<<G_, TPB, 0, stream_>>>(dm_, xs, bc, CGrad3{{cv(bs_), cv(bsh_), cv(bt_)}}, o);
        launchCheck("grad_corr");
    }
}

namespace
{
/// Calls f(std::integral_constant<int, W>) with the smallest compiled row
/// width W that holds every row (0: rows of any length).
template <class F>
void dispatchW(int maxW, F&& f)
{
    if (maxW <= 7) f(std::integral_constant<int, 7>{});
    else if (maxW <= 16) f(std::integral_constant<int, 16>{});
    else f(std::integral_constant<int, 0>{});
}
}  // namespace

/// Enqueues body(0..n-1) -- n solver iterations -- on the stream.  The
/// first time a (key, n) pair is seen the iterations are captured into a
/// CUDA graph, which later calls replay: a chunk then costs one launch.
/// key must name everything the kernels' arguments depend on.
template <class F>
void Ctx::launchChunk(const std::string& key, int n, F&& body)
{
    // Event-timed iterations stay eager: an event recorded during capture
    // becomes a graph dependency, not a timestamp.
    // The caller counts the chunk's kernels; counts taken inside body are
    // dropped so eager and replayed chunks count alike.
    const int64_t counted = launches_;
    if (!useGraphs_ || ktime_)
    {
        // a timed chunk starts behind a short sleep, so that its events and
        // kernels are all queued before the GPU reaches the first event: on
        // an idle stream an event's timestamp would also hold the time the
        // host took to submit the kernel after it
        if (ktime_) k_hold<<<1, 32, 0, stream_>>>(kHoldUs);
        for (int i = 0; i < n; ++i) body(i);
        launches_ = counted;
        return;
    }
    const std::string k = key + "#" + std::to_string(n) + (ktime_ ? "t" : "");
    auto it = graphs_.find(k);
    if (it == graphs_.end())
    {
        cudaGraph_t g = nullptr;
        CFG_CUDA(cudaStreamBeginCapture(stream_, cudaStreamCaptureModeThreadLocal));
        for (int i = 0; i < n; ++i) body(i);
        launches_ = counted;
        CFG_CUDA(cudaStreamEndCapture(stream_, &g));
        cudaGraphExec_t ge = nullptr;
        const cudaError_t e = cudaGraphInstantiate(&ge, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) fail(CFG_ECUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
        it = graphs_.emplace(k, ge).first;
    }
    CFG_CUDA(cudaGraphLaunch(it->second, stream_));
}

/// Appends to the graph being captured on stream_ a conditional while-node
/// whose body holds what body() enqueues followed by k_loop_cond on the
/// solver state st_: the device re-runs the body until the solve is done.
/// The body is captured on bodyStream_ into the node's own graph.
template <class F>
void Ctx::captureWhile(int maxBodies, F&& body)
{
    CFG_CUDA(cudaMemsetAsync(loopCount_, 0, sizeof(int), stream_));
    cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nDeps = 0;
    CFG_CUDA(cudaStreamGetCaptureInfo(stream_, &cs, nullptr, &g, &deps, &nDeps));
    if (cs != cudaStreamCaptureStatusActive) fail(CFG_EINVAL, "device loops need a stream under capture");
    cudaGraphConditionalHandle h;
    CFG_CUDA(cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault));
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    CFG_CUDA(cudaGraphAddNode(&node, g, deps, nDeps, &np));
    CFG_CUDA(cudaStreamUpdateCaptureDependencies(stream_, &node, 1, cudaStreamSetCaptureDependencies));
    cudaGraph_t bodyGraph = np.conditional.phGraph_out[0];
    CFG_CUDA(cudaStreamBeginCaptureToGraph(bodyStream_, bodyGraph, nullptr, nullptr, 0,
                                           cudaStreamCaptureModeThreadLocal));
    const cudaStream_t outer = stream_;
    stream_ = bodyStream_;
    try
    {
        body();
        k_loop_cond<<<1, 32, 0, stream_>>>(h, st_, loopCount_, maxBodies);
        launchCheck("loop_cond");
    }
    catch (...)
    {
        stream_ = outer;
        cudaGraph_t junk = nullptr;
        cudaStreamEndCapture(bodyStream_, &junk);
        throw;
    }
    stream_ = outer;
    cudaGraph_t captured = nullptr;
    CFG_CUDA(cudaStreamEndCapture(bodyStream_, &captured));
}

namespace
{
std::string ptrKey(const char* kind, std::initializer_list<const void*> ps, int extra = 0)
{
    std::string s(kind);
    char buf[32];
    for (const void* p : ps)
    {
        std::snprintf(buf, sizeof buf, ":%p", p);
        s += buf;
    }
    std::snprintf(buf, sizeof buf, ":%d", extra);
    return s + buf;
}
}  // namespace

void Ctx::runCG(const double* vals, const double* diag, const double* b, double* x, double tol, int maxIter,
                cfg_solver_report* rep, int normType)
{
    const DMat A{dm_.nC, dm_.mStart, dm_.mCol};
    SolveState init{};
    init.tol = tol;
    init.maxIter = maxIter;
    init.nComp = 1;
    init.normType = normType;
    CFG_CUDA(cudaMemcpyAsync(st_, &init, sizeof(SolveState), cudaMemcpyHostToDevice, stream_));
    if (devLoop_)
    {
        k_state_reset<<<1, 32, 0, stream_>>>(st_, tol, maxIter, 1, normType);
        dispatchW(maxW_, [&](auto Wc) {
            constexpr int W = decltype(Wc)::value;
            k_cg_init<W><<<GS_, TPB, 0, stream_>>>(A, vals, diag, b, x, cr_, cp_, partials_, st_);
            constexpr int CH = 8;
            captureWhile((maxIter + CH - 1) / CH + 1, [&] {
                for (int k = 0; k < CH; ++k)
                {
                    k_cg_spmv<W><<<GS_, TPB, 0, stream_>>>(A, vals, cp_, cAp_, partials_, st_);
                    k_cg_update<double><<<GS_, TPB, 0, stream_>>>(dm_.nC, diag, cp_, cAp_, x, cr_, partials_, st_);
                    k_cg_p<double><<<GS_, TPB, 0, stream_>>>(dm_.nC, diag, cr_, cp_, st_);
                }
                launchCheck("cg_iter", 0);
            });
        });
        if (tally_) k_state_tally<<<1, 32, 0, stream_>>>(st_, 1, tally_);
        launchCheck("cg_tally");
        *rep = cfg_solver_report{};
        return;
    }
    dispatchW(maxW_, [&](auto Wc) {
        constexpr int W = decltype(Wc)::value;
        k_cg_init<W><<<GS_, TPB, 0, stream_>>>(A, vals, diag, b, x, cr_, cp_, partials_, st_);
        launchCheck("cg_init");
        int launched = 0;
        int chunk = 8;
        int itBefore = 0, lastChunk = 0;
        for (;;)
        {
            CFG_CUDA(cudaMemcpyAsync(stHost_, st_, sizeof(SolveState), cudaMemcpyDeviceToHost, stream_));
            CFG_CUDA(cudaStreamSynchronize(stream_));
            if (lastChunk > 0)
            {
                // only the iterations that ran (the rest returned on the done flag)
                static const int slots[3] = {KS_CG_SPMV, KS_CG_UPDATE, KS_CG_P};
                harvest(std::min(lastChunk, std::max(0, stHost_->it[0] - itBefore)), slots, 3);
            }
            itBefore = stHost_->it[0];
            if (stHost_->allDone || launched >= maxIter) break;
            const int n = std::min(chunk, maxIter - launched);
            launchChunk(ptrKey("cg", {vals, diag, x}, W), n, [&](int k) {
                tmark(k, 0);
                k_cg_spmv<W><<<GS_, TPB, 0, stream_>>>(A, vals, cp_, cAp_, partials_, st_);
                tmark(k, 1);
                k_cg_update<double><<<GS_, TPB, 0, stream_>>>(dm_.nC, diag, cp_, cAp_, x, cr_, partials_, st_);
                tmark(k, 2);
                k_cg_p<double><<<GS_, TPB, 0, stream_>>>(dm_.nC, diag, cr_, cp_, st_);
                tmark(k, 3);
                launchCheck("cg_iter", 0);
            });
            launches_ += 3 * n;
            launched += n;
            lastChunk = n;
            chunk = std::min(chunk * 2, 64);
        }
    });
    rep->iterations = stHost_->it[0];
    rep->converged = stHost_->conv[0];
    rep->initial_residual = stHost_->init[0];
    rep->final_residual = stHost_->conv[0] && stHost_->it[0] == 0 ? stHost_->init[0] : stHost_->fin[0];
}

void Ctx::runBiCG3(const double* vals, const double* diag, V3P b, V3P x, int nComp, double tol, int maxIter,
                   cfg_solver_report* reps)
{
    const DMat A{dm_.nC, dm_.mStart, dm_.mCol};
    SolveState init{};
    init.tol = tol;
    init.maxIter = maxIter;
    init.nComp = nComp;
    const int n = dm_.nC;
    if (devLoop_)
    {
        k_state_reset<<<1, 32, 0, stream_>>>(st_, tol, maxIter, nComp, 0);
        auto dloop = [&](auto Wc, auto NCc) {
            constexpr int W = decltype(Wc)::value;
            constexpr int NC = decltype(NCc)::value;
            k_bi_init<W, NC><<<GS_, TPB, 0, stream_>>>(A, vals, diag, bInvD_, b, x, br_, br0_, bp_, bv_, partials_, st_);
            constexpr int CH = 4;
            captureWhile((maxIter + CH - 1) / CH + 1, [&] {
                for (int k = 0; k < CH; ++k)
                {
                    k_bi_p<NC><<<GS_, TPB, 0, stream_>>>(n, bInvD_, br_, bp_, bv_, bz_, st_);
                    k_bi_spmv1<W, NC><<<GS_, TPB, 0, stream_>>>(A, vals, bz_, bv_, br0_, partials_, st_);
                    k_bi_spmv2<W, NC><<<GS_, TPB, 0, stream_>>>(A, vals, bInvD_, br_, bv_, bt_, partials_, st_);
                    k_bi_x<NC><<<GS_, TPB, 0, stream_>>>(n, bInvD_, x, bz_, bv_, bt_, br_, br0_, partials_, st_);
                }
                launchCheck("bicg_iter", 0);
            });
        };
        dispatchW(maxW_, [&](auto Wc) {
            if (nComp == 3) dloop(Wc, std::integral_constant<int, 3>{});
            else dloop(Wc, std::integral_constant<int, 1>{});
        });
        if (tally_) k_state_tally<<<1, 32, 0, stream_>>>(st_, nComp, tally_);
        launchCheck("bicg_tally");
        for (int q = 0; q < nComp; ++q) reps[q] = cfg_solver_report{};
        return;
    }
    CFG_CUDA(cudaMemcpyAsync(st_, &init, sizeof(SolveState), cudaMemcpyHostToDevice, stream_));
    auto loop = [&](auto Wc, auto NCc) {
        constexpr int W = decltype(Wc)::value;
        constexpr int NC = decltype(NCc)::value;
        k_bi_init<W, NC><<<GS_, TPB, 0, stream_>>>(A, vals, diag, bInvD_, b, x, br_, br0_, bp_, bv_, partials_, st_);
        launchCheck("bicg_init");
        int itBefore = 0, lastChunk = 0, activeBefore = NC;
        auto itMax = [&] {
            int m = 0;
            for (int q = 0; q < NC; ++q) m = std::max(m, stHost_->it[q]);
            return m;
        };
        for (int launched = 0, chunk = 4;;)
        {
            CFG_CUDA(cudaMemcpyAsync(stHost_, st_, sizeof(SolveState), cudaMemcpyDeviceToHost, stream_));
            CFG_CUDA(cudaStreamSynchronize(stream_));
            if (lastChunk > 0)
            {
                static const int slots[4] = {KS_BI_P, KS_BI_SPMV1, KS_BI_SPMV2, KS_BI_X};
                harvest(std::min(lastChunk, std::max(0, itMax() - itBefore)), slots, 4, activeBefore);
            }
            itBefore = itMax();
            activeBefore = 0;
            for (int q = 0; q < NC; ++q) activeBefore += stHost_->done[q] ? 0 : 1;
            if (stHost_->allDone || launched >= maxIter) break;
            // timed launches go one iteration at a time, so each is charged
            // with the components that were still iterating
            const int m = ktime_ ? 1 : std::min(chunk, maxIter - launched);
            launchChunk(ptrKey("bicg", {vals, diag, x.c[0], x.c[1], x.c[2]}, W * 8 + NC), m, [&](int k) {
                tmark(k, 0);
                k_bi_p<NC><<<GS_, TPB, 0, stream_>>>(n, bInvD_, br_, bp_, bv_, bz_, st_);
                tmark(k, 1);
                k_bi_spmv1<W, NC><<<GS_, TPB, 0, stream_>>>(A, vals, bz_, bv_, br0_, partials_, st_);
                tmark(k, 2);
                k_bi_spmv2<W, NC><<<GS_, TPB, 0, stream_>>>(A, vals, bInvD_, br_, bv_, bt_, partials_, st_);
                tmark(k, 3);
                k_bi_x<NC><<<GS_, TPB, 0, stream_>>>(n, bInvD_, x, bz_, bv_, bt_, br_, br0_, partials_, st_);
                tmark(k, 4);
                launchCheck("bicg_iter", 0);
            });
            launches_ += 4 * m;
            launched += m;
            lastChunk = m;
            chunk = std::min(chunk * 2, 32);
        }
    };
    dispatchW(maxW_, [&](auto Wc) {
        if (nComp == 3) loop(Wc, std::integral_constant<int, 3>{});
        else loop(Wc, std::integral_constant<int, 1>{});
    });
    for (int q = 0; q < nComp; ++q)
    {
        reps[q].iterations = stHost_->it[q];
        reps[q].converged = stHost_->conv[q];
        reps[q].initial_residual = stHost_->init[q];
        reps[q].final_residual = stHost_->fin[q];
    }
}

/// The momentum BiCGStab of runBiCG3 with the FP32 AMG V-cycle of the
/// momentum matrix as right preconditioner (z = M p, s^ = M s in place of
/// the reference's D^-1 scaling, Matrix.cpp:262-300); the three components
/// iterate in lockstep, each with its own scalars and stopping test, and a
/// V-cycle serves all components still iterating.  The hierarchy's values
/// must be this matrix's (amgValues).  Host-polled chunks of iterations,
/// each chunk a CUDA graph after its first launch.
void Ctx::runBiCGAmg(const double* vals, const double* diag, V3P b, V3P x, double tol, int maxIter,
                     cfg_solver_report* reps)
{
    const DMat A{dm_.nC, dm_.mStart, dm_.mCol};
    SolveState init{};
    init.tol = tol;
    init.maxIter = maxIter;
    init.nComp = 3;
    const int n = dm_.nC;
    const int* done = reinterpret_cast<const int*>(reinterpret_cast<const char*>(st_) + offsetof(SolveState, done));
    const int vk = amgCycleKernels(kAmgMomentum);
    CFG_CUDA(cudaMemcpyAsync(st_, &init, sizeof(SolveState), cudaMemcpyHostToDevice, stream_));
    auto loop = [&](auto Wc) {
        constexpr int W = decltype(Wc)::value;
        k_bi_init<W, 3><<<GS_, TPB, 0, stream_>>>(A, vals, diag, bInvD_, b, x, br_, br0_, bp_, bv_, partials_, st_);
        launchCheck("bicga_init");
        int itBefore = 0, lastChunk = 0, activeBefore = 3;
        auto itMax = [&] {
            int m = 0;
            for (int q = 0; q < 3; ++q) m = std::max(m, stHost_->it[q]);
            return m;
        };
        for (int launched = 0, chunk = 2;;)
        {
            CFG_CUDA(cudaMemcpyAsync(stHost_, st_, sizeof(SolveState), cudaMemcpyDeviceToHost, stream_));
            CFG_CUDA(cudaStreamSynchronize(stream_));
            if (lastChunk > 0)
            {
                static const int slots[11] = {KS_BIA_P,     KS_AMGV_PRE0, KS_AMGV_COARSE, KS_AMGV_POST0,
                                              KS_BIA_SPMV1, KS_BIA_S,     KS_AMGV_PRE0,   KS_AMGV_COARSE,
                                              KS_AMGV_POST0, KS_BIA_SPMV2, KS_BIA_X};
                harvest(std::min(lastChunk, std::max(0, itMax() - itBefore)), slots, 11, activeBefore);
            }
            itBefore = itMax();
            activeBefore = 0;
            for (int q = 0; q < 3; ++q) activeBefore += stHost_->done[q] ? 0 : 1;
            if (stHost_->allDone || launched >= maxIter) break;
            const int m = ktime_ ? 1 : std::min(chunk, maxIter - launched);
            launchChunk(ptrKey("bicga", {vals, diag, x.c[0], x.c[1], x.c[2]}, W), m, [&](int k) {
                const std::function<void(int)> markZ = [&](int j) { tmark(k, 2 + j); };
                const std::function<void(int)> markS = [&](int j) { tmark(k, 7 + j); };
                tmark(k, 0);
                launchK(pdl_, k_bia_p<3>, GS_, TPB, 0, stream_, n, br_, bp_, bv_, st_);
                tmark(k, 1);
                amgCycle3(kAmgMomentum, cv(bp_), bz_, done, kAmgScaleMomentum, ktime_ ? markZ : std::function<void(int)>{});
                tmark(k, 4);
                launchK(pdl_, k_bi_spmv1<W, 3>, GS_, TPB, 0, stream_, A, vals, bz_, bv_, br0_, partials_, st_);
                tmark(k, 5);
                launchK(pdl_, k_bia_s<3>, GS_, TPB, 0, stream_, n, br_, bv_, bs_, st_);
                tmark(k, 6);
                amgCycle3(kAmgMomentum, cv(bs_), bsh_, done, kAmgScaleMomentum, ktime_ ? markS : std::function<void(int)>{});
                tmark(k, 9);
                launchK(pdl_, k_bia_spmv2<W, 3>, GS_, TPB, 0, stream_, A, vals, bsh_, bs_, bt_, partials_, st_);
                tmark(k, 10);
                launchK(pdl_, k_bia_x<3>, GS_, TPB, 0, stream_, n, x, bz_, bs_, bsh_, bt_, br_, br0_, partials_, st_);
                tmark(k, 11);
                launchCheck("bicga_iter", 0);
            });
            launches_ += static_cast<int64_t>(m) * (5 + 2 * vk);
            launched += m;
            lastChunk = m;
            chunk = std::min(chunk * 2, 16);
        }
    };
    dispatchW(maxW_, [&](auto Wc) { loop(Wc); });
    for (int q = 0; q < 3; ++q)
    {
        reps[q].iterations = stHost_->it[q];
        reps[q].converged = stHost_->conv[q];
        reps[q].initial_residual = stHost_->init[q];
        reps[q].final_residual = stHost_->fin[q];
    }
}

/// Blocks for a grid-stride row loop over `rows` rows.
int Ctx::rowGrid(int rows) const
{
    if (rowBlocksPerSM_ <= 0) return std::max(1, (rows + RPT * TPB - 1) / (RPT * TPB));
    return std::max(1, std::min((rows + TPB - 1) / TPB, sms_ * rowBlocksPerSM_));
}

template <class T>
void Ctx::dicSetupT(DDicT<T>& D, const double* vals, const T* diag)
{
    k_dic_gather<T><<<std::max(1, std::min((nLo_ + TPB - 1) / TPB, 4096)), TPB, 0, stream_>>>(nLo_, D.lSrc, vals, D.lVal);
    k_dic_gather<T><<<std::max(1, std::min((nUp_ + TPB - 1) / TPB, 4096)), TPB, 0, stream_>>>(nUp_, D.uSrc, vals, D.uVal);
    launchCheck("dic_gather");
    dispatchW(maxW_, [&](auto Wc) {
        constexpr int W = decltype(Wc)::value;
        for (const DicPhase& ph : dicPhase_)
        {
            k_dic_factor<W, T><<<rowGrid(ph.cnt), TPB, 0, stream_>>>(D, ph, diag);
            launchCheck("dic_factor");
        }
    });
}

template <class T>
void Ctx::dicApplyT(const DDicT<T>& D, const T* r, T* z)
{
    const int C = D.nColours;
    dispatchW(maxW_, [&](auto Wc) {
        constexpr int W = decltype(Wc)::value;
        for (int c = 0; c < C; ++c)
            k_dic_fwd<W, T><<<rowGrid(dicPhase_[c].cnt), TPB, 0, stream_>>>(D, dicPhase_[c], r, z, c == C - 1,
                                                                            partials_, st_);
        if (C == 1)
        {
            // no backward phase: a one-block final reduction of the forward partials
            const DicPhase none{0, 0, 0, dicPartials_ - 1};
            k_dic_bwd<W, T><<<1, TPB, 0, stream_>>>(D, none, r, z, 1, dicPartials_, partials_, st_);
        }
        for (int c = C - 2; c >= 0; --c)
            k_dic_bwd<W, T><<<rowGrid(dicPhase_[c].cnt), TPB, 0, stream_>>>(
                D, dicPhase_[c], r, z, c == 0, c == 0 ? dicPartials_ - 1 : 0, partials_, st_);
    });
    launchCheck("dic_apply", C == 1 ? 2 : 2 * C - 1);
}

void Ctx::dicSetup(const double* vals, const double* diag) { dicSetupT<double>(dic_, vals, diag); }
void Ctx::dicApply(const double* r, double* z) { dicApplyT<double>(dic_, r, z); }

/// PCG of Matrix.cpp:153-222 with z = M^-1 r from the multicolour DIC, on
/// values and vectors of type T; the DIC must be set up for these values.
template <class T>
void Ctx::dicCGT(const DDicT<T>& D, const T* vals, const T* diag, const T* b, T* x, T* r, T* p, T* Ap, T* z,
                 double tol, int maxIter, int normType, cfg_solver_report* rep)
{
    const DMat A{dm_.nC, dm_.mStart, dm_.mCol};
    SolveState init{};
    init.tol = tol;
    init.maxIter = maxIter;
    init.nComp = 1;
    init.normType = normType;
    if (devLoop_)
    {
        k_state_reset<<<1, 32, 0, stream_>>>(st_, tol, maxIter, 1, normType);
        dispatchW(maxW_, [&](auto Wc) {
            constexpr int W = decltype(Wc)::value;
            k_cg_init<W, T><<<GS_, TPB, 0, stream_>>>(A, vals, diag, b, x, r, p, partials_, st_);
            dicApplyT<T>(D, r, z);
            k_cg_pz<T><<<GS_, TPB, 0, stream_>>>(dm_.nC, z, p, st_);
            constexpr int CH = 8;
            captureWhile((maxIter + CH - 1) / CH + 1, [&] {
                for (int k = 0; k < CH; ++k)
                {
                    k_cg_spmv<W, T><<<GS_, TPB, 0, stream_>>>(A, vals, p, Ap, partials_, st_);
                    k_cg_update_nz<T><<<GS_, TPB, 0, stream_>>>(dm_.nC, p, Ap, x, r, partials_, st_);
                    dicApplyT<T>(D, r, z);
                    k_cg_pz<T><<<GS_, TPB, 0, stream_>>>(dm_.nC, z, p, st_);
                }
                launchCheck("dic_cg_iter", 0);
            });
        });
        if (tally_) k_state_tally<<<1, 32, 0, stream_>>>(st_, 1, tally_);
        launchCheck("dic_cg_tally");
        *rep = cfg_solver_report{};
        return;
    }
    CFG_CUDA(cudaMemcpyAsync(st_, &init, sizeof(SolveState), cudaMemcpyHostToDevice, stream_));
    dispatchW(maxW_, [&](auto Wc) {
        constexpr int W = decltype(Wc)::value;
        k_cg_init<W, T><<<GS_, TPB, 0, stream_>>>(A, vals, diag, b, x, r, p, partials_, st_);
        launchCheck("cg_init");
        dicApplyT<T>(D, r, z);
        k_cg_pz<T><<<GS_, TPB, 0, stream_>>>(dm_.nC, z, p, st_);
        launchCheck("cg_pz");
        int launched = 0;
        int chunk = 8;
        int itBefore = 0, lastChunk = 0;
        for (;;)
        {
            CFG_CUDA(cudaMemcpyAsync(stHost_, st_, sizeof(SolveState), cudaMemcpyDeviceToHost, stream_));
            CFG_CUDA(cudaStreamSynchronize(stream_));
            if (lastChunk > 0)
            {
                static const int slots[4] = {KS_CG_SPMV, KS_CG_UPDATE, KS_DIC_APPLY, KS_CG_P};
                harvest(std::min(lastChunk, std::max(0, stHost_->it[0] - itBefore)), slots, 4);
            }
            itBefore = stHost_->it[0];
            if (stHost_->allDone || launched >= maxIter) break;
            const int n = std::min(chunk, maxIter - launched);
            lastChunk = n;
            launchChunk(ptrKey("diccg", {vals, diag, x, r, p, Ap, z, D.lVal}, W), n, [&](int k) {
                tmark(k, 0);
                k_cg_spmv<W, T><<<GS_, TPB, 0, stream_>>>(A, vals, p, Ap, partials_, st_);
                tmark(k, 1);
                k_cg_update_nz<T><<<GS_, TPB, 0, stream_>>>(dm_.nC, p, Ap, x, r, partials_, st_);
                tmark(k, 2);
                dicApplyT<T>(D, r, z);
                tmark(k, 3);
                k_cg_pz<T><<<GS_, TPB, 0, stream_>>>(dm_.nC, z, p, st_);
                tmark(k, 4);
                launchCheck("dic_cg_iter", 0);
            });
            launches_ += (3 + (D.nColours == 1 ? 2 : 2 * D.nColours - 1)) * static_cast<long>(n);
            launched += n;
            chunk = std::min(chunk * 2, 64);
        }
    });
    rep->iterations = stHost_->it[0];
    rep->converged = stHost_->conv[0];
    rep->initial_residual = stHost_->init[0];
    rep->final_residual = stHost_->conv[0] && stHost_->it[0] == 0 ? stHost_->init[0] : stHost_->fin[0];
}

void Ctx::runDICCG(const double* vals, const double* diag, const double* b, double* x, double tol, int maxIter,
                   cfg_solver_report* rep, int normType)
{
    dicSetup(vals, diag);
    dicCGT<double>(dic_, vals, diag, b, x, cr_, cp_, cAp_, cz_, tol, maxIter, normType, rep);
}

/// fvMatrix::solve for the momentum equation (fvMatrix.cpp:73-129): x from
/// zero, nonOrth+1 passes when the laplacian is corrected, each restoring the
/// base rhs and adding the corrector evaluated on the current x.
void Ctx::solveMomentum(int nonOrth, int gradScheme, double tol, int maxIter, int64_t& inner)
{
    const int n = dm_.nC;
    for (int q = 0; q < 3; ++q) CFG_CUDA(cudaMemsetAsync(ux_.c[q], 0, n * sizeof(double), stream_));
    const bool corr = schemes_.laplacian_corrected != 0;
    const int passes = corr ? std::max(1, nonOrth + 1) : 1;
    const BcTab ub{{uc_[0], uc_[1], uc_[2]}, {uk_[0], uk_[1], uk_[2]}};
    for (int pass = 0; pass < passes; ++pass)
    {
        if (corr)
        {
            const double* xs[3] = {ux_.c[0], ux_.c[1], ux_.c[2]};
            V3P g[3] = {gA_, gB_, Hf_};  // Hf_ is free until the solve ends
            // gradCells with 3 components uses bs_/bsh_/bt_ as scratch
            gradCells(xs, 3, ub, gradScheme, false, g);
            k_corrector<3><<<G_, TPB, 0, stream_>>>(dm_, gU_, CGrad3{{cv(g[0]), cv(g[1]), cv(g[2])}},
                                                   cv(uBase_), uRhs_);
            launchCheck("corrector_U");
        }
        else
        {
            for (int q = 0; q < 3; ++q)
                CFG_CUDA(cudaMemcpyAsync(uRhs_.c[q], uBase_.c[q], n * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
        }
        cfg_solver_report reps[3];
        if (uPrecond_ == CFG_PRECOND_AMG)
        {
            if (pass == 0)
            {
                // the FP32 AMG hierarchy follows this outer iteration's
                // momentum matrix (the pressure solve refreshes its own)
                const int nE = nSlicesEntries_;
                if (!uVal32_) uVal32_ = alloc<float>(static_cast<size_t>(nE));
                k_to_float<<<std::max(1, std::min((nE + TPB - 1) / TPB, 8192)), TPB, 0, stream_>>>(nE, mVal_, uVal32_);
                launchCheck("amg_u_float");
                amgValues(kAmgMomentum, mVal_, uDiag_, uVal32_);
                amgVectors3(kAmgMomentum);
            }
            runBiCGAmg(mVal_, uDiag_, uRhs_, ux_, tol, maxIter, reps);
        }
        else runBiCG3(mVal_, uDiag_, uRhs_, ux_, 3, tol, maxIter, reps);
        for (int q = 0; q < 3; ++q) inner += reps[q].iterations;
    }
}

void Ctx::setKernelTiming(bool on)
{
    if (on && kev_.empty())
    {
        kev_.resize(kEvPerIter * 64);
        for (auto& e : kev_) CFG_CUDA(cudaEventCreate(&e));
    }
    ktime_ = on;
    for (auto& r : kstat) r[0] = r[1] = 0.0;
    for (auto& c : kcomp) c = 0.0;
}

/// Event j of iteration k of the chunk being enqueued (kernel timing on).
void Ctx::tmark(int k, int j)
{
    if (ktime_) CFG_CUDA(cudaEventRecord(kev_[kEvPerIter * k + j], stream_));
}

/// Adds the first `ran` iterations of the last timed chunk to kstat: the
/// interval between events j and j+1 of an iteration is kernel slots[j];
/// `active` components were iterating in each.
void Ctx::harvest(int ran, const int* slots, int nSlots, int active)
{
    if (!ktime_) return;
    for (int k = 0; k < ran; ++k)
        for (int j = 0; j < nSlots; ++j)
        {
            float ms = 0;
            CFG_CUDA(cudaEventElapsedTime(&ms, kev_[kEvPerIter * k + j], kev_[kEvPerIter * k + j + 1]));
            kstat[slots[j]][0] += 1;
            kstat[slots[j]][1] += ms;
            kcomp[slots[j]] += active;
        }
}

void Ctx::setNu(double nu)
{
    if (nu == lastNu_) return;
    // harmonicFaceGamma of a uniform cell viscosity (laplacianScheme.cpp:146-171)
    const Mesh& M = mesh_;
    const int64_t nF = M.nFaces(), nI = M.nInternal();
    std::vector<double> g(static_cast<size_t>(nF));
    for (int64_t f = 0; f < nF; ++f)
    {
        if (f < nI)
        {
            const double gp = nu, gn = nu;
            const Vec& cP = M.C[M.owner[f]];
            const Vec& cN = M.C[M.neighbour[f]];
            const Vec& cf = M.Cf[f];
            const Vec a{cf.x - cP.x, cf.y - cP.y, cf.z - cP.z}, b{cN.x - cf.x, cN.y - cf.y, cN.z - cf.z};
            const double dP = std::sqrt(hdot(a, a)), dN = std::sqrt(hdot(b, b));
            const double tot = dP + dN;
            g[f] = (tot > 0 && gp > 0 && gn > 0) ? tot * gp * gn / (dN * gp + dP * gn) : 0.5 * (gp + gn);
        }
        else
        {
            g[f] = nu;
        }
    }
    CFG_CUDA(cudaMemcpyAsync(gU_, g.data(), nF * sizeof(double), cudaMemcpyHostToDevice, stream_));
    CFG_CUDA(cudaStreamSynchronize(stream_));
    lastNu_ = nu;
}

void Ctx::checkMomentumBcs() const
{
    // the reference builds the momentum matrix with the BC linearisation of
    // every component; symmetry / wall velocity conditions give components
    // different diagonals, which solveIncompressibleSimple rejects
    // (simpleSolver.cpp:123-138), and an unknown type is fatal at the first
    // linearisation (volFields.cpp:279-282)
    for (size_t pi = 0; pi < mesh_.patches.size(); ++pi)
    {
        if (mesh_.patches[pi].size == 0) continue;
        const int t = uType_[pi];
        if (t == CFG_BC_SYMMETRY || t == CFG_BC_WALL)
            fail(CFG_ENUMERIC, "SIMPLE: momentum diagonal differs between components");
        if (t == CFG_BC_EMPTY) fail(CFG_ESETUP, "volVectorField: unknown patch bc type 'empty'");
        const int pt = pType_[pi];
        if (pt == CFG_BC_WALL || pt == CFG_BC_EMPTY) fail(CFG_ESETUP, "volScalarField: unknown patch bc type");
    }
}

void Ctx::solvePressure(int nonOrth, int gradScheme, double tol, int maxIter, int precond, int64_t& inner,
                        const double* x0)
{
    const int n = dm_.nC;
    if (x0) CFG_CUDA(cudaMemcpyAsync(px_, x0, n * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    else CFG_CUDA(cudaMemsetAsync(px_, 0, n * sizeof(double), stream_));
    const bool corr = schemes_.laplacian_corrected != 0;
    const int passes = corr ? std::max(1, nonOrth + 1) : 1;
    const BcTab pb{{pc_, pc_, pc_}, {pk_, pk_, pk_}};
    for (int pass = 0; pass < passes; ++pass)
    {
        if (corr)
        {
            const double* xs[1] = {px_};
            V3P g[1] = {gA_};
            gradCells(xs, 1, pb, gradScheme, false, g);
            k_corrector<1><<<G_, TPB, 0, stream_>>>(dm_, rAUf_, CGrad3{{cv(gA_)}}, CV3P{{pBase_, pBase_, pBase_}},
                                                   V3P{{pRhs_, pRhs_, pRhs_}});
            launchCheck("corrector_p");
        }
        else
        {
            CFG_CUDA(cudaMemcpyAsync(pRhs_, pBase_, n * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
        }
        // a training pair of the learned preconditioner: the residual this
        // solve starts from, and (below) the correction it converges to
        const bool collect = collectOn_ && pass == 0 && static_cast<int>(collected_.size()) < collectMax_;
        std::vector<double> x0;
        if (collect)
        {
            std::vector<double> r(static_cast<size_t>(n));
            mpnnResidualHost(pVal_d_, pRhs_, px_, r.data());
            collected_.push_back(std::move(r));
            x0.resize(static_cast<size_t>(n));
            fromDevCells(x0.data(), px_, 1, 0);
        }
        if (pass == 0 && (precond == CFG_PRECOND_MPNN || precond == CFG_PRECOND_AMG_MPNN))
        {
            // the network's initial guess from the residual of the given one
            if (!mpnn_) fail(CFG_ESETUP, "pressure: the learned preconditioner needs cfg_mpnn_create");
            mpnnGuess(pVal_d_, pDiag_, pRhs_, px_);
        }
        cfg_solver_report rep;
        if (precond == CFG_PRECOND_DIC) runDICCG(pVal_d_, pDiag_, pRhs_, px_, tol, maxIter, &rep);
        else if (precond == CFG_PRECOND_MPNN)
        {
            if (!mpnn_) fail(CFG_ESETUP, "pressure: the learned preconditioner needs cfg_mpnn_create");
            int64_t o[3];
            mpnnFcg(pVal_d_, pDiag_, pRhs_, px_, tol, maxIter, 25, o, 0);
            rep.iterations = static_cast<int32_t>(o[0] + o[1]);
            lastFallbackIters += o[1];
        }
        else if (precond == CFG_PRECOND_AMG || precond == CFG_PRECOND_AMG_MPNN)
        {
            // the FP32 AMG hierarchy follows this outer iteration's matrix
            if (pass == 0)
            {
                const int nE = nSlicesEntries_;
                if (!pVal32_) pVal32_ = alloc<float>(static_cast<size_t>(nE));
                k_to_float<<<std::max(1, std::min((nE + TPB - 1) / TPB, 8192)), TPB, 0, stream_>>>(nE, pVal_d_, pVal32_);
                launchCheck("amg_float");
                amgValues(kAmgPressure, pVal_d_, pDiag_, pVal32_);
                amgFresh_ = false;  // the Poisson system, if any, must refresh its own
            }
            amgFcg(pVal_d_, pRhs_, px_, tol, maxIter, 0, &rep);
        }
        else if (precond == CFG_PRECOND_IR32)
        {
            if (devLoop_) fail(CFG_EINVAL, "pressure: the mixed-precision refinement is host driven");
            if (pass == 0)
            {
                // the FP32 copy of this outer iteration's matrix and its FP32 DIC factor
                ensureMixed();
                const int nE = nSlicesEntries_;
                k_to_float<<<std::max(1, std::min((nE + TPB - 1) / TPB, 8192)), TPB, 0, stream_>>>(nE, pVal_d_, pVal32_);
                k_to_float<<<G_, TPB, 0, stream_>>>(n, pDiag_, pDiag32_);
                launchCheck("ir32_float", 2);
                dicSetupT<float>(dic32_, pVal_d_, pDiag32_);
                amgFresh_ = false;  // pVal32_ now holds this matrix
            }
            runIR32(pVal_d_, pDiag_, pRhs_, px_, tol, maxIter, 1e-4, &rep);
        }
        else runCG(pVal_d_, pDiag_, pRhs_, px_, tol, maxIter, &rep);
        inner += rep.iterations;
        if (collect)
        {
            std::vector<double> x1(static_cast<size_t>(n));
            fromDevCells(x1.data(), px_, 1, 0);
            for (size_t i = 0; i < x1.size(); ++i) x1[i] -= x0[i];
            collectedT_.push_back(std::move(x1));
        }
    }
}

/// A host cell array in the original numbering (element c at
/// host[c * stride + off]) copied into device slot order.
void Ctx::toDevCells(double* dev, const double* host, int stride, int off)
{
    const int nC = dm_.nC;
    if (identityOrder_ && stride == 1)
    {
        CFG_CUDA(cudaMemcpyAsync(dev, host + off, nC * sizeof(double), cudaMemcpyHostToDevice, stream_));
        CFG_CUDA(cudaStreamSynchronize(stream_));
        return;
    }
    hostTmp_.resize(static_cast<size_t>(nC));
    for (int i = 0; i < nC; ++i) hostTmp_[i] = host[static_cast<size_t>(perm_[i]) * stride + off];
    CFG_CUDA(cudaMemcpyAsync(dev, hostTmp_.data(), nC * sizeof(double), cudaMemcpyHostToDevice, stream_));
    CFG_CUDA(cudaStreamSynchronize(stream_));
}

/// The inverse of toDevCells.
void Ctx::fromDevCells(double* host, const double* dev, int stride, int off)
{
    const int nC = dm_.nC;
    if (identityOrder_ && stride == 1)
    {
        CFG_CUDA(cudaMemcpyAsync(host + off, dev, nC * sizeof(double), cudaMemcpyDeviceToHost, stream_));
        CFG_CUDA(cudaStreamSynchronize(stream_));
        return;
    }
    hostTmp_.resize(static_cast<size_t>(nC));
    CFG_CUDA(cudaMemcpyAsync(hostTmp_.data(), dev, nC * sizeof(double), cudaMemcpyDeviceToHost, stream_));
    CFG_CUDA(cudaStreamSynchronize(stream_));
    for (int i = 0; i < nC; ++i) host[static_cast<size_t>(perm_[i]) * stride + off] = hostTmp_[i];
}

int Ctx::deviceCell(int64_t c) const { return c < 0 ? -1 : inv_[static_cast<size_t>(c)]; }

/// dev[q][i] = aos[perm[i] nc + q]: interleaved original-order cell values to
/// device-numbered component arrays (perm null: the identity)
__global__ void k_cells_scatter(int n, int nc, const int* __restrict__ perm, const double* __restrict__ aos,
                                double* d0, double* d1, double* d2)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const size_t o = static_cast<size_t>(perm ? perm[i] : i) * nc;
        d0[i] = aos[o];
        if (nc == 3)
        {
            d1[i] = aos[o + 1];
            d2[i] = aos[o + 2];
        }
    }
}

/// The inverse of k_cells_scatter.
__global__ void k_cells_gather(int n, int nc, const int* __restrict__ perm, double* __restrict__ aos,
                               const double* s0, const double* s1, const double* s2)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const size_t o = static_cast<size_t>(perm ? perm[i] : i) * nc;
        aos[o] = s0[i];
        if (nc == 3)
        {
            aos[o + 1] = s1[i];
            aos[o + 2] = s2[i];
        }
    }
}

void Ctx::cellsToDev(double* const* dev, int nc, const double* host)
{
    const int nC = dm_.nC;
    if (nc == 1 && identityOrder_)
    {
        CFG_CUDA(cudaMemcpyAsync(dev[0], host, nC * sizeof(double), cudaMemcpyHostToDevice, stream_));
        return;
    }
    CFG_CUDA(cudaMemcpyAsync(ioStage_, host, static_cast<size_t>(nC) * nc * sizeof(double), cudaMemcpyHostToDevice,
                             stream_));
    k_cells_scatter<<<GS_, TPB, 0, stream_>>>(nC, nc, dPerm_, ioStage_, dev[0], nc == 3 ? dev[1] : nullptr,
                                              nc == 3 ? dev[2] : nullptr);
    launchCheck("cells_scatter");
}

void Ctx::cellsFromDev(double* host, const double* const* dev, int nc)
{
    const int nC = dm_.nC;
    if (nc == 1 && identityOrder_)
    {
        CFG_CUDA(cudaMemcpyAsync(host, dev[0], nC * sizeof(double), cudaMemcpyDeviceToHost, stream_));
        return;
    }
    k_cells_gather<<<GS_, TPB, 0, stream_>>>(nC, nc, dPerm_, ioStage_, dev[0], nc == 3 ? dev[1] : nullptr,
                                             nc == 3 ? dev[2] : nullptr);
    launchCheck("cells_gather");
    CFG_CUDA(cudaMemcpyAsync(host, ioStage_, static_cast<size_t>(nC) * nc * sizeof(double), cudaMemcpyDeviceToHost,
                             stream_));
}

/// Fields in: one host-to-device copy per field (from the caller's buffers,
/// pinned or not), then the device transposes and renumbers.  The stage is
/// shared, so each field's scatter runs before the next copy overwrites it
/// (both are ordered on the context's stream).
void Ctx::upload(const double* U, const double* p, const double* phi)
{
    const int nF = dm_.nF;
    if (U)
    {
        double* const d[3] = {U_.c[0], U_.c[1], U_.c[2]};
        cellsToDev(d, 3, U);
    }
    if (p)
    {
        double* const d[1] = {p_};
        cellsToDev(d, 1, p);
    }
    if (phi) CFG_CUDA(cudaMemcpyAsync(phi_, phi, nF * sizeof(double), cudaMemcpyHostToDevice, stream_));
    CFG_CUDA(cudaStreamSynchronize(stream_));
}

void Ctx::download(double* U, double* p, double* phi)
{
    const int nF = dm_.nF;
    if (U)
    {
        const double* const s[3] = {U_.c[0], U_.c[1], U_.c[2]};
        cellsFromDev(U, s, 3);
    }
    if (p)
    {
        const double* const s[1] = {p_};
        cellsFromDev(p, s, 1);
    }
    if (phi) CFG_CUDA(cudaMemcpyAsync(phi, phi_, nF * sizeof(double), cudaMemcpyDeviceToHost, stream_));
    CFG_CUDA(cudaStreamSynchronize(stream_));
}

void Ctx::initFlux(const double* u0)
{
    refreshBc();
    const BcTab ub{{uc_[0], uc_[1], uc_[2]}, {uk_[0], uk_[1], uk_[2]}};
    if (u0)
    {
        std::vector<double> t(static_cast<size_t>(dm_.nC));
        for (int q = 0; q < 3; ++q)
        {
            std::fill(t.begin(), t.end(), u0[q]);
            CFG_CUDA(cudaMemcpyAsync(U_.c[q], t.data(), dm_.nC * sizeof(double), cudaMemcpyHostToDevice, stream_));
            CFG_CUDA(cudaStreamSynchronize(stream_));
        }
    }
    // correctBoundaryFlux(U) (+ updatePhiInternal first when seeded; the
    // internal flux is untouched otherwise, as in simpleFoamApp.cpp:94-95)
    if (u0)
    {
        k_flux_internal<<<GF_, TPB, 0, stream_>>>(dm_, cv(U_), phi_);
        launchCheck("flux_internal");
    }
    // boundary faces: the flux kernel into scratch, then only the boundary
    // part copied over, so internal faces keep their values
    const int nF = dm_.nF, nI = dm_.nI;
    k_flux<<<GF_, TPB, 0, stream_>>>(dm_, cv(U_), ub, dEmptyFace_, fScratch_);
    launchCheck("flux");
    if (nF > nI)
        CFG_CUDA(cudaMemcpyAsync(phi_ + nI, fScratch_ + nI, (nF - nI) * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    CFG_CUDA(cudaStreamSynchronize(stream_));
}

/// The host side of an outer iteration's set-up: the boundary tables, the
/// momentum boundary checks and the laminar face viscosity.
void Ctx::prepareIterate(const cfg_simple_controls& ctl)
{
    CFG_CUDA(cudaSetDevice(device_));
    refreshBc();
    checkMomentumBcs();
    if (!turb_) setNu(ctl.nu);  // with a RANS model the model's nu + nut is the diffusivity
    if (ctl.p_ref_cell >= dm_.nC) fail(CFG_EINVAL, "p_ref_cell beyond the last cell");
    if (ctl.u_precond != CFG_PRECOND_JACOBI && ctl.u_precond != CFG_PRECOND_AMG)
        fail(CFG_EINVAL, "SIMPLE: u_precond must be CFG_PRECOND_JACOBI or CFG_PRECOND_AMG");
    if (ctl.u_precond == CFG_PRECOND_AMG && devLoop_)
        fail(CFG_EINVAL, "SIMPLE: the AMG momentum preconditioner is host driven (no device-side loops)");
    // the time term (simpleSolver.cpp:75-97): dt and the old velocity together
    if (ctl.dt > 0 || ctl.u_time_old != 0)
    {
        if (!(ctl.dt > 0)) fail(CFG_EINVAL, "SIMPLE: an old velocity was supplied with no time step");
        if (ctl.u_time_old != 1 && ctl.u_time_old != 2)
            fail(CFG_EINVAL, "SIMPLE: a time step was supplied with no velocity at the previous time level");
        if (ctl.u_time_old == 2 && !oldUploaded_)
            fail(CFG_EINVAL, "SIMPLE: u_time_old 2 needs cfg_fields_upload_old first");
        if (!uOld_.c[0])
            for (int q = 0; q < 3; ++q) uOld_.c[q] = alloc<double>(dm_.nC);
        if (ctl.u_time_old == 1)
            for (int q = 0; q < 3; ++q)
                CFG_CUDA(cudaMemcpyAsync(uOld_.c[q], U_.c[q], dm_.nC * sizeof(double), cudaMemcpyDeviceToDevice,
                                         stream_));
    }
}

void Ctx::uploadOld(const double* U)
{
    CFG_CUDA(cudaSetDevice(device_));
    if (!uOld_.c[0])
        for (int q = 0; q < 3; ++q) uOld_.c[q] = alloc<double>(dm_.nC);
    double* const dev[3] = {uOld_.c[0], uOld_.c[1], uOld_.c[2]};
    cellsToDev(dev, 3, U);
    CFG_CUDA(cudaStreamSynchronize(stream_));
    oldUploaded_ = true;
}

/// Enqueues one SIMPLE outer iteration (simpleSolver.cpp:52-357) on stream_,
/// ending with the copy of its scalars to scalHost_.  With devLoop_ the
/// linear solvers iterate in device-side loops and nothing here waits for
/// the device, so the whole iteration can be captured into a CUDA graph; the
/// inner iteration counts then arrive in the S_*INNER slots.  Otherwise the
/// solvers poll their state from the host and add their counts to `uInner`
/// and `pInner`.
void Ctx::enqueueOuter(const cfg_simple_controls& ctl, int64_t& uInner, int64_t& pInner)
{
    const int nC = dm_.nC;
    const int gs = schemes_.grad;
    const double alpha = schemes_.div == CFG_DIV_BLEND ? schemes_.blend_coeff : (schemes_.div == CFG_DIV_LINEAR ? 1.0 : 0.0);
    const BcTab ub{{uc_[0], uc_[1], uc_[2]}, {uk_[0], uk_[1], uk_[2]}};
    const BcTab hb{{hc_[0], hc_[1], hc_[2]}, {hk_[0], hk_[1], hk_[2]}};
    const BcTab pb{{pc_, pc_, pc_}, {pk_, pk_, pk_}};
    const bool doAdjust = needReference_ && nFreeUFaces_ > 0;
    const int refCell = deviceCell(ctl.p_ref_cell);
    CFG_CUDA(cudaMemsetAsync(scal_, 0, S_COUNT * sizeof(double), stream_));
    tally_ = scal_ + S_TINNER;
    if (turb_) turbCorrect(lastTurbInner);  // simpleSolver.cpp:52
    tally_ = scal_ + S_UINNER;
    // ---- momentum ----
    {
        const double* xs[1] = {p_};
        V3P g[1] = {gPn_};
        gradCells(xs, 1, pb, gs, true, g);
    }
    const bool timeTerm = ctl.dt > 0;
    MomArgs ma{phi_, gU_, ub, alpha, {ctl.body_force[0], ctl.body_force[1], ctl.body_force[2]}, cv(gPn_),
               linUpwindGrad(ub, gs), {}, mVal_, uDiag_, uBase_, timeTerm ? ctl.dt : 0.0,
               timeTerm ? cv(uOld_) : CV3P{}};
    ma.gUc = CGrad3{{cv(gA_), cv(gB_), cv(Hf_)}};
    k_assemble_U<<<G_, TPB, 0, stream_>>>(dm_, ma);
    launchCheck("assemble_U");
    uPrecond_ = ctl.u_precond;
    solveMomentum(ctl.non_orth_correctors, gs, ctl.linear_tol, ctl.linear_max_iter, uInner);
    uPrecond_ = CFG_PRECOND_JACOBI;
    k_hfree<<<G_, TPB, 0, stream_>>>(dm_, uDiag_, cv(U_), cv(ux_), ctl.relax_u, Hf_, rAUr_);
    launchCheck("hfree");
    // ---- predictor flux ----
    k_flux<<<GF_, TPB, 0, stream_>>>(dm_, cv(Hf_), hb, nullptr, phi_);
    launchCheck("flux");
    if (doAdjust)
    {
        k_adjust_sums<<<1, 32, 0, stream_>>>(phi_, dpStart_, dpSize_, dpFree_, static_cast<int>(mesh_.patches.size()),
                                             scal_);
        launchCheck("adjust_sums");
        k_adjust_scale<<<GF_, TPB, 0, stream_>>>(dm_.nB, dm_.nI, dFreeFace_, phi_, scal_);
        launchCheck("adjust_scale");
    }
    // ---- pressure ----
    k_face_interp<<<GF_, TPB, 0, stream_>>>(dm_, rAUr_, rAUf_);
    launchCheck("face_interp");
    k_assemble_p<<<G_, TPB, 0, stream_>>>(dm_, phi_, rAUf_, pc_, pk_, pVal_d_, pDiag_, pBase_, scal_, refCell,
                                          ctl.p_ref_value);
    launchCheck("assemble_p");
    tally_ = scal_ + S_PINNER;
    solvePressure(ctl.non_orth_correctors, gs, ctl.linear_tol, ctl.linear_max_iter, ctl.p_precond, pInner);
    tally_ = nullptr;
    {
        const double* xs[1] = {px_};
        V3P g[1] = {gPF_};
        gradCells(xs, 1, pb, gs, true, g);
    }
    k_correct_flux<<<GF_, TPB, 0, stream_>>>(dm_, px_, cv(gPF_), rAUf_, pc_, pk_, schemes_.laplacian_corrected, phi_);
    launchCheck("correct_flux");
    k_pstep<<<G_, TPB, 0, stream_>>>(nC, px_, p_, scal_);
    launchCheck("pstep");
    k_update<<<G_, TPB, 0, stream_>>>(nC, px_, p_, U_, cv(Hf_), cv(gPF_), cv(gPn_), rAUr_, ctl.relax_p,
                                      ctl.p_relax_start, scal_);
    launchCheck("update");
    k_continuity<<<G_, TPB, 0, stream_>>>(dm_, phi_, scal_, S_CONT_AFTER);
    launchCheck("continuity");
    CFG_CUDA(cudaMemcpyAsync(scalHost_, scal_, S_COUNT * sizeof(double), cudaMemcpyDeviceToHost, stream_));
}

/// The host's reading of an outer iteration's scalars (simpleSolver.cpp:
/// 334-390): the result fields, and 1 when the loop stops (diverged or
/// converged).
int Ctx::finishOuter(const cfg_simple_controls& ctl, int iter, double& contLag1, double& contLag2,
                     cfg_simple_result& res)
{
    const double* S = scalHost_;
    const double contErr = S[S_CONT], errAfter = S[S_CONT_AFTER], pDeltaMax = S[S_PDELTA];
    const double uRes = S[S_DUMAX] / std::max(S[S_UMAX], 1e-300);
    if (ctl.verbose)
        std::printf("[chflow] SIMPLE iter %d: continuity %g (corrected %g, dp %g, dU %g)\n", iter, contErr, errAfter,
                    pDeltaMax, uRes);
    res.iterations = iter;
    res.final_continuity_error = contErr;
    res.final_momentum_residual = uRes;
    res.last_dp = pDeltaMax;
    res.last_continuity_corrected = errAfter;
    if (!std::isfinite(contErr) || !std::isfinite(pDeltaMax) || S[S_NONFINITE] > 0)
    {
        res.diverged = 1;
        if (ctl.verbose) std::printf("[chflow] error: SIMPLE: diverged at iteration %d\n", iter);
        return 1;
    }
    const bool settled = contErr <= contLag2 * 1.01 + 1e-12;
    const bool momentumSettled = !(ctl.momentum_tol > 0) || uRes <= ctl.momentum_tol;
    if (momentumSettled &&
        (contErr < ctl.continuity_tol || (iter >= 5 && ctl.pcorr_tol > 0 && pDeltaMax < ctl.pcorr_tol && settled)))
    {
        res.converged = 1;
        return 1;
    }
    contLag2 = contLag1;
    contLag1 = contErr;
    return 0;
}

void Ctx::deviceInner(int64_t& u, int64_t& p, int64_t& t) const
{
    u = static_cast<int64_t>(scalHost_[S_UINNER]);
    p = static_cast<int64_t>(scalHost_[S_PINNER]);
    t = static_cast<int64_t>(scalHost_[S_TINNER]);
}

void Ctx::iterate(const cfg_simple_controls& ctl, cfg_simple_result& res)
{
    prepareIterate(ctl);
    std::memset(&res, 0, sizeof res);
    lastTurbInner = 0;
    double contLag1 = INFINITY, contLag2 = INFINITY;
    launches_ = 0;
    for (int k = 0; k < 8; ++k) lastMs[k] = 0.0;
    CFG_CUDA(cudaEventRecord(tm_.ev[0], stream_));
    for (int iter = 1; iter <= ctl.max_iterations; ++iter)
    {
        enqueueOuter(ctl, res.u_inner_iterations, res.p_inner_iterations);
        CFG_CUDA(cudaStreamSynchronize(stream_));
        if (finishOuter(ctl, iter, contLag1, contLag2, res)) break;
    }
    CFG_CUDA(cudaEventRecord(tm_.ev[1], stream_));
    CFG_CUDA(cudaEventSynchronize(tm_.ev[1]));
    float ms = 0;
    CFG_CUDA(cudaEventElapsedTime(&ms, tm_.ev[0], tm_.ev[1]));
    lastMs[7] = ms;
    lastLaunches = launches_;
}

/// solveTransientIncompressiblePiso (pisoSolver.cpp:13-237), one time step
void Ctx::pisoStep(const cfg_piso_controls& ctl, cfg_piso_result& res)
{
    CFG_CUDA(cudaSetDevice(device_));
    if (!(ctl.dt > 0)) fail(CFG_EINVAL, "PISO: non-positive time step");
    refreshBc();
    checkMomentumBcs();
    // the RANS model advances first, with the step's dt, and hands the
    // momentum equation nu + nut on faces (pisoSolver.cpp:29-30)
    lastTurbInner = 0;
    if (turb_) turbCorrect(lastTurbInner, ctl.dt);
    else setNu(ctl.nu);
    std::memset(&res, 0, sizeof res);
    const int nC = dm_.nC;
    const int gs = schemes_.grad;
    const double alpha = schemes_.div == CFG_DIV_BLEND ? schemes_.blend_coeff : (schemes_.div == CFG_DIV_LINEAR ? 1.0 : 0.0);
    const BcTab ub{{uc_[0], uc_[1], uc_[2]}, {uk_[0], uk_[1], uk_[2]}};
    const BcTab hb{{hc_[0], hc_[1], hc_[2]}, {hk_[0], hk_[1], hk_[2]}};
    const BcTab pb{{pc_, pc_, pc_}, {pk_, pk_, pk_}};
    if (!uOld_.c[0])
        for (int q = 0; q < 3; ++q) uOld_.c[q] = alloc<double>(nC);
    launches_ = 0;
    CFG_CUDA(cudaEventRecord(tm_.ev[0], stream_));
    CFG_CUDA(cudaMemsetAsync(scal_, 0, S_COUNT * sizeof(double), stream_));
    {
        const double* xs[1] = {p_};
        V3P g[1] = {gPn_};
        gradCells(xs, 1, pb, gs, true, g);
    }
    for (int q = 0; q < 3; ++q)
        CFG_CUDA(cudaMemcpyAsync(uOld_.c[q], U_.c[q], nC * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    MomArgs ma{phi_, gU_, ub, alpha, {ctl.body_force[0], ctl.body_force[1], ctl.body_force[2]}, cv(gPn_),
               linUpwindGrad(ub, gs), {}, mVal_, uDiag_, uBase_, ctl.dt, cv(uOld_)};
    ma.gUc = CGrad3{{cv(gA_), cv(gB_), cv(Hf_)}};
    k_assemble_U<<<G_, TPB, 0, stream_>>>(dm_, ma);
    launchCheck("assemble_U");
    solveMomentum(ctl.non_orth_correctors, gs, ctl.linear_tol, ctl.linear_max_iter, res.u_inner_iterations);
    for (int q = 0; q < 3; ++q)
        CFG_CUDA(cudaMemcpyAsync(U_.c[q], ux_.c[q], nC * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    const DMat A{nC, dm_.mStart, dm_.mCol};
    auto hbya = [&]() {
        dispatchW(maxW_, [&](auto Wc) {
            constexpr int W = decltype(Wc)::value;
            k_piso_hbya<W><<<G_, TPB, 0, stream_>>>(A, mVal_, uDiag_, cv(uRhs_), cv(U_), cv(gPn_), dm_.V, rAUr_, Hf_);
        });
        launchCheck("piso_hbya");
    };
    hbya();
    k_face_interp<<<GF_, TPB, 0, stream_>>>(dm_, rAUr_, rAUf_);
    launchCheck("face_interp");
    for (int corr = 1; corr <= ctl.correctors; ++corr)
    {
        if (corr > 1) hbya();
        CFG_CUDA(cudaMemsetAsync(scal_, 0, S_COUNT * sizeof(double), stream_));
        k_flux<<<GF_, TPB, 0, stream_>>>(dm_, cv(Hf_), hb, nullptr, phi_);
        launchCheck("flux");
        k_assemble_p<<<G_, TPB, 0, stream_>>>(dm_, phi_, rAUf_, pc_, pk_, pVal_d_, pDiag_, pBase_, scal_, -1, 0.0);
        launchCheck("assemble_p");
        solvePressure(ctl.non_orth_correctors, gs, ctl.linear_tol, ctl.linear_max_iter, ctl.p_precond,
                      res.p_inner_iterations, p_);
        k_pstep<<<G_, TPB, 0, stream_>>>(nC, px_, p_, scal_);
        launchCheck("pstep");
        CFG_CUDA(cudaMemcpyAsync(p_, px_, nC * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
        {
            const double* xs[1] = {p_};
            V3P g[1] = {gPF_};
            gradCells(xs, 1, pb, gs, true, g);
        }
        k_piso_update<<<G_, TPB, 0, stream_>>>(nC, cv(Hf_), rAUr_, cv(gPF_), U_);
        launchCheck("piso_update");
        k_correct_flux<<<GF_, TPB, 0, stream_>>>(dm_, p_, cv(gPF_), rAUf_, pc_, pk_, schemes_.laplacian_corrected,
                                                 phi_);
        launchCheck("correct_flux");
        k_continuity<<<G_, TPB, 0, stream_>>>(dm_, phi_, scal_, S_CONT_AFTER);
        launchCheck("continuity");
        CFG_CUDA(cudaMemcpyAsync(scalHost_, scal_, S_COUNT * sizeof(double), cudaMemcpyDeviceToHost, stream_));
        CFG_CUDA(cudaStreamSynchronize(stream_));
        const double* S = scalHost_;
        res.predicted_continuity_error = S[S_CONT];
        res.continuity_error = S[S_CONT_AFTER];
        res.pressure_correction_max = S[S_PSTEP];
        res.correctors_used = corr;
        if (!std::isfinite(res.continuity_error) || !std::isfinite(res.pressure_correction_max))
        {
            res.diverged = 1;
            break;
        }
        if (res.continuity_error < ctl.continuity_tol)
        {
            res.converged = 1;
            break;
        }
    }
    CFG_CUDA(cudaEventRecord(tm_.ev[1], stream_));
    CFG_CUDA(cudaEventSynchronize(tm_.ev[1]));
    float ms = 0;
    CFG_CUDA(cudaEventElapsedTime(&ms, tm_.ev[0], tm_.ev[1]));
    res.device_ms = ms;
    lastLaunches = launches_;
}

void Ctx::probeEquations(const cfg_simple_controls& ctl, const double* xprobe, double* out)
{
    // the equations of one outer iteration built from the current fields,
    // as oracle/ref_driver.cpp's `eqns` mode builds them; out holds, in
    // order: gradPn (3N), U diag (3N), U h0 (3N), U h1 (3N), rAUf (F),
    // divPhi (N), contErr (1), p diag (N), p h0 (N), p h1 (N), gradPFull (3N),
    // phiCorrected (F).  Vectors are component-major.
    CFG_CUDA(cudaSetDevice(device_));
    refreshBc();
    checkMomentumBcs();
    setNu(ctl.nu);
    const int nC = dm_.nC, nF = dm_.nF;
    const int gs = schemes_.grad;
    const double alpha = schemes_.div == CFG_DIV_BLEND ? schemes_.blend_coeff : (schemes_.div == CFG_DIV_LINEAR ? 1.0 : 0.0);
    const BcTab ub{{uc_[0], uc_[1], uc_[2]}, {uk_[0], uk_[1], uk_[2]}};
    const BcTab pb{{pc_, pc_, pc_}, {pk_, pk_, pk_}};
    const DMat A{nC, dm_.mStart, dm_.mCol};
    double* o = out;
    // cell arrays back in the original numbering, face arrays as they are
    auto d2hC = [&](const double* src) {
        fromDevCells(o, src, 1, 0);
        o += nC;
    };
    auto d2hF = [&](const double* src) {
        CFG_CUDA(cudaMemcpyAsync(o, src, nF * sizeof(double), cudaMemcpyDeviceToHost, stream_));
        CFG_CUDA(cudaStreamSynchronize(stream_));
        o += nF;
    };
    CFG_CUDA(cudaMemsetAsync(scal_, 0, S_COUNT * sizeof(double), stream_));
    double* xp = cr_;
    toDevCells(xp, xprobe, 1, 0);
    {
        const double* xs[1] = {p_};
        V3P g[1] = {gPn_};
        gradCells(xs, 1, pb, gs, true, g);
    }
    for (int q = 0; q < 3; ++q) d2hC(gPn_.c[q]);
    MomArgs ma{phi_, gU_, ub, alpha, {ctl.body_force[0], ctl.body_force[1], ctl.body_force[2]}, cv(gPn_),
               linUpwindGrad(ub, gs), {}, mVal_, uDiag_, uBase_, 0.0, CV3P{}};
    ma.gUc = CGrad3{{cv(gA_), cv(gB_), cv(Hf_)}};
    k_assemble_U<<<G_, TPB, 0, stream_>>>(dm_, ma);
    launchCheck("assemble_U");
    // one pass with maxIter 0: rhs = base + corrector(x = 0)
    for (int q = 0; q < 3; ++q) CFG_CUDA(cudaMemsetAsync(ux_.c[q], 0, nC * sizeof(double), stream_));
    if (schemes_.laplacian_corrected)
    {
        const double* xs[3] = {ux_.c[0], ux_.c[1], ux_.c[2]};
        V3P g[3] = {gA_, gB_, Hf_};
        gradCells(xs, 3, ub, gs, false, g);
        k_corrector<3><<<G_, TPB, 0, stream_>>>(dm_, gU_, CGrad3{{cv(g[0]), cv(g[1]), cv(g[2])}}, cv(uBase_), uRhs_);
        launchCheck("corrector_U");
    }
    else
    {
        for (int q = 0; q < 3; ++q)
            CFG_CUDA(cudaMemcpyAsync(uRhs_.c[q], uBase_.c[q], nC * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    }
    for (int q = 0; q < 3; ++q) d2hC(uDiag_);
    for (int pass = 0; pass < 2; ++pass)
        for (int q = 0; q < 3; ++q)
        {
            k_explicit_op<<<G_, TPB, 0, stream_>>>(A, mVal_, uDiag_, uRhs_.c[q], pass ? xp : ux_.c[0], cAp_);
            launchCheck("explicit_op");
            d2hC(cAp_);
        }
    k_hfree<<<G_, TPB, 0, stream_>>>(dm_, uDiag_, cv(U_), cv(ux_), 1.0, Hf_, rAUr_);
    launchCheck("hfree");
    k_face_interp<<<GF_, TPB, 0, stream_>>>(dm_, rAUr_, rAUf_);
    launchCheck("face_interp");
    d2hF(rAUf_);
    const int refCell = ctl.p_ref_cell >= 0 && ctl.p_ref_cell < nC ? deviceCell(ctl.p_ref_cell) : -1;
    k_assemble_p<<<G_, TPB, 0, stream_>>>(dm_, phi_, rAUf_, pc_, pk_, pVal_d_, pDiag_, pBase_, scal_, refCell,
                                          ctl.p_ref_value);
    launchCheck("assemble_p");
    std::vector<double> hostScal(S_COUNT);
    CFG_CUDA(cudaMemcpyAsync(hostScal.data(), scal_, S_COUNT * sizeof(double), cudaMemcpyDeviceToHost, stream_));
    CFG_CUDA(cudaStreamSynchronize(stream_));
    k_divphi<<<G_, TPB, 0, stream_>>>(dm_, phi_, cAp_);
    launchCheck("divphi");
    d2hC(cAp_);
    *o++ = hostScal[S_CONT];
    // pressure equation rhs = base + corrector(x = 0)
    CFG_CUDA(cudaMemsetAsync(px_, 0, nC * sizeof(double), stream_));
    if (schemes_.laplacian_corrected)
    {
        const double* xs[1] = {px_};
        V3P g[1] = {gA_};
        gradCells(xs, 1, pb, gs, false, g);
        k_corrector<1><<<G_, TPB, 0, stream_>>>(dm_, rAUf_, CGrad3{{cv(gA_)}}, CV3P{{pBase_, pBase_, pBase_}},
                                               V3P{{pRhs_, pRhs_, pRhs_}});
        launchCheck("corrector_p");
    }
    else
    {
        CFG_CUDA(cudaMemcpyAsync(pRhs_, pBase_, nC * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    }
    d2hC(pDiag_);
    for (int pass = 0; pass < 2; ++pass)
    {
        k_explicit_op<<<G_, TPB, 0, stream_>>>(A, pVal_d_, pDiag_, pRhs_, pass ? xp : px_, cAp_);
        launchCheck("explicit_op");
        d2hC(cAp_);
    }
    {
        const double* xs[1] = {xp};
        V3P g[1] = {gPF_};
        gradCells(xs, 1, pb, gs, true, g);
    }
    for (int q = 0; q < 3; ++q) d2hC(gPF_.c[q]);
    CFG_CUDA(cudaMemcpyAsync(fScratch_, phi_, nF * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    k_correct_flux<<<GF_, TPB, 0, stream_>>>(dm_, xp, cv(gPF_), rAUf_, pc_, pk_, schemes_.laplacian_corrected,
                                             fScratch_);
    launchCheck("correct_flux");
    d2hF(fScratch_);
}

void Ctx::probeDIC(const double* r, double* z, double* rDinv)
{
    // the DIC of the pressure matrix last assembled (by probeEquations or an
    // outer iteration): factor, then one application to r
    CFG_CUDA(cudaSetDevice(device_));
    SolveState init{};
    init.maxIter = 1;
    CFG_CUDA(cudaMemcpyAsync(st_, &init, sizeof(SolveState), cudaMemcpyHostToDevice, stream_));
    dicSetup(pVal_d_, pDiag_);
    toDevCells(cr_, r, 1, 0);
    dicApply(cr_, cz_);
    fromDevCells(z, cz_, 1, 0);
    fromDevCells(rDinv, dic_.rDinv, 1, 0);
}

void Ctx::gradient(const double* data, const double* bvals, int scheme, int volQuirk, double* out)
{
    // fvc::grad of one cell field with fixed boundary face values
    CFG_CUDA(cudaSetDevice(device_));
    const int nB = dm_.nB;
    double* x = cr_;
    double* k = bScratch_;
    double* c0 = bScratch_ + nB;
    toDevCells(x, data, 1, 0);
    CFG_CUDA(cudaMemcpyAsync(k, bvals, nB * sizeof(double), cudaMemcpyHostToDevice, stream_));
    CFG_CUDA(cudaMemsetAsync(c0, 0, nB * sizeof(double), stream_));
    const BcTab bt{{c0, c0, c0}, {k, k, k}};
    const double* xs[1] = {x};
    V3P g[1] = {gPF_};
    gradCells(xs, 1, bt, scheme, volQuirk != 0, g);
    for (int q = 0; q < 3; ++q) fromDevCells(out, gPF_.c[q], 3, q);
}

/// The FP32 copies of the pressure system and the vectors of its FP32
/// solves (mixed-precision refinement), allocated on first use.
void Ctx::ensureMixed()
{
    if (mixedReady_) return;
    const int nC = dm_.nC;
    if (!pVal32_) pVal32_ = alloc<float>(static_cast<size_t>(nSlicesEntries_));
    pDiag32_ = alloc<float>(nC);
    r32_ = alloc<float>(nC);
    p32_ = alloc<float>(nC);
    Ap32_ = alloc<float>(nC);
    z32_ = alloc<float>(nC);
    e32_ = alloc<float>(nC);
    b32_ = alloc<float>(nC);
    dic32_.nColours = dic_.nColours;
    dic32_.rows = dic_.rows;
    dic32_.lStart = dic_.lStart;
    dic32_.lCol = dic_.lCol;
    dic32_.lSrc = dic_.lSrc;
    dic32_.uStart = dic_.uStart;
    dic32_.uCol = dic_.uCol;
    dic32_.uSrc = dic_.uSrc;
    dic32_.lVal = alloc<float>(nLo_);
    dic32_.uVal = alloc<float>(nUp_);
    dic32_.rD = alloc<float>(nC);
    dic32_.rDinv = alloc<float>(nC);
    mixedReady_ = true;
}

/// FP32 DIC-PCG corrections inside FP64 iterative refinement, on the
/// pressure system whose FP32 copy and FP32 DIC factor are current: each
/// refinement step computes r = b - A x and the reference's test |r|inf /
/// |b|inf < tol in FP64 (Matrix.cpp:166-180), solves A32 e = r32 in FP32 to
/// innerTol (2-norm relative), and adds e to x in FP64.  rep counts the
/// inner iterations (at most maxIter over all steps).
void Ctx::runIR32(const double* vals, const double* diag, const double* b, double* x, double tol, int maxIter,
                  double innerTol, cfg_solver_report* rep)
{
    const int nC = dm_.nC;
    const DMat A{nC, dm_.mStart, dm_.mCol};
    int64_t inner = 0;
    int outer = 0;
    double init = -1.0, fin = 0.0;
    bool conv = false;
    for (;;)
    {
        SolveState s0{};
        s0.tol = tol;
        s0.maxIter = 0;
        s0.normType = 0;
        CFG_CUDA(cudaMemcpyAsync(st_, &s0, sizeof(SolveState), cudaMemcpyHostToDevice, stream_));
        dispatchW(maxW_, [&](auto Wc) {
            constexpr int W = decltype(Wc)::value;
            k_cg_init<W, double><<<GS_, TPB, 0, stream_>>>(A, vals, diag, b, x, cr_, cz_, partials_, st_);
        });
        launchCheck("ir_residual");
        CFG_CUDA(cudaMemcpyAsync(stHost_, st_, sizeof(SolveState), cudaMemcpyDeviceToHost, stream_));
        CFG_CUDA(cudaStreamSynchronize(stream_));
        fin = stHost_->init[0];
        if (init < 0) init = fin;
        conv = stHost_->conv[0] != 0;
        if (conv || std::isnan(fin) || inner >= maxIter || outer >= 64) break;
        k_to_float<<<G_, TPB, 0, stream_>>>(nC, cr_, b32_);
        CFG_CUDA(cudaMemsetAsync(e32_, 0, nC * sizeof(float), stream_));
        cfg_solver_report r2{};
        dicCGT<float>(dic32_, pVal32_, pDiag32_, b32_, e32_, r32_, p32_, Ap32_, z32_, innerTol,
                      static_cast<int>(std::min<int64_t>(2000, maxIter - inner)), 1, &r2);
        k_add_f32<<<G_, TPB, 0, stream_>>>(nC, e32_, x);
        launchCheck("ir_update");
        inner += r2.iterations;
        ++outer;
        if (r2.iterations == 0) break;  // no progress in FP32
    }
    rep->iterations = static_cast<int32_t>(inner);
    rep->converged = conv;
    rep->initial_residual = init;
    rep->final_residual = fin;
}

void Ctx::poissonSetup(int64_t refCell)
{
    CFG_CUDA(cudaSetDevice(device_));
    refreshBc();
    const int nC = dm_.nC, nF = dm_.nF;
    if (refCell >= nC) fail(CFG_EINVAL, "cfg_poisson_setup: reference cell beyond the last cell");
    ensureMixed();
    if (!poissonReady_)
    {
        pb64_ = alloc<double>(nC);
        px64_ = alloc<double>(nC);
        poissonReady_ = true;
    }
    // unit face coefficient, no flux: laplacianFace(1) and the p conditions
    k_fill<<<GF_, TPB, 0, stream_>>>(nF, 1.0, rAUf_);
    CFG_CUDA(cudaMemsetAsync(fScratch_, 0, nF * sizeof(double), stream_));
    CFG_CUDA(cudaMemsetAsync(scal_, 0, S_COUNT * sizeof(double), stream_));
    k_assemble_p<<<G_, TPB, 0, stream_>>>(dm_, fScratch_, rAUf_, pc_, pk_, pVal_d_, pDiag_, pBase_, scal_,
                                          deviceCell(refCell), 0.0);
    launchCheck("poisson_assemble");
    const int nE = nSlicesEntries_;
    k_to_float<<<std::max(1, std::min((nE + TPB - 1) / TPB, 8192)), TPB, 0, stream_>>>(nE, pVal_d_, pVal32_);
    k_to_float<<<G_, TPB, 0, stream_>>>(nC, pDiag_, pDiag32_);
    launchCheck("poisson_float");
    dicSetupT<double>(dic_, pVal_d_, pDiag_);
    dicSetupT<float>(dic32_, pVal_d_, pDiag32_);
    amgFresh_ = false;
    CFG_CUDA(cudaStreamSynchronize(stream_));
}

void Ctx::poissonAmg(double* out)
{
    if (!poissonReady_) fail(CFG_EINVAL, "cfg_poisson_amg_setup: call cfg_poisson_setup first");
    CFG_CUDA(cudaSetDevice(device_));
    amgValues(kAmgPressure, pVal_d_, pDiag_, pVal32_);
    amgFresh_ = true;
    amgInfo(out);
}

void Ctx::poissonAmgApply(const double* r, double* z)
{
    if (!amgFresh_)
    {
        double info[11];
        poissonAmg(info);
    }
    toDevCells(cr_, r, 1, 0);
    amgApply(cr_, cz_);
    fromDevCells(z, cz_, 1, 0);
}

void Ctx::poissonAmgApply3(const double* r, double* z, const int32_t done[3])
{
    if (!amgFresh_)
    {
        double info[11];
        poissonAmg(info);
    }
    // the three vectors in the momentum solver's p and z buffers, the done
    // flags in the solver state (as the momentum BiCGStab hands them over)
    for (int q = 0; q < 3; ++q) toDevCells(bp_.c[q], r + static_cast<size_t>(q) * dm_.nC, 1, 0);
    amgVectors3(kAmgPressure);
    SolveState s0{};
    for (int q = 0; q < 3; ++q) s0.done[q] = done[q];
    CFG_CUDA(cudaMemcpyAsync(st_, &s0, sizeof(SolveState), cudaMemcpyHostToDevice, stream_));
    for (int q = 0; q < 3; ++q) toDevCells(bz_.c[q], z + static_cast<size_t>(q) * dm_.nC, 1, 0);
    // the pressure V-cycle's coarse-correction scale, so that each component
    // equals the single V-cycle's result
    amgCycle3(kAmgPressure, cv(bp_), bz_, reinterpret_cast<const int*>(reinterpret_cast<const char*>(st_) + offsetof(SolveState, done)),
              kAmgScalePressure);
    for (int q = 0; q < 3; ++q) fromDevCells(z + static_cast<size_t>(q) * dm_.nC, bz_.c[q], 1, 0);
}

void Ctx::poissonSolve(const double* b, double* x, int method, double tol, int maxIter, int innerMax, double innerTol,
                       double* out)
{
    // out: inner iterations, outer iterations, converged, true |b-Ax|2/|b|2,
    //      device ms, initial true relative residual
    if (!poissonReady_) fail(CFG_EINVAL, "cfg_poisson_solve: call cfg_poisson_setup first");
    CFG_CUDA(cudaSetDevice(device_));
    const int nC = dm_.nC;
    const DMat A{nC, dm_.mStart, dm_.mCol};
    toDevCells(pb64_, b, 1, 0);
    toDevCells(px64_, x, 1, 0);
    // true residual |b - A x|2 / |b|2 in FP64 (r left in cr_)
    auto trueRel = [&]() {
        SolveState s0{};
        s0.normType = 1;
        s0.maxIter = 0;
        CFG_CUDA(cudaMemcpyAsync(st_, &s0, sizeof(SolveState), cudaMemcpyHostToDevice, stream_));
        dispatchW(maxW_, [&](auto Wc) {
            constexpr int W = decltype(Wc)::value;
            k_cg_init<W, double><<<GS_, TPB, 0, stream_>>>(A, pVal_d_, pDiag_, pb64_, px64_, cr_, cz_, partials_, st_);
        });
        launchCheck("true_residual");
        CFG_CUDA(cudaMemcpyAsync(stHost_, st_, sizeof(SolveState), cudaMemcpyDeviceToHost, stream_));
        CFG_CUDA(cudaStreamSynchronize(stream_));
        return stHost_->init[0] / stHost_->bnorm[0];
    };
    // the AMG hierarchy is set up outside the timed solve, as the DIC
    // factors are (cfg_poisson_amg_setup reports what it costs)
    if ((method == 4 || method == 5) && !amgFresh_)
    {
        double info[11];
        poissonAmg(info);
    }
    CFG_CUDA(cudaStreamSynchronize(stream_));
    const double rel0 = trueRel();
    CFG_CUDA(cudaEventRecord(tm_.ev[2], stream_));
    int64_t inner = 0;
    int outer = 0;
    cfg_solver_report rep{};
    if (method == 0)
    {
        runCG(pVal_d_, pDiag_, pb64_, px64_, tol, maxIter, &rep, 1);
        inner = rep.iterations;
        outer = 1;
    }
    else if (method == 1)
    {
        dicCGT<double>(dic_, pVal_d_, pDiag_, pb64_, px64_, cr_, cp_, cAp_, cz_, tol, maxIter, 1, &rep);
        inner = rep.iterations;
        outer = 1;
    }
    else if (method == 2)
    {
        // FP32 DIC-PCG corrections inside FP64 iterative refinement
        double rel = rel0;
        while (rel > tol && outer < 100 && inner < maxIter)
        {
            k_to_float<<<G_, TPB, 0, stream_>>>(nC, cr_, b32_);
            CFG_CUDA(cudaMemsetAsync(e32_, 0, nC * sizeof(float), stream_));
            dicCGT<float>(dic32_, pVal32_, pDiag32_, b32_, e32_, r32_, p32_, Ap32_, z32_, innerTol,
                          std::min(innerMax, static_cast<int>(maxIter - inner)), 1, &rep);
            inner += rep.iterations;
            k_add_f32<<<G_, TPB, 0, stream_>>>(nC, e32_, px64_);
            launchCheck("ir_update");
            ++outer;
            rel = trueRel();
        }
    }
    else if (method == 3)
    {
        // flexible CG with the learned preconditioner, DIC-PCG when it stalls
        if (!mpnn_) fail(CFG_EINVAL, "cfg_poisson_solve: fcg_mpnn needs cfg_mpnn_create");
        int64_t o[3];
        mpnnFcg(pVal_d_, pDiag_, pb64_, px64_, tol, maxIter, 25, o, 1);
        inner = o[0] + o[1];
        outer = 1 + static_cast<int>(o[2]);
        lastFallbackIters = o[1];
    }
    else if (method == 4)
    {
        // flexible CG with the FP32 AMG V-cycle, every scalar on the device
        amgFcg(pVal_d_, pb64_, px64_, tol, maxIter, 1, &rep);
        inner = rep.iterations;
        outer = 1;
    }
    else if (method == 5)
    {
        // the same with the learned correction after each V-cycle (host
        // driven: the network's application is its own launch sequence);
        // DIC-PCG when it stalls
        if (!mpnn_) fail(CFG_EINVAL, "cfg_poisson_solve: fcg_amg_mpnn needs cfg_mpnn_create");
        int64_t o[3];
        mpnnFcg(pVal_d_, pDiag_, pb64_, px64_, tol, maxIter, 25, o, 1, 2);
        inner = o[0] + o[1];
        outer = 1 + static_cast<int>(o[2]);
        lastFallbackIters = o[1];
    }
    else
    {
        fail(CFG_EINVAL, "cfg_poisson_solve: unknown method");
    }
    CFG_CUDA(cudaEventRecord(tm_.ev[3], stream_));
    CFG_CUDA(cudaEventSynchronize(tm_.ev[3]));
    float ms = 0;
    CFG_CUDA(cudaEventElapsedTime(&ms, tm_.ev[2], tm_.ev[3]));
    const double rel = trueRel();
    fromDevCells(x, px64_, 1, 0);
    out[0] = static_cast<double>(inner);
    out[1] = outer;
    out[2] = rel <= tol ? 1.0 : 0.0;
    out[3] = rel;
    out[4] = ms;
    out[5] = rel0;
}

// the FP64 DIC-PCG is also the fallback of the learned preconditioner (mpnn.cu)
template void Ctx::dicCGT<double>(const DDicT<double>&, const double*, const double*, const double*, double*, double*,
                                  double*, double*, double*, double, int, int, cfg_solver_report*);

}  // namespace cfg
