// The reference's RANS models with Spalding wall functions, on the device,
// as its RansModel advances them once per SIMPLE outer iteration
// (src/3d/src/turbulence/turbulenceModel.cpp, wallFunction.cpp; called from
// simpleSolver.cpp:52 and fed to the momentum laplacian as nuEffFace,
// simpleSolver.cpp:97): standard k-epsilon (kEpsilon.cpp), Menter's
// k-omega SST (kOmegaSST.cpp), the shielded DES length on k-epsilon
// (desModel.cpp) and the gamma-transition intermittency on k-epsilon
// (transitionModel.cpp).  The k-epsilon flow is described below; the others
// change the hooks noted at their kernels.
//
// Per outer iteration (RansModel::correctTurbulence, turbulenceModel.cpp):
//   strain rate |S| and production nut 2 S:S from the U-component gradients;
//   the wall layer: u_tau, y+ and the wall nut of every wall face from
//     Spalding's law (bisection), the wall epsilon u_tau^3 / (kappa y);
//   k: div(phi,k) - laplacian(nu + nut/sigmaK, k) + (eps/k) k = P, relaxed;
//   epsilon: ... + C2 (eps/k) eps = C1 (eps/k) P, relaxed;
//   wall-adjacent cells set to the log-layer equilibrium;
//   nut = Cmu k^2 / eps; nuEff on faces = nu + harmonic(nut), nu + wall nut
//     on wall faces.
// Each scalar equation is assembled by cell gathers in the reference's term
// and face order and solved with the same Jacobi-BiCGStab and
// non-orthogonal passes (fvMatrix::solve with nonOrth 2, tol 1e-8).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <queue>
#include <utility>
#include <vector>

#include "ctx.h"
#include "kernels.cuh"

namespace cfg
{

namespace
{

constexpr double kCmu = 0.09, kC1 = 1.44, kC2 = 1.92, kSigmaK = 1.0, kSigmaE = 1.3;
constexpr double kKappa = 0.41, kSpaldingC = 5.5676;
// k-omega SST (KOmegaSST.h): Menter 2003 constants, the two gammas formed as
// the reference forms them
constexpr double kBetaStar = 0.09, kBeta1 = 0.075, kBeta2 = 0.0828;
constexpr double kSigK1 = 0.85, kSigK2 = 1.0, kSigW1 = 0.5, kSigW2 = 0.856, kA1 = 0.31;
constexpr double kSqrtBetaStar = 0.3, kProdLimit = 10.0;
constexpr double kGamma1 = kBeta1 / kBetaStar - kSigW1 * kKappa * kKappa / kSqrtBetaStar;
constexpr double kGamma2 = kBeta2 / kBetaStar - kSigW2 * kKappa * kKappa / kSqrtBetaStar;
enum TurbModel
{
    TM_KEPS = 0,
    TM_SST = 1,
    TM_DES = 2,
    TM_TRANSITION = 3
};
constexpr double kFloor = 1e-12, kDissFloor = 1e-12;
constexpr double kLinTol = 1e-8;
constexpr int kLinMaxIter = 2000, kNonOrth = 2;

/// Spalding's y+(u+) (wallFunction.cpp:7-16)
__device__ double spalding_yplus(double uPlus)
{
    if (uPlus <= 0) return 0;
    const double ku = kKappa * uPlus;
    const double damp = exp(-kKappa * kSpaldingC);
    return uPlus + damp * (exp(ku) - 1.0 - ku - 0.5 * ku * ku - ku * ku * ku / 6.0);
}

/// wallState (wallFunction.cpp:93-108) with the bisection of :21-38 on
/// f(u+) = u+ y+(u+)
__device__ void wall_state(double uPar, double y, double nu, double& uTau, double& yPlus, double& nut)
{
    uTau = yPlus = nut = 0.0;
    if (!(uPar > 0) || !(y > 0) || !(nu > 0)) return;
    const double a = uPar * y / nu;
    double lo = 0.0, hi = 1.0;
    while (hi * spalding_yplus(hi) < a)
    {
        lo = hi;
        hi *= 2.0;
        if (hi > 1e6) break;
    }
    for (int i = 0; i < 100 && hi - lo > 1e-13 * hi; ++i)
    {
        const double mid = 0.5 * (lo + hi);
        if (mid * spalding_yplus(mid) > a) hi = mid;
        else lo = mid;
    }
    const double uPlus = 0.5 * (lo + hi);
    uTau = uPar / uPlus;
    yPlus = a / uPlus;
    nut = uTau * uTau * y / uPar - nu;
    if (nut < 0) nut = 0;
}

/// |S| and the production nut 2 S:S (computeStrainRate, :197-226)
__global__ void __launch_bounds__(TPB) k_turb_strain(int n, CGrad3 g, const double* __restrict__ nut,
                                                     double* __restrict__ strain, double* __restrict__ prod)
{
    ROW_LOOP(c, n)
    {
        double s2 = 0;
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int j = 0; j < 3; ++j)
            {
                const double sij = 0.5 * (g.g[i].c[j][c] + g.g[j].c[i][c]);
                s2 += sij * sij;
            }
        strain[c] = sqrt(2.0 * s2);
        prod[c] = nut[c] * 2.0 * s2;
    }
}

/// the wall layer (computeWallLayer, :228-256): one thread per wall face;
/// the epsilon condition of the face becomes the wall value
__global__ void __launch_bounds__(TPB) k_turb_wall(int nW, const int* __restrict__ wFace, const int* __restrict__ wCell,
                                                   const double* __restrict__ wDist, DMesh m, CV3P U, double nu,
                                                   int model, double* uTau, double* yPlus, double* nutWall,
                                                   double* ec, double* ek)
{
    ROW_LOOP(i, nW)
    {
        const int f = wFace[i], c = wCell[i];
        const double sx = m.sfx[f], sy = m.sfy[f], sz = m.sfz[f];
        const double a = sqrt(sx * sx + sy * sy + sz * sz);
        const double nx = sx / a, ny = sy / a, nz = sz / a;
        const double ux = U.c[0][c], uy = U.c[1][c], uz = U.c[2][c];
        const double dn = ux * nx + uy * ny + uz * nz;
        const double px = ux - nx * dn, py = uy - ny * dn, pz = uz - nz * dn;
        const double par = sqrt(px * px + py * py + pz * pz);
        double ut, yp, nt;
        wall_state(par, wDist[i], nu, ut, yp, nt);
        uTau[i] = ut;
        yPlus[i] = yp;
        nutWall[i] = nt;
        const double y = wDist[i];
        double e;
        if (model == TM_SST)
        {
            // omega of the viscous sublayer and of the log layer in
            // quadrature (KOmegaSST::wallDissipation)
            const double wVis = 6.0 * nu / (kBeta1 * y * y);
            const double wLog = ut / (sqrt(kBetaStar) * kKappa * y);
            e = sqrt(wVis * wVis + wLog * wLog);
        }
        else
        {
            e = pow(ut, 3.0) / (kKappa * y);
        }
        const int b = f - m.nI;
        ec[b] = 0.0;
        ek[b] = e < kDissFloor ? kDissFloor : e;
    }
}

/// harmonicFaceGamma of a cell field (laplacianScheme.cpp:37-62), wall
/// faces overridden by nu + wallNut sigma[owner] (diffusionFace,
/// turbulenceModel.cpp:184-195) or by the wall nut alone (refreshFaceNut)
__global__ void __launch_bounds__(TPB) k_turb_face_gamma(DMesh m, const double* __restrict__ dP,
                                                         const double* __restrict__ dN, const double* __restrict__ cell,
                                                         const int* __restrict__ wallOf, const double* __restrict__ nutWall,
                                                         double wallBase, double wallSigma,
                                                         const double* __restrict__ wallSigmaCell, double add,
                                                         double* __restrict__ out)
{
    ROW_LOOP(f, m.nF)
    {
        const int o = m.own[f];
        double g;
        if (f < m.nI)
        {
            const double gp = cell[o], gn = cell[m.nbr[f]];
            const double tot = dP[f] + dN[f];
            g = (tot > 0 && gp > 0 && gn > 0) ? tot * gp * gn / (dN[f] * gp + dP[f] * gn) : 0.5 * (gp + gn);
        }
        else
        {
            g = cell[o];
            const int w = wallOf ? wallOf[f - m.nI] : -1;
            if (w >= 0) g = wallBase + nutWall[w] * (wallSigmaCell ? wallSigmaCell[o] : wallSigma);
        }
        out[f] = add + g;
    }
}

/// gamma = nu + nut sigma (the cell diffusivity of the k or epsilon equation)
__global__ void __launch_bounds__(TPB) k_turb_gamma(int n, double nu, const double* __restrict__ nut, double sigma,
                                                    double* __restrict__ gamma)
{
    ROW_LOOP(c, n) gamma[c] = nu + nut[c] * sigma;
}

/// sources of the k equation: Sp = V eps/k (destructionSp) and V P
__global__ void __launch_bounds__(TPB) k_turb_src_k(int n, const double* __restrict__ V, const double* __restrict__ k,
                                                    const double* __restrict__ eps, const double* __restrict__ prod,
                                                    double* __restrict__ sp, double* __restrict__ src)
{
    ROW_LOOP(c, n)
    {
        const double kk = k[c] < kFloor ? kFloor : k[c];
        sp[c] = V[c] * eps[c] / kk;
        src[c] = V[c] * prod[c];
    }
}

/// sources of the epsilon equation (kEpsilon.cpp:60-67): with the new k
__global__ void __launch_bounds__(TPB) k_turb_src_e(int n, const double* __restrict__ V, const double* __restrict__ k,
                                                    const double* __restrict__ eps, const double* __restrict__ prod,
                                                    double* __restrict__ sp, double* __restrict__ src)
{
    ROW_LOOP(c, n)
    {
        const double kk = k[c] < kFloor ? kFloor : k[c];
        const double e = eps[c] < kDissFloor ? kDissFloor : eps[c];
        src[c] = V[c] * kC1 * e * prod[c] / kk;
        sp[c] = V[c] * kC2 * e / kk;
    }
}

/// a scalar transport equation [ddt(T)] + div(phi,T) - laplacianFace(gamma,T)
/// + Sp T = src, in the reference's term order per cell (fvm::ddt when dt >
/// 0, divScheme.cpp:64-77; fvm::div; laplacianFace; then the source and the
/// implicit Sp)
__global__ void __launch_bounds__(TPB) k_assemble_S(DMesh m, const double* __restrict__ phi,
                                                    const double* __restrict__ gamma, const double* __restrict__ bc,
                                                    const double* __restrict__ bk, double alpha,
                                                    const double* __restrict__ sp, const double* __restrict__ src,
                                                    const double* __restrict__ src2, double dt,
                                                    const double* __restrict__ old, double* __restrict__ val,
                                                    double* __restrict__ diagOut, double* __restrict__ base)
{
    ROW_LOOP(c, m.nC)
    {
        const int sl = c >> 5, lane = c & 31;
        const int e0 = m.cfStart[sl] + lane, e1 = m.cfStart[sl + 1];
        double diag = 0.0, r = 0.0;
        if (dt > 0)
        {
            const double a = m.V[c] / dt;
            diag = a;
            r = a * old[c];
        }
        for (int e = e0; e < e1; e += 32)  // convection
        {
            const int code = m.cfCode[e];
            if (code < 0) break;
            const int f = code >> 1, side = code & 1;
            const double p = phi[f];
            if (f < m.nI)
            {
                double wPo = 0.0, wNo = 0.0;
                if (p >= 0) wPo = 1.0;
                else wNo = 1.0;
                if (alpha > 0)
                {
                    wPo = alpha * m.ow[f] + (1.0 - alpha) * wPo;
                    wNo = alpha * (1.0 - m.ow[f]) + (1.0 - alpha) * wNo;
                }
                diag += side ? -(p * wNo) : p * wPo;
            }
            else
            {
                const int b = m.cfOther[e];
                diag += p * bc[b];
                r += (-p) * bk[b];
            }
        }
        for (int e = e0; e < e1; e += 32)  // diffusion
        {
            const int code = m.cfCode[e];
            if (code < 0) break;
            const int f = code >> 1;
            const double coef = gamma[f] * m.oc[f];
            if (f < m.nI)
            {
                diag += coef;
            }
            else
            {
                const int b = m.cfOther[e];
                diag += (-coef) * (bc[b] - 1.0);
                r += coef * bk[b];
            }
        }
        // the implicit source on the diagonal, the explicit ones on the
        // right-hand side in the order they are added, after the face terms
        diag += sp[c];
        r += src[c];
        if (src2) r += src2[c];
        diagOut[c] = diag;
        base[c] = r;
        const int me1 = m.mStart[sl + 1];
        for (int e = m.mStart[sl] + lane; e < me1; e += 32)
        {
            const int code = m.mCode[e];
            if (code == -1) break;
            double v;
            if (code == -2)
            {
                v = diag;
            }
            else
            {
                const int f = code >> 1, side = code & 1;
                const double p = phi[f];
                double wPo = 0.0, wNo = 0.0;
                if (p >= 0) wPo = 1.0;
                else wNo = 1.0;
                if (alpha > 0)
                {
                    wPo = alpha * m.ow[f] + (1.0 - alpha) * wPo;
                    wNo = alpha * (1.0 - m.ow[f]) + (1.0 - alpha) * wNo;
                }
                const double conv = side ? -(p * wPo) : p * wNo;
                v = conv + (-(gamma[f] * m.oc[f]));
            }
            val[e] = v;
        }
    }
}

__global__ void __launch_bounds__(TPB) k_turb_fill(int n, double v, double* __restrict__ a)
{
    ROW_LOOP(c, n) a[c] = v;
}

/// x_new = std::max(old + relax (x - old), floor), or clamped to [0, 1]
/// (the intermittency, TransitionModel::solveGamma)
__global__ void __launch_bounds__(TPB) k_turb_relax(int n, const double* __restrict__ x, double relax, double floorV,
                                                    int clamp01, double* __restrict__ field)
{
    ROW_LOOP(c, n)
    {
        const double old = field[c];
        const double v = old + relax * (x[c] - old);
        if (clamp01)
        {
            const double lo = v < 0.0 ? 0.0 : v;
            field[c] = lo > 1.0 ? 1.0 : lo;
        }
        else
        {
            field[c] = v < floorV ? floorV : v;
        }
    }
}

/// imposeWallEquilibrium (:288-318): each wall-adjacent cell takes the
/// log-layer k and epsilon of its wall face with the largest k (the first
/// in face order on ties)
__global__ void __launch_bounds__(TPB) k_turb_wall_eq(DMesh m, const int* __restrict__ wallOf,
                                                      const double* __restrict__ uTau,
                                                      const double* __restrict__ wDist, int model, double* k,
                                                      double* eps)
{
    ROW_LOOP(c, m.nC)
    {
        const int sl = c >> 5, lane = c & 31;
        const int e1 = m.cfStart[sl + 1];
        double kEq = 0.0, dEq = 0.0;
        for (int e = m.cfStart[sl] + lane; e < e1; e += 32)
        {
            const int code = m.cfCode[e];
            if (code < 0) break;
            const int f = code >> 1;
            if (f < m.nI) continue;
            const int w = wallOf[f - m.nI];
            if (w < 0 || !(uTau[w] > 0)) continue;
            const double ut = uTau[w];
            double kk, d;
            if (model == TM_SST)
            {
                // KOmegaSST::wallEquilibrium
                kk = ut * ut / sqrt(kBetaStar);
                d = ut / (sqrt(kBetaStar) * kKappa * wDist[w]);
            }
            else
            {
                kk = ut * ut / sqrt(kCmu);
                d = pow(ut, 3.0) / (kKappa * wDist[w]);
            }
            if (!(kk > 0) || !(d > 0)) continue;
            if (kk > kEq)
            {
                kEq = kk;
                dEq = d;
            }
        }
        if (kEq > 0)
        {
            k[c] = kEq;
            eps[c] = dEq;
        }
    }
}

/// nut = max(Cmu k^2 / eps, 0) with the floors (kEpsilon.cpp:83-91)
__global__ void __launch_bounds__(TPB) k_turb_nut(int n, const double* __restrict__ k, const double* __restrict__ eps,
                                                  double* __restrict__ nut)
{
    ROW_LOOP(c, n)
    {
        const double kk = k[c] < kFloor ? kFloor : k[c];
        const double e = eps[c] < kDissFloor ? kDissFloor : eps[c];
        const double v = kCmu * kk * kk / e;
        nut[c] = v < 0.0 ? 0.0 : v;
    }
}

// ---- k-omega SST (kOmegaSST.cpp) -------------------------------------------

__device__ __forceinline__ double dmax(double a, double b) { return a < b ? b : a; }
__device__ __forceinline__ double dmin(double a, double b) { return b < a ? b : a; }

/// F1 (KOmegaSST::f1, Menter 1994 Eq. 10: the outer operator a min)
__device__ double sst_f1(double k, double omega, double y, double nu, double cdKw)
{
    const double kk = dmax(k, kFloor);
    const double w = dmax(omega, kDissFloor);
    const double yy = dmax(y, 1e-12);
    const double cd = dmax(cdKw, 1e-10);
    const double arg = dmin(dmax(sqrt(kk) / (kBetaStar * w * yy), 500.0 * nu / (yy * yy * w)),
                            4.0 * kSigW2 * kk / (cd * yy * yy));
    return tanh(pow(arg, 4.0));
}

/// F2 (KOmegaSST::f2, Menter 1994 Eq. 8)
__device__ double sst_f2(double k, double omega, double y, double nu)
{
    const double kk = dmax(k, kFloor);
    const double w = dmax(omega, kDissFloor);
    const double yy = dmax(y, 1e-12);
    const double arg = dmax(2.0 * sqrt(kk) / (kBetaStar * w * yy), 500.0 * nu / (yy * yy * w));
    return tanh(arg * arg);
}

__device__ __forceinline__ double dot3(const CGrad3& g, int a, int b, int c)
{
    return g.g[a].c[0][c] * g.g[b].c[0][c] + g.g[a].c[1][c] * g.g[b].c[1][c] + g.g[a].c[2][c] * g.g[b].c[2][c];
}

/// The k equation's coefficients (RansModel::solveK with KOmegaSST's
/// kDiffusivity, destructionSp and kProduction): sigma_k = F1 sigmaK1 +
/// (1 - F1) sigmaK2 with F1 of the current k and omega and CD_komega of
/// their gradients (g.g[0] = grad omega, g.g[1] = grad k); gamma = nu + nut
/// sigma_k; Sp = V beta* omega; source V min(P, 10 beta* k omega).
__global__ void __launch_bounds__(TPB) k_sst_k_coefs(int n, const double* __restrict__ V, const double* __restrict__ k,
                                                     const double* __restrict__ w, const double* __restrict__ y,
                                                     CGrad3 g, const double* __restrict__ prod,
                                                     const double* __restrict__ nut, double nu,
                                                     double* __restrict__ sig, double* __restrict__ gamma,
                                                     double* __restrict__ sp, double* __restrict__ src)
{
    ROW_LOOP(c, n)
    {
        const double wg = dmax(w[c], kDissFloor);
        const double cd = dmax(2.0 * kSigW2 / wg * dot3(g, 0, 1, c), 1e-10);
        const double f1 = sst_f1(k[c], w[c], y[c], nu, cd);
        const double s = f1 * kSigK1 + (1.0 - f1) * kSigK2;
        sig[c] = s;
        gamma[c] = nu + nut[c] * s;
        sp[c] = V[c] * kBetaStar * wg;
        const double kk = dmax(k[c], kFloor);
        src[c] = V[c] * dmin(prod[c], kProdLimit * kBetaStar * kk * wg);
    }
}

/// omega production (KOmegaSST::omegaProduction, Menter 2003 consistent form)
__device__ double sst_omega_production(double gamma, double strain, double omega, double f2)
{
    const double s = dmax(strain, 0.0);
    const double w = dmax(omega, kDissFloor);
    const double bradshaw = dmax(kA1 * w, f2 * s);
    const double cap = kProdLimit / kA1 * kBetaStar * w * bradshaw;
    return gamma * dmin(s * s, cap);
}

/// The omega equation's coefficients (KOmegaSST::solveDissipation), with
/// the new k and the current omega: blended sigma_w, gamma_w, beta_w; the
/// production and the signed cross-diffusion as two right-hand-side terms in
/// that order; Sp = V beta_w omega.
__global__ void __launch_bounds__(TPB) k_sst_w_coefs(int n, const double* __restrict__ V, const double* __restrict__ k,
                                                     const double* __restrict__ w, const double* __restrict__ y,
                                                     CGrad3 g, const double* __restrict__ strain,
                                                     const double* __restrict__ nut, double nu,
                                                     double* __restrict__ sig, double* __restrict__ gamma,
                                                     double* __restrict__ sp, double* __restrict__ src,
                                                     double* __restrict__ src2)
{
    ROW_LOOP(c, n)
    {
        const double wOld = w[c];
        const double wg = dmax(wOld, kDissFloor);
        const double gwk = dot3(g, 0, 1, c);
        const double cdKw = dmax(2.0 * kSigW2 / wg * gwk, 1e-10);
        const double f1 = sst_f1(k[c], wOld, y[c], nu, cdKw);
        const double f2 = sst_f2(k[c], wOld, y[c], nu);
        const double sigW = f1 * kSigW1 + (1.0 - f1) * kSigW2;
        const double gamW = f1 * kGamma1 + (1.0 - f1) * kGamma2;
        const double betW = f1 * kBeta1 + (1.0 - f1) * kBeta2;
        sig[c] = sigW;
        gamma[c] = nu + nut[c] * sigW;
        src[c] = V[c] * sst_omega_production(gamW, strain[c], wg, f2);
        const double cd = (1.0 - f1) * 2.0 * kSigW2 / wg * gwk;
        src2[c] = V[c] * cd;
        sp[c] = V[c] * betW * wg;
    }
}

/// nut = a1 k / max(a1 omega, |S| F2) (KOmegaSST::updateNut)
__global__ void __launch_bounds__(TPB) k_sst_nut(int n, const double* __restrict__ k, const double* __restrict__ w,
                                                 const double* __restrict__ y, const double* __restrict__ strain,
                                                 double nu, double* __restrict__ nut)
{
    ROW_LOOP(c, n)
    {
        const double kk = dmax(k[c], kFloor);
        const double ww = dmax(w[c], kDissFloor);
        const double f2 = sst_f2(kk, ww, y[c], nu);
        const double denom = dmax(kA1 * ww, strain[c] * f2);
        nut[c] = dmax(kA1 * kk / denom, 0.0);
    }
}

// ---- DES (desModel.cpp) and gamma transition (transitionModel.cpp) ---------

/// DesModel::updateNut: epsilon replaced by k^1.5 / min(kappa d, C_DES V^1/3)
/// and nut = Cmu k^2 / epsilon
__global__ void __launch_bounds__(TPB) k_des_nut(int n, const double* __restrict__ k, const double* __restrict__ y,
                                                 const double* __restrict__ V, double cDES, double* __restrict__ eps,
                                                 double* __restrict__ nut)
{
    ROW_LOOP(c, n)
    {
        const double delta = cbrt(V[c]);
        const double ell = dmin(kKappa * y[c], cDES * delta);
        const double kk = dmax(k[c], kFloor);
        const double e = dmax(kk * sqrt(kk) / ell, kDissFloor);
        eps[c] = e;
        nut[c] = kCmu * kk * kk / e;
    }
}

/// The intermittency source a(x) (1 - gamma), a = amp tanh((x - x_t)/width):
/// implicit where a > 0, explicit on the old gamma elsewhere
/// (TransitionModel::solveGamma)
__global__ void __launch_bounds__(TPB) k_trans_src(int n, const double* __restrict__ V, const double* __restrict__ cx,
                                                   const double* __restrict__ gam, double amp, double onset,
                                                   double width, double* __restrict__ sp, double* __restrict__ src)
{
    ROW_LOOP(c, n)
    {
        const double a = amp * tanh((cx[c] - onset) / width);
        if (a > 0)
        {
            sp[c] = V[c] * a;
            src[c] = V[c] * a;
        }
        else
        {
            sp[c] = 0.0;
            src[c] = V[c] * a * (1.0 - gam[c]);
        }
    }
}

/// nut *= gamma (TransitionModel::updateNut)
__global__ void __launch_bounds__(TPB) k_trans_nut(int n, const double* __restrict__ gam, double* __restrict__ nut)
{
    ROW_LOOP(c, n) nut[c] *= gam[c];
}

}  // namespace

struct TurbState
{
    bool on = false;
    int model = TM_KEPS;
    double nu = 0, intensity = 0.05, lengthScale = -1, relaxation = 0.7;
    double cDES = 0.61;                          // des
    double onsetX = 0, width = 0, rate = 4.0;    // gammaTransition
    double* y = nullptr;                         // cell wall distance (SST, DES)
    double *sig = nullptr, *src2 = nullptr;      // SST: per-cell sigma, second source
    double *gam = nullptr, *gc = nullptr, *gk = nullptr, *cx = nullptr;  // transition: gamma, its BC, cell x
    int nW = 0;
    int *wFace = nullptr, *wCell = nullptr, *wallOf = nullptr;
    double *wDist = nullptr, *uTau = nullptr, *yPlus = nullptr, *nutWall = nullptr;
    double *k = nullptr, *eps = nullptr, *nut = nullptr, *strain = nullptr, *prod = nullptr;
    double *gammaC = nullptr, *gammaF = nullptr, *sp = nullptr, *src = nullptr;
    double *kc = nullptr, *kk = nullptr, *ec = nullptr, *ek = nullptr;
    double *dP = nullptr, *dN = nullptr;
};

void TurbDeleter::operator()(TurbState* t) const { delete t; }

namespace
{

/// RansModel::cellWallDistance (turbulenceModel.cpp:405-468): Dijkstra over
/// the cell graph from the wall-adjacent cells, each seeded with the normal
/// distance of its nearest wall face, a face crossing costing the
/// owner-neighbour centre distance, with the reference's 1e-12 relative
/// bands on stale entries and on improvements.  Cells out of reach take the
/// largest distance reached (the box diagonal when there are no walls).
/// Pops come in (distance, cell) order, so the result does not depend on
/// the order faces are visited.  Original cell order.
std::vector<double> cellWallDistance(const Mesh& M, const std::vector<int64_t>& wallFaces,
                                     const std::vector<double>& wDist)
{
    const int64_t nC = M.nCells, nI = M.nInternal();
    std::vector<double> dist(static_cast<size_t>(nC), -1.0);
    for (size_t i = 0; i < wallFaces.size(); ++i)
    {
        const size_t o = static_cast<size_t>(M.owner[static_cast<size_t>(wallFaces[i])]);
        if (dist[o] < 0 || wDist[i] < dist[o]) dist[o] = wDist[i];
    }
    std::vector<int64_t> start(static_cast<size_t>(nC) + 1, 0), adj(2 * static_cast<size_t>(nI));
    for (int64_t f = 0; f < nI; ++f)
    {
        ++start[static_cast<size_t>(M.owner[static_cast<size_t>(f)]) + 1];
        ++start[static_cast<size_t>(M.neighbour[static_cast<size_t>(f)]) + 1];
    }
    for (int64_t c = 0; c < nC; ++c) start[c + 1] += start[c];
    {
        std::vector<int64_t> fill(start.begin(), start.end() - 1);
        for (int64_t f = 0; f < nI; ++f)
        {
            adj[static_cast<size_t>(fill[static_cast<size_t>(M.owner[static_cast<size_t>(f)])]++)] = f;
            adj[static_cast<size_t>(fill[static_cast<size_t>(M.neighbour[static_cast<size_t>(f)])]++)] = f;
        }
    }
    using Node = std::pair<double, int64_t>;
    std::priority_queue<Node, std::vector<Node>, std::greater<Node>> pq;
    for (int64_t c = 0; c < nC; ++c)
        if (dist[static_cast<size_t>(c)] >= 0) pq.push({dist[static_cast<size_t>(c)], c});
    while (!pq.empty())
    {
        const Node top = pq.top();
        pq.pop();
        const double d = top.first;
        const int64_t c = top.second;
        if (d > dist[static_cast<size_t>(c)] + 1e-12 * (d + 1.0)) continue;
        for (int64_t e = start[static_cast<size_t>(c)]; e < start[static_cast<size_t>(c) + 1]; ++e)
        {
            const size_t f = static_cast<size_t>(adj[static_cast<size_t>(e)]);
            const int64_t o = M.owner[f];
            const int64_t n = o == c ? M.neighbour[f] : o;
            const Vec& dv = M.d[f];
            const double nd = d + std::sqrt(dv.x * dv.x + dv.y * dv.y + dv.z * dv.z);
            double& dn = dist[static_cast<size_t>(n)];
            if (dn < 0 || nd < dn - 1e-12 * (nd + 1.0))
            {
                dn = nd;
                pq.push({nd, n});
            }
        }
    }
    double reached = 0;
    for (const double v : dist) reached = std::max(reached, v);
    if (reached <= 0)
    {
        Vec lo = M.points[0], hi = M.points[0];
        for (const Vec& p : M.points)
        {
            lo = Vec{std::min(lo.x, p.x), std::min(lo.y, p.y), std::min(lo.z, p.z)};
            hi = Vec{std::max(hi.x, p.x), std::max(hi.y, p.y), std::max(hi.z, p.z)};
        }
        const Vec dd{hi.x - lo.x, hi.y - lo.y, hi.z - lo.z};
        reached = std::sqrt(dd.x * dd.x + dd.y * dd.y + dd.z * dd.z);
    }
    for (double& v : dist)
        if (v < 0) v = reached;
    return dist;
}

int modelOf(const std::string& model)
{
    if (model == "kEpsilon") return TM_KEPS;
    if (model == "kOmegaSST") return TM_SST;
    if (model == "des") return TM_DES;
    if (model == "gammaTransition") return TM_TRANSITION;
    return -1;
}

}  // namespace

std::string Ctx::turbulenceModelName() const
{
    if (!turb_) return "laminar";
    static const char* const names[4] = {"kEpsilon", "kOmegaSST", "des", "gammaTransition"};
    return names[turb_->model];
}

void Ctx::turbulenceParams(double cDES, double reOnset, double onsetWidth, double gammaRate)
{
    turbCDES_ = cDES;
    turbReOnset_ = reOnset;
    turbOnsetWidth_ = onsetWidth;
    turbGammaRate_ = gammaRate;
}

/// uReference (turbulenceModel.cpp:148-160): the largest fixed inlet
/// velocity, else the largest cell velocity
double Ctx::turbURef()
{
    const Mesh& M = mesh_;
    double uRef = 0;
    for (size_t pi = 0; pi < M.patches.size(); ++pi)
    {
        if (M.patches[pi].type != "inlet" || uType_[pi] != CFG_BC_FIXED_VALUE) continue;
        const Vec& v = uVal_[pi];
        uRef = std::max(uRef, std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z));
    }
    if (uRef > 0) return uRef;
    const int nC = dm_.nC;
    std::vector<double> U(3 * static_cast<size_t>(nC));
    download(U.data(), nullptr, nullptr);
    for (int c = 0; c < nC; ++c)
        uRef = std::max(uRef, std::sqrt(U[3 * c] * U[3 * c] + U[3 * c + 1] * U[3 * c + 1] + U[3 * c + 2] * U[3 * c + 2]));
    return uRef;
}

void Ctx::turbulenceSetup(const std::string& model, double intensity, double lengthScale, double relaxation,
                          double nu)
{
    CFG_CUDA(cudaSetDevice(device_));
    if (model == "laminar")
    {
        turb_.reset();
        lastNu_ = NAN;  // the momentum diffusivity goes back to the molecular one
        return;
    }
    const int tm = modelOf(model);
    if (tm < 0)
        fail(CFG_ESETUP, "turbulence: model '" + model +
                             "' is not on the GPU path (laminar | kEpsilon | kOmegaSST | des | gammaTransition)");
    if (!(intensity >= 0)) fail(CFG_ESETUP, "turbulence: intensity must be non-negative");
    if (!(relaxation > 0 && relaxation <= 1)) fail(CFG_ESETUP, "turbulence: relaxation must be in (0, 1]");
    if (!(nu > 0)) fail(CFG_ESETUP, "turbulence: molecular viscosity must be positive");
    if (tm == TM_DES && !(turbCDES_ > 0)) fail(CFG_ESETUP, "des: C_DES must be positive");
    if (tm == TM_TRANSITION && !(turbReOnset_ > 0))
        fail(CFG_ESETUP, "gammaTransition: turbulence{ reOnset } must be a positive Re threshold");
    if (tm == TM_TRANSITION && !(turbGammaRate_ > 0)) fail(CFG_ESETUP, "gammaTransition: gammaRate must be positive");
    const Mesh& M = mesh_;
    const int nC = dm_.nC, nF = dm_.nF, nI = dm_.nI, nB = dm_.nB;
    std::unique_ptr<TurbState> t(new TurbState());
    t->on = true;
    t->model = tm;
    t->nu = nu;
    t->intensity = intensity;
    t->lengthScale = lengthScale;
    t->relaxation = relaxation;
    t->cDES = turbCDES_;
    t->rate = turbGammaRate_;
    // wall faces, patch by patch, with the owner's normal distance (:131-146)
    std::vector<int> wFace, wCell, wallOf(static_cast<size_t>(std::max(nB, 1)), -1);
    std::vector<int64_t> wFaceOrig;
    std::vector<double> wDist;
    std::vector<double> kc(nB), kk(nB, 0.0), ec(nB), ek(nB, 0.0), gc(nB), gk(nB, 0.0);
    for (const auto& p : M.patches)
    {
        const bool wall = p.type == "wall", inlet = p.type == "inlet";
        for (int64_t f = p.start; f < p.start + p.size; ++f)
        {
            const int b = static_cast<int>(f - nI);
            // k: fixedValue on inlets, zeroGradient elsewhere; the
            // dissipation variable: fixedValue on walls and inlets (RansModel
            // ctor, :122-128); the intermittency fixed (0) on inlets only
            // (TransitionModel ctor)
            kc[b] = inlet ? 0.0 : 1.0;
            ec[b] = (wall || inlet) ? 0.0 : 1.0;
            gc[b] = inlet ? 0.0 : 1.0;
            if (!wall) continue;
            const Vec& sf = M.Sf[static_cast<size_t>(f)];
            const double a = std::sqrt(sf.x * sf.x + sf.y * sf.y + sf.z * sf.z);
            if (a <= 0) fail(CFG_EMESH, "turbulence: zero-area wall face");
            const Vec& d = M.d[static_cast<size_t>(f)];
            const double y = d.x * (sf.x / a) + d.y * (sf.y / a) + d.z * (sf.z / a);
            if (!(y > 0)) fail(CFG_EMESH, "turbulence: wall face not outside its owner cell");
            wallOf[b] = static_cast<int>(wFace.size());
            wFace.push_back(static_cast<int>(f));
            wFaceOrig.push_back(f);
            wCell.push_back(inv_[static_cast<size_t>(M.owner[static_cast<size_t>(f)])]);
            wDist.push_back(y);
        }
    }
    t->nW = static_cast<int>(wFace.size());
    // the initial state (initializeFields of the model, RansModel::initializeUniform)
    const double uRef = turbURef();
    double L = lengthScale;
    if (!(L > 0))
    {
        Vec lo = M.points[0], hi = M.points[0];
        for (const Vec& p : M.points)
        {
            lo = Vec{std::min(lo.x, p.x), std::min(lo.y, p.y), std::min(lo.z, p.z)};
            hi = Vec{std::max(hi.x, p.x), std::max(hi.y, p.y), std::max(hi.z, p.z)};
        }
        const Vec d{hi.x - lo.x, hi.y - lo.y, hi.z - lo.z};
        L = 0.07 * std::sqrt(d.x * d.x + d.y * d.y + d.z * d.z);
    }
    double k0 = 1.5 * std::pow(uRef * intensity, 2);
    double e0;
    if (tm == TM_SST)
        e0 = std::sqrt(std::max(k0, kFloor)) / (std::pow(kCmu, 0.25) * L);  // omega = k^1/2 / (Cmu^1/4 L)
    else
        e0 = std::pow(kCmu, 0.25) * std::pow(std::max(k0, kFloor), 1.5) / L;
    k0 = std::max(k0, kFloor);
    e0 = std::max(e0, kDissFloor);
    for (const auto& p : M.patches)
        if (p.type == "inlet")
            for (int64_t f = p.start; f < p.start + p.size; ++f)
            {
                kk[static_cast<size_t>(f - nI)] = k0;
                ek[static_cast<size_t>(f - nI)] = e0;
            }
    if (tm == TM_TRANSITION)
    {
        // x_t = nu Re_crit / U_ref and the onset width (TransitionModel::initializeFields)
        if (!(uRef > 0)) fail(CFG_ESETUP, "gammaTransition: no velocity scale to place the onset");
        t->onsetX = nu * turbReOnset_ / uRef;
        t->width = turbOnsetWidth_ > 0 ? turbOnsetWidth_ : 0.05 * t->onsetX;
    }
    // face distances of the harmonic interpolation (laplacianScheme.cpp:47-51)
    std::vector<double> dP(static_cast<size_t>(nF), 0.0), dN(static_cast<size_t>(nF), 0.0);
    for (int f = 0; f < nI; ++f)
    {
        const Vec& cP = M.C[static_cast<size_t>(M.owner[f])];
        const Vec& cN = M.C[static_cast<size_t>(M.neighbour[f])];
        const Vec& cf = M.Cf[static_cast<size_t>(f)];
        const Vec a{cf.x - cP.x, cf.y - cP.y, cf.z - cP.z}, b{cN.x - cf.x, cN.y - cf.y, cN.z - cf.z};
        dP[f] = std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z);
        dN[f] = std::sqrt(b.x * b.x + b.y * b.y + b.z * b.z);
    }
    t->wFace = upload(wFace);
    t->wCell = upload(wCell);
    t->wallOf = upload(wallOf);
    t->wDist = upload(wDist);
    t->dP = upload(dP);
    t->dN = upload(dN);
    t->kc = upload(kc);
    t->kk = upload(kk);
    t->ec = upload(ec);
    t->ek = upload(ek);
    if (tm == TM_SST || tm == TM_DES)
    {
        const std::vector<double> y = cellWallDistance(M, wFaceOrig, wDist);
        std::vector<double> yd(static_cast<size_t>(nC));
        for (int c = 0; c < nC; ++c) yd[c] = y[static_cast<size_t>(perm_[c])];
        t->y = upload(yd);
    }
    if (tm == TM_SST)
    {
        t->sig = alloc<double>(nC);
        t->src2 = alloc<double>(nC);
    }
    if (tm == TM_TRANSITION)
    {
        std::vector<double> cx(static_cast<size_t>(nC));
        for (int c = 0; c < nC; ++c) cx[c] = M.C[static_cast<size_t>(perm_[c])].x;
        t->cx = upload(cx);
        t->gc = upload(gc);
        t->gk = upload(gk);
        t->gam = alloc<double>(nC);  // zero
    }
    t->uTau = alloc<double>(std::max(t->nW, 1));
    t->yPlus = alloc<double>(std::max(t->nW, 1));
    t->nutWall = alloc<double>(std::max(t->nW, 1));
    CFG_CUDA(cudaMemsetAsync(t->nutWall, 0, std::max(t->nW, 1) * sizeof(double), stream_));
    CFG_CUDA(cudaMemsetAsync(t->uTau, 0, std::max(t->nW, 1) * sizeof(double), stream_));
    CFG_CUDA(cudaMemsetAsync(t->yPlus, 0, std::max(t->nW, 1) * sizeof(double), stream_));
    for (double** a : {&t->k, &t->eps, &t->nut, &t->strain, &t->prod, &t->gammaC, &t->sp, &t->src})
        *a = alloc<double>(nC);
    t->gammaF = alloc<double>(nF);
    k_turb_fill<<<G_, TPB, 0, stream_>>>(nC, k0, t->k);
    k_turb_fill<<<G_, TPB, 0, stream_>>>(nC, e0, t->eps);
    CFG_CUDA(cudaMemsetAsync(t->strain, 0, nC * sizeof(double), stream_));
    CFG_CUDA(cudaMemsetAsync(t->prod, 0, nC * sizeof(double), stream_));
    launchCheck("turb_init", 2);
    turb_.reset(t.release());
    turbRefreshNut();
    CFG_CUDA(cudaStreamSynchronize(stream_));
}

/// updateNut of the model + refreshFaceNut: nut, then the momentum
/// diffusivity on faces
void Ctx::turbRefreshNut()
{
    TurbState& t = *turb_;
    const int nC = dm_.nC;
    switch (t.model)
    {
    case TM_SST: k_sst_nut<<<G_, TPB, 0, stream_>>>(nC, t.k, t.eps, t.y, t.strain, t.nu, t.nut); break;
    case TM_DES: k_des_nut<<<G_, TPB, 0, stream_>>>(nC, t.k, t.y, dm_.V, t.cDES, t.eps, t.nut); break;
    default:
        k_turb_nut<<<G_, TPB, 0, stream_>>>(nC, t.k, t.eps, t.nut);
        if (t.model == TM_TRANSITION) k_trans_nut<<<G_, TPB, 0, stream_>>>(nC, t.gam, t.nut);
    }
    k_turb_face_gamma<<<GF_, TPB, 0, stream_>>>(dm_, t.dP, t.dN, t.nut, t.wallOf, t.nutWall, 0.0, 1.0, nullptr, t.nu,
                                               gU_);
    launchCheck("turb_nut", 2);
    lastNu_ = NAN;  // gU_ now holds nu + nutFace
}

/// One scalar equation of the model, solved and relaxed into `field`:
/// div(phi,T) - laplacianFace(diffusionFace(gamma, sigma), T) + Sp T = src
/// (+ src2), with gamma = nu + nut sigma from a constant sigma, or gamma and
/// a per-cell sigma already in t.gammaC / sigCell; the wall faces take
/// nu + nutWall sigma[owner] unless `wallOverride` is off (the plain
/// harmonic face gamma of the intermittency).
void Ctx::turbSolveScalar(const double* bc, const double* bk, const double* sigCell, double sigma, bool wallOverride,
                          const double* src2, double* field, double floorV, bool clamp01, double dt, int64_t& inner)
{
    TurbState& t = *turb_;
    const int nC = dm_.nC;
    const double alpha = schemes_.div == CFG_DIV_BLEND ? schemes_.blend_coeff : (schemes_.div == CFG_DIV_LINEAR ? 1.0 : 0.0);
    if (!sigCell)
    {
        k_turb_gamma<<<G_, TPB, 0, stream_>>>(nC, t.nu, t.nut, sigma, t.gammaC);
        launchCheck("turb_gamma");
    }
    k_turb_face_gamma<<<GF_, TPB, 0, stream_>>>(dm_, t.dP, t.dN, t.gammaC, wallOverride ? t.wallOf : nullptr,
                                               t.nutWall, t.nu, sigma, sigCell, 0.0, t.gammaF);
    launchCheck("turb_face_gamma");
    double* x = ux_.c[0];
    double* base = uBase_.c[0];
    double* rhs = uRhs_.c[0];
    // the old field of a time step is the field itself: it changes only at
    // the relaxation below
    k_assemble_S<<<G_, TPB, 0, stream_>>>(dm_, phi_, t.gammaF, bc, bk, alpha, t.sp, t.src, src2, dt, field, mVal_,
                                         uDiag_, base);
    launchCheck("turb_assemble");
    CFG_CUDA(cudaMemsetAsync(x, 0, nC * sizeof(double), stream_));
    const bool corr = schemes_.laplacian_corrected != 0;
    const int passes = corr ? kNonOrth + 1 : 1;
    const BcTab tb{{bc, bc, bc}, {bk, bk, bk}};
    for (int pass = 0; pass < passes; ++pass)
    {
        if (corr)
        {
            const double* xs[1] = {x};
            V3P g[1] = {gA_};
            gradCells(xs, 1, tb, schemes_.grad, false, g);
            k_corrector<1><<<G_, TPB, 0, stream_>>>(dm_, t.gammaF, CGrad3{{cv(gA_)}}, CV3P{{base, base, base}},
                                                   V3P{{rhs, rhs, rhs}});
            launchCheck("turb_corrector");
        }
        else
        {
            CFG_CUDA(cudaMemcpyAsync(rhs, base, nC * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
        }
        cfg_solver_report rep[3];
        runBiCG3(mVal_, uDiag_, V3P{{rhs, rhs, rhs}}, V3P{{x, x, x}}, 1, kLinTol, kLinMaxIter, rep);
        inner += rep[0].iterations;
    }
    k_turb_relax<<<G_, TPB, 0, stream_>>>(nC, x, t.relaxation, floorV, clamp01 ? 1 : 0, field);
    launchCheck("turb_relax");
}

/// RansModel::correctTurbulence(dt) for the model in hand (dt = 0 in
/// SIMPLE, the step's dt in PISO, pisoSolver.cpp:29).
void Ctx::turbCorrect(int64_t& inner, double dt)
{
    TurbState& t = *turb_;
    const int nC = dm_.nC;
    const BcTab ub{{uc_[0], uc_[1], uc_[2]}, {uk_[0], uk_[1], uk_[2]}};
    // strain rate from the U-component gradients (makeFaceValueFn faces)
    {
        const double* xs[3] = {U_.c[0], U_.c[1], U_.c[2]};
        V3P g[3] = {gA_, gB_, Hf_};
        gradCells(xs, 3, ub, schemes_.grad, false, g);
        k_turb_strain<<<G_, TPB, 0, stream_>>>(nC, CGrad3{{cv(gA_), cv(gB_), cv(Hf_)}}, t.nut, t.strain, t.prod);
        launchCheck("turb_strain");
    }
    if (t.nW > 0)
    {
        k_turb_wall<<<std::max(1, (t.nW + TPB - 1) / TPB), TPB, 0, stream_>>>(
            t.nW, t.wFace, t.wCell, t.wDist, dm_, cv(U_), t.nu, t.model, t.uTau, t.yPlus, t.nutWall, t.ec, t.ek);
        launchCheck("turb_wall");
    }
    if (t.model == TM_SST)
    {
        // fvc::grad of omega and of k (the volScalarField overload, each
        // with its own conditions; one field per call, gB_ being the
        // single-field scratch) into gA_ and Hf_
        auto gradWK = [&] {
            const double* xw[1] = {t.eps};
            const double* xk[1] = {t.k};
            const BcTab tw{{t.ec, t.ec, t.ec}, {t.ek, t.ek, t.ek}};
            const BcTab tk{{t.kc, t.kc, t.kc}, {t.kk, t.kk, t.kk}};
            V3P gw[1] = {gA_};
            V3P gk[1] = {Hf_};
            gradCells(xw, 1, tw, schemes_.grad, true, gw);
            gradCells(xk, 1, tk, schemes_.grad, true, gk);
        };
        gradWK();
        k_sst_k_coefs<<<G_, TPB, 0, stream_>>>(nC, dm_.V, t.k, t.eps, t.y, CGrad3{{cv(gA_), cv(Hf_), cv(Hf_)}},
                                               t.prod, t.nut, t.nu, t.sig, t.gammaC, t.sp, t.src);
        launchCheck("sst_k_coefs");
        turbSolveScalar(t.kc, t.kk, t.sig, 0.0, true, nullptr, t.k, kFloor, false, dt, inner);
        gradWK();  // with the new k
        k_sst_w_coefs<<<G_, TPB, 0, stream_>>>(nC, dm_.V, t.k, t.eps, t.y, CGrad3{{cv(gA_), cv(Hf_), cv(Hf_)}},
                                               t.strain, t.nut, t.nu, t.sig, t.gammaC, t.sp, t.src, t.src2);
        launchCheck("sst_w_coefs");
        turbSolveScalar(t.ec, t.ek, t.sig, 0.0, true, t.src2, t.eps, kDissFloor, false, dt, inner);
    }
    else
    {
        // k
        k_turb_src_k<<<G_, TPB, 0, stream_>>>(nC, dm_.V, t.k, t.eps, t.prod, t.sp, t.src);
        launchCheck("turb_src_k");
        turbSolveScalar(t.kc, t.kk, nullptr, 1.0 / kSigmaK, true, nullptr, t.k, kFloor, false, dt, inner);
        // epsilon, with the new k
        k_turb_src_e<<<G_, TPB, 0, stream_>>>(nC, dm_.V, t.k, t.eps, t.prod, t.sp, t.src);
        launchCheck("turb_src_e");
        turbSolveScalar(t.ec, t.ek, nullptr, 1.0 / kSigmaE, true, nullptr, t.eps, kDissFloor, false, dt, inner);
        if (t.model == TM_TRANSITION)
        {
            // the intermittency (TransitionModel::solveGamma): sigma 1, the
            // plain harmonic face gamma, clamped to [0, 1]
            const double amp = t.rate * turbURef() / t.onsetX;
            k_trans_src<<<G_, TPB, 0, stream_>>>(nC, dm_.V, t.cx, t.gam, amp, t.onsetX, t.width, t.sp, t.src);
            launchCheck("trans_src");
            turbSolveScalar(t.gc, t.gk, nullptr, 1.0, false, nullptr, t.gam, 0.0, true, dt, inner);
        }
    }
    if (t.nW > 0)
    {
        k_turb_wall_eq<<<G_, TPB, 0, stream_>>>(dm_, t.wallOf, t.uTau, t.wDist, t.model, t.k, t.eps);
        launchCheck("turb_wall_eq");
    }
    turbRefreshNut();
}

/// k, the dissipation variable, nut and (gammaTransition) the intermittency
/// to (save) or from a device buffer of 4 nCells
void Ctx::turbCopy(double* buf, bool save)
{
    TurbState& t = *turb_;
    const size_t n = static_cast<size_t>(dm_.nC);
    double* f[4] = {t.k, t.eps, t.nut, t.gam};
    for (int i = 0; i < 4; ++i)
        if (f[i])
            CFG_CUDA(cudaMemcpyAsync(save ? buf + i * n : f[i], save ? f[i] : buf + i * n, n * sizeof(double),
                                     cudaMemcpyDeviceToDevice, stream_));
}

void Ctx::turbulenceFields(double* k, double* eps, double* nut, double* nuEffFace)
{
    if (!turb_) fail(CFG_EINVAL, "cfg_turbulence_fields: no turbulence model set up");
    CFG_CUDA(cudaSetDevice(device_));
    if (k) fromDevCells(k, turb_->k, 1, 0);
    if (eps) fromDevCells(eps, turb_->eps, 1, 0);
    if (nut) fromDevCells(nut, turb_->nut, 1, 0);
    if (nuEffFace)
    {
        CFG_CUDA(cudaMemcpyAsync(nuEffFace, gU_, dm_.nF * sizeof(double), cudaMemcpyDeviceToHost, stream_));
        CFG_CUDA(cudaStreamSynchronize(stream_));
    }
}

}  // namespace cfg
