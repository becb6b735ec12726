// The standard k-epsilon RANS model with Spalding wall functions, on the
// device, as the reference's RansModel / KEpsilon advance it once per SIMPLE
// outer iteration (src/3d/src/turbulence/turbulenceModel.cpp,
// kEpsilon.cpp, wallFunction.cpp; called from simpleSolver.cpp:52 and fed
// to the momentum laplacian as nuEffFace, simpleSolver.cpp:97).
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
#include <cmath>
#include <cstring>

#include "ctx.h"
#include "kernels.cuh"

namespace cfg
{

namespace
{

constexpr double kCmu = 0.09, kC1 = 1.44, kC2 = 1.92, kSigmaK = 1.0, kSigmaE = 1.3;
constexpr double kKappa = 0.41, kSpaldingC = 5.5676;
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
                                                   double* uTau, double* yPlus, double* nutWall, double* ec,
                                                   double* ek)
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
        const double e = pow(ut, 3.0) / (kKappa * wDist[i]);
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
                                                         double wallBase, double wallSigma, double add,
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
            const int w = wallOf[f - m.nI];
            if (w >= 0) g = wallBase + nutWall[w] * wallSigma;
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

/// a scalar transport equation div(phi,T) - laplacianFace(gamma,T) + Sp T =
/// src, in the reference's term order per cell (fvm::div, laplacianFace,
/// then the source and the implicit Sp)
__global__ void __launch_bounds__(TPB) k_assemble_S(DMesh m, const double* __restrict__ phi,
                                                    const double* __restrict__ gamma, const double* __restrict__ bc,
                                                    const double* __restrict__ bk, double alpha,
                                                    const double* __restrict__ sp, const double* __restrict__ src,
                                                    double* __restrict__ val, double* __restrict__ diagOut,
                                                    double* __restrict__ base)
{
    ROW_LOOP(c, m.nC)
    {
        const int sl = c >> 5, lane = c & 31;
        const int e0 = m.cfStart[sl] + lane, e1 = m.cfStart[sl + 1];
        double diag = 0.0, r = 0.0;
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
        // the implicit source on the diagonal, the explicit one on the
        // right-hand side, each after the face terms
        diag += sp[c];
        r += src[c];
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

/// x_new = std::max(old + relax (x - old), floor)
__global__ void __launch_bounds__(TPB) k_turb_relax(int n, const double* __restrict__ x, double relax, double floorV,
                                                    double* __restrict__ field)
{
    ROW_LOOP(c, n)
    {
        const double old = field[c];
        const double v = old + relax * (x[c] - old);
        field[c] = v < floorV ? floorV : v;
    }
}

/// imposeWallEquilibrium (:288-318): each wall-adjacent cell takes the
/// log-layer k and epsilon of its wall face with the largest k (the first
/// in face order on ties)
__global__ void __launch_bounds__(TPB) k_turb_wall_eq(DMesh m, const int* __restrict__ wallOf,
                                                      const double* __restrict__ uTau,
                                                      const double* __restrict__ wDist, double* k, double* eps)
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
            const double kk = ut * ut / sqrt(kCmu);
            const double d = pow(ut, 3.0) / (kKappa * wDist[w]);
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

}  // namespace

struct TurbState
{
    bool on = false;
    double nu = 0, intensity = 0.05, lengthScale = -1, relaxation = 0.7;
    int nW = 0;
    int *wFace = nullptr, *wCell = nullptr, *wallOf = nullptr;
    double *wDist = nullptr, *uTau = nullptr, *yPlus = nullptr, *nutWall = nullptr;
    double *k = nullptr, *eps = nullptr, *nut = nullptr, *strain = nullptr, *prod = nullptr;
    double *gammaC = nullptr, *gammaF = nullptr, *sp = nullptr, *src = nullptr;
    double *kc = nullptr, *kk = nullptr, *ec = nullptr, *ek = nullptr;
    double *dP = nullptr, *dN = nullptr;
};

void TurbDeleter::operator()(TurbState* t) const { delete t; }

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
    if (model != "kEpsilon") fail(CFG_ESETUP, "turbulence: model '" + model + "' is not on the GPU path (laminar | kEpsilon)");
    if (!(intensity >= 0)) fail(CFG_ESETUP, "turbulence: intensity must be non-negative");
    if (!(relaxation > 0 && relaxation <= 1)) fail(CFG_ESETUP, "turbulence: relaxation must be in (0, 1]");
    if (!(nu > 0)) fail(CFG_ESETUP, "turbulence: molecular viscosity must be positive");
    const Mesh& M = mesh_;
    const int nC = dm_.nC, nF = dm_.nF, nI = dm_.nI, nB = dm_.nB;
    std::unique_ptr<TurbState> t(new TurbState());
    t->on = true;
    t->nu = nu;
    t->intensity = intensity;
    t->lengthScale = lengthScale;
    t->relaxation = relaxation;
    // wall faces, patch by patch, with the owner's normal distance (:131-146)
    std::vector<int> wFace, wCell, wallOf(static_cast<size_t>(std::max(nB, 1)), -1);
    std::vector<double> wDist;
    std::vector<double> kc(nB), kk(nB, 0.0), ec(nB), ek(nB, 0.0);
    for (const auto& p : M.patches)
    {
        const bool wall = p.type == "wall", inlet = p.type == "inlet";
        for (int64_t f = p.start; f < p.start + p.size; ++f)
        {
            const int b = static_cast<int>(f - nI);
            // k: fixedValue on inlets, zeroGradient elsewhere; epsilon:
            // fixedValue on walls and inlets (RansModel ctor, :122-128)
            kc[b] = inlet ? 0.0 : 1.0;
            ec[b] = (wall || inlet) ? 0.0 : 1.0;
            if (!wall) continue;
            const Vec& sf = M.Sf[static_cast<size_t>(f)];
            const double a = std::sqrt(sf.x * sf.x + sf.y * sf.y + sf.z * sf.z);
            if (a <= 0) fail(CFG_EMESH, "turbulence: zero-area wall face");
            const Vec& d = M.d[static_cast<size_t>(f)];
            const double y = d.x * (sf.x / a) + d.y * (sf.y / a) + d.z * (sf.z / a);
            if (!(y > 0)) fail(CFG_EMESH, "turbulence: wall face not outside its owner cell");
            wallOf[b] = static_cast<int>(wFace.size());
            wFace.push_back(static_cast<int>(f));
            wCell.push_back(inv_[static_cast<size_t>(M.owner[static_cast<size_t>(f)])]);
            wDist.push_back(y);
        }
    }
    t->nW = static_cast<int>(wFace.size());
    // the initial state (KEpsilon::initializeFields, RansModel::initializeUniform)
    double uRef = 0;
    for (size_t pi = 0; pi < M.patches.size(); ++pi)
    {
        if (M.patches[pi].type != "inlet" || uType_[pi] != CFG_BC_FIXED_VALUE) continue;
        const Vec& v = uVal_[pi];
        uRef = std::max(uRef, std::sqrt(v.x * v.x + v.y * v.y + v.z * v.z));
    }
    if (!(uRef > 0))
    {
        std::vector<double> U(3 * static_cast<size_t>(nC));
        download(U.data(), nullptr, nullptr);
        for (int c = 0; c < nC; ++c)
            uRef = std::max(uRef, std::sqrt(U[3 * c] * U[3 * c] + U[3 * c + 1] * U[3 * c + 1] + U[3 * c + 2] * U[3 * c + 2]));
    }
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
    double e0 = std::pow(kCmu, 0.25) * std::pow(std::max(k0, kFloor), 1.5) / L;
    k0 = std::max(k0, kFloor);
    e0 = std::max(e0, kDissFloor);
    for (const auto& p : M.patches)
        if (p.type == "inlet")
            for (int64_t f = p.start; f < p.start + p.size; ++f)
            {
                kk[static_cast<size_t>(f - nI)] = k0;
                ek[static_cast<size_t>(f - nI)] = e0;
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

/// updateNut + refreshFaceNut: nut, then the momentum diffusivity on faces
void Ctx::turbRefreshNut()
{
    TurbState& t = *turb_;
    k_turb_nut<<<G_, TPB, 0, stream_>>>(dm_.nC, t.k, t.eps, t.nut);
    k_turb_face_gamma<<<GF_, TPB, 0, stream_>>>(dm_, t.dP, t.dN, t.nut, t.wallOf, t.nutWall, 0.0, 1.0, t.nu, gU_);
    launchCheck("turb_nut", 2);
    lastNu_ = NAN;  // gU_ now holds nu + nutFace
}

/// One scalar equation of the model, solved and relaxed into `field`.
void Ctx::turbSolveScalar(double sigma, bool isK, double* field, double floorV, int64_t& inner)
{
    TurbState& t = *turb_;
    const int nC = dm_.nC;
    const double alpha = schemes_.div == CFG_DIV_BLEND ? schemes_.blend_coeff : (schemes_.div == CFG_DIV_LINEAR ? 1.0 : 0.0);
    const double* bc = isK ? t.kc : t.ec;
    const double* bk = isK ? t.kk : t.ek;
    // diffusionFace(nu + nut sigma, sigma)
    k_turb_gamma<<<G_, TPB, 0, stream_>>>(nC, t.nu, t.nut, sigma, t.gammaC);
    k_turb_face_gamma<<<GF_, TPB, 0, stream_>>>(dm_, t.dP, t.dN, t.gammaC, t.wallOf, t.nutWall, t.nu, sigma, 0.0,
                                               t.gammaF);
    launchCheck("turb_gamma", 2);
    double* x = ux_.c[0];
    double* base = uBase_.c[0];
    double* rhs = uRhs_.c[0];
    k_assemble_S<<<G_, TPB, 0, stream_>>>(dm_, phi_, t.gammaF, bc, bk, alpha, t.sp, t.src, mVal_, uDiag_, base);
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
    k_turb_relax<<<G_, TPB, 0, stream_>>>(nC, x, t.relaxation, floorV, field);
    launchCheck("turb_relax");
}

void Ctx::turbCorrect(int64_t& inner)
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
            t.nW, t.wFace, t.wCell, t.wDist, dm_, cv(U_), t.nu, t.uTau, t.yPlus, t.nutWall, t.ec, t.ek);
        launchCheck("turb_wall");
    }
    // k
    k_turb_src_k<<<G_, TPB, 0, stream_>>>(nC, dm_.V, t.k, t.eps, t.prod, t.sp, t.src);
    launchCheck("turb_src_k");
    turbSolveScalar(1.0 / kSigmaK, true, t.k, kFloor, inner);
    // epsilon, with the new k
    k_turb_src_e<<<G_, TPB, 0, stream_>>>(nC, dm_.V, t.k, t.eps, t.prod, t.sp, t.src);
    launchCheck("turb_src_e");
    turbSolveScalar(1.0 / kSigmaE, false, t.eps, kDissFloor, inner);
    if (t.nW > 0)
    {
        k_turb_wall_eq<<<G_, TPB, 0, stream_>>>(dm_, t.wallOf, t.uTau, t.wDist, t.k, t.eps);
        launchCheck("turb_wall_eq");
    }
    turbRefreshNut();
}

/// k, epsilon and nut to (save) or from a device buffer of 3 nCells
void Ctx::turbCopy(double* buf, bool save)
{
    TurbState& t = *turb_;
    const size_t n = static_cast<size_t>(dm_.nC);
    double* f[3] = {t.k, t.eps, t.nut};
    for (int i = 0; i < 3; ++i)
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
