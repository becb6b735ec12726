// Detail blocks of a coupled 1D-3D network and their batched evaluation.
//
// DetailBlock (src/coupling/src/coupledNetwork.cpp:462-620, 644-767,
// 768-877, 878-926, 1080-1152, 1154-1195) is a 3D duct region between one
// inlet and one outlet patch: lossAt(q) writes the inlet rate q (flat, or a
// parabolic / 1/7-power section profile normalised to carry q exactly),
// runs SIMPLE from the region's previous state, and measures the pressure
// drop as rho times the difference of the volume-weighted mean kinematic
// pressure of the first and last cross-sections.  The reference evaluates a
// network's blocks one after another (coupledNetwork.cpp:1454-1487); here a
// batch runs them concurrently, one CUDA stream per block, with a schedule
// (concurrent workers, solver grid per block) chosen by measurement.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <limits>
#include <thread>

#include "ctx.h"
#include "kernels.cuh"

namespace cfg
{

namespace
{

/// Volume-weighted pressure sums of the first and last cross-section and
/// the flux sums of the inlet and outlet patches: block b of 4 reduces list
/// b in a fixed order.  out = {pV0, V0, pV1, V1, phiIn, phiOut}.
__global__ void __launch_bounds__(TPB) k_detail_measure(const int* __restrict__ first, int nFirst,
                                                        const int* __restrict__ last, int nLast, int inStart, int nIn,
                                                        int outStart, int nOut, const double* __restrict__ V,
                                                        const double* __restrict__ p, const double* __restrict__ phi,
                                                        double* out)
{
    double s[2] = {0.0, 0.0};
    const int b = blockIdx.x;
    if (b < 2)
    {
        const int* list = b == 0 ? first : last;
        const int n = b == 0 ? nFirst : nLast;
        for (int k = threadIdx.x; k < n; k += TPB)
        {
            const int c = list[k];
            s[0] += p[c] * V[c];
            s[1] += V[c];
        }
    }
    else
    {
        const int st = b == 2 ? inStart : outStart;
        const int n = b == 2 ? nIn : nOut;
        for (int k = threadIdx.x; k < n; k += TPB) s[0] += phi[st + k];
    }
    block_sum<2>(s);
    if (threadIdx.x != 0) return;
    if (b < 2)
    {
        out[2 * b] = s[0];
        out[2 * b + 1] = s[1];
    }
    else
    {
        out[2 + b] = s[0];
    }
}

Vec patchArea(const Mesh& M, int patch)
{
    const auto& pt = M.patches[static_cast<size_t>(patch)];
    Vec s{0, 0, 0};
    for (int64_t f = pt.start; f < pt.start + pt.size; ++f) s = s + M.Sf[static_cast<size_t>(f)];
    return s;
}

double comp(const Vec& v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }
double hdot(const Vec& a, const Vec& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }

/// The box of the mesh points (polyMesh::minX / maxX).
struct Box
{
    double lo[3], hi[3];
};

Box pointBox(const Mesh& M)
{
    Box b{{M.points[0].x, M.points[0].y, M.points[0].z}, {M.points[0].x, M.points[0].y, M.points[0].z}};
    for (const Vec& p : M.points)
    {
        const double x[3] = {p.x, p.y, p.z};
        for (int k = 0; k < 3; ++k)
        {
            b.lo[k] = std::min(b.lo[k], x[k]);
            b.hi[k] = std::max(b.hi[k], x[k]);
        }
    }
    return b;
}

/// The cells of the first and the last cross-section the flow meets.  Cells
/// are ranked by (axial centre, index) and taken in flow order; a section is
/// a run of cells whose centres lie within `band` of the run's first one
/// (DetailBlock::buildSections, coupledNetwork.cpp:644-667).
void endSections(const Mesh& M, int axis, int flowSign, double band, std::vector<int64_t>& first,
                 std::vector<int64_t>& last)
{
    const size_t n = static_cast<size_t>(M.nCells);
    std::vector<std::pair<double, int64_t>> rank(n);
    for (size_t c = 0; c < n; ++c) rank[c] = {comp(M.C[c], axis), static_cast<int64_t>(c)};
    std::sort(rank.begin(), rank.end());
    // position i in flow order
    auto at = [&](size_t i) -> const std::pair<double, int64_t>& { return rank[flowSign > 0 ? i : n - 1 - i]; };
    size_t runs = 0, lastStart = 0;
    for (size_t i = 0; i < n;)
    {
        const double anchor = at(i).first;
        size_t j = i + 1;
        while (j < n && std::abs(at(j).first - anchor) <= band) ++j;
        if (runs == 0)
            for (size_t k = i; k < j; ++k) first.push_back(at(k).second);
        lastStart = i;
        ++runs;
        i = j;
    }
    if (runs < 2)
        fail(CFG_ESETUP, "detailBlock: the detailed region has fewer than two cross-sections to measure a drop between");
    for (size_t k = lastStart; k < n; ++k) last.push_back(at(k).second);
}

/// Bit k set: wall patches close the section on both sides across axis k
/// (each wall counted on the axis its area vector points along most).
unsigned wallBoundedAxes(const Mesh& M, int flowAxis)
{
    unsigned low = 0, high = 0;
    for (int pi = 0; pi < static_cast<int>(M.patches.size()); ++pi)
    {
        if (M.patches[static_cast<size_t>(pi)].type != "wall") continue;
        const Vec a = patchArea(M, pi);
        if (!(std::sqrt(hdot(a, a)) > 0)) continue;
        const double s[3] = {a.x, a.y, a.z};
        int k = 0;
        if (std::abs(s[1]) > std::abs(s[k])) k = 1;
        if (std::abs(s[2]) > std::abs(s[k])) k = 2;
        (s[k] < 0 ? low : high) |= 1u << k;
    }
    return low & high & ~(1u << flowAxis);
}

/// Per-face weights of a shaped inlet profile (parabolic or 1/7 power in the
/// normalised transverse coordinate of each bounded axis, the axes'
/// factors multiplied in ascending axis order), scaled so the weighted
/// section area equals the section area: the rate written stays the rate
/// given (DetailBlock::buildInletProfile, coupledNetwork.cpp:768-877).
std::vector<double> profileWeights(const Mesh& M, int inlet, double inletArea, unsigned axes, bool parabolic,
                                   const Box& box, const std::string& shape)
{
    double mid[3], half[3];
    for (int k = 0; k < 3; ++k)
    {
        if (!(axes >> k & 1u)) continue;
        if (!(box.hi[k] > box.lo[k]))
            fail(CFG_ESETUP, "detailBlock: the inlet section has no extent to spread a profile over");
        mid[k] = 0.5 * (box.hi[k] + box.lo[k]);
        half[k] = 0.5 * (box.hi[k] - box.lo[k]);
    }
    const auto& pin = M.patches[static_cast<size_t>(inlet)];
    std::vector<double> w(static_cast<size_t>(pin.size));
    double sumA = 0, sumWA = 0;
    double least = std::numeric_limits<double>::max();
    for (int64_t j = 0; j < pin.size; ++j)
    {
        const Vec& fc = M.Cf[static_cast<size_t>(pin.start + j)];
        const double x[3] = {fc.x, fc.y, fc.z};
        double f = 1.0;
        for (int k = 0; k < 3; ++k)
        {
            if (!(axes >> k & 1u)) continue;
            const double eta = (x[k] - mid[k]) / half[k];
            f *= parabolic ? 1.0 - eta * eta : std::pow(1.0 - std::abs(eta), 1.0 / 7.0);
        }
        least = std::min(least, f);
        w[static_cast<size_t>(j)] = f;
    }
    if (!(least > 0)) fail(CFG_ESETUP, "detailBlock: the inlet profile '" + shape + "' writes a zero or reversed weight on a face");
    for (int64_t j = 0; j < pin.size; ++j)
    {
        const double a = M.magSf[static_cast<size_t>(pin.start + j)];
        sumWA += w[static_cast<size_t>(j)] * a;
        sumA += a;
    }
    if (!(sumA > 0) || !(sumWA > 0)) fail(CFG_ESETUP, "detailBlock: the inlet section integrates to no area");
    if (std::abs(sumA - inletArea) > 1e-9 * inletArea)
        fail(CFG_ESETUP, "detailBlock: the inlet patch's face areas do not add to its area vector");
    const double mean = sumWA / sumA;
    for (double& x : w) x = x / mean;
    return w;
}

}  // namespace

struct DetailState
{
    int inlet = -1, outlet = -1, axis = 0, flowSign = 1;
    double inletArea = 0, rho = 1;
    // the block's RANS model, created at its first lossAt (after the inlet
    // velocity it scales with is written), as coupledNetwork.cpp:1112-1113
    std::string turbModel = "laminar";
    double turbIntensity = 0.05, turbLength = -1, turbRelax = 0.7, turbNu = 1e-4;
    std::vector<int64_t> inletFaces;
    std::vector<double> inletWeights;  // empty: flat
    std::vector<int> first, last;      // device slots of the first and last cross-section
    int* dFirst = nullptr;
    int* dLast = nullptr;
    double* dOut = nullptr;
    double* hOut = nullptr;
};

void Ctx::detailSetup(const std::string& shape, double rho)
{
    CFG_CUDA(cudaSetDevice(device_));
    const Mesh& M = mesh_;
    if (!(rho > 0)) fail(CFG_EINVAL, "detailBlock: nu and rho must be positive");
    std::unique_ptr<DetailState> d(new DetailState());
    d->rho = rho;
    const int nP = static_cast<int>(M.patches.size());
    for (int pi = 0; pi < nP; ++pi)
    {
        const std::string& t = M.patches[static_cast<size_t>(pi)].type;
        if (t == "inlet" && d->inlet < 0) d->inlet = pi;
        else if (t == "outlet" && d->outlet < 0) d->outlet = pi;
    }
    if (d->inlet < 0 || d->outlet < 0)
        fail(CFG_ESETUP, "detailBlock: the detailed region needs one patch of type inlet and one of type outlet");
    const Vec inSf = patchArea(M, d->inlet), outSf = patchArea(M, d->outlet);
    d->inletArea = std::sqrt(hdot(inSf, inSf));
    if (!(d->inletArea > 0)) fail(CFG_ESETUP, "detailBlock: the inlet patch has no area");
    const Vec sum = inSf + outSf;
    if (std::sqrt(hdot(sum, sum)) > 1e-6 * d->inletArea)
        fail(CFG_ESETUP, "detailBlock: the inlet and outlet patches are not opposed");
    const Vec nrm{inSf.x / d->inletArea, inSf.y / d->inletArea, inSf.z / d->inletArea};
    d->axis = 0;
    if (std::abs(nrm.y) > std::abs(comp(nrm, d->axis))) d->axis = 1;
    if (std::abs(nrm.z) > std::abs(comp(nrm, d->axis))) d->axis = 2;
    d->flowSign = comp(nrm, d->axis) < 0 ? 1 : -1;

    const Box box = pointBox(M);
    {
        std::vector<int64_t> c0, c1;
        endSections(M, d->axis, d->flowSign, 1e-9 * std::max(std::abs(box.hi[d->axis] - box.lo[d->axis]), 1e-30), c0, c1);
        for (int64_t c : c0) d->first.push_back(inv_[static_cast<size_t>(c)]);
        for (int64_t c : c1) d->last.push_back(inv_[static_cast<size_t>(c)]);
    }
    if (shape != "flat")
    {
        if (shape != "parabolic" && shape != "power1over7")
            fail(CFG_ESETUP, "detailBlock: the inlet profile '" + shape +
                                 "' is not one this block can write (flat, parabolic, power1over7)");
        const unsigned axes = wallBoundedAxes(M, d->axis);
        if (!axes)
            fail(CFG_ESETUP, "detailBlock: the inlet profile '" + shape +
                                 "' has no wall-confined transverse direction to vary along");
        d->inletWeights = profileWeights(M, d->inlet, d->inletArea, axes, shape == "parabolic", box, shape);
        const auto& pin = M.patches[static_cast<size_t>(d->inlet)];
        for (int64_t j = 0; j < pin.size; ++j) d->inletFaces.push_back(pin.start + j);
    }
    d->dFirst = upload(d->first);
    d->dLast = upload(d->last);
    d->dOut = alloc<double>(8);
    CFG_CUDA(cudaMallocHost(&d->hOut, 8 * sizeof(double)));
    detail_.reset(d.release());
}

/// lossAt's host side before the solve (coupledNetwork.cpp:1080-1113): the
/// block's boundary conditions for rate q (applyBoundary, :878-926), the
/// boundary flux, the RANS model on the first call, and the outer
/// iteration's host set-up.
void Ctx::detailPrepare(double q, const cfg_simple_controls& ctl)
{
    if (!detail_) fail(CFG_EINVAL, "cfg_detail_loss: call cfg_detail_setup first");
    if (!(q > 0)) fail(CFG_EINVAL, "detailBlock: asked for the drop of a detailed region at a non-positive rate");
    CFG_CUDA(cudaSetDevice(device_));
    DetailState& d = *detail_;
    const Mesh& M = mesh_;
    double inletU[3] = {0, 0, 0};
    inletU[d.axis] = d.flowSign * q / d.inletArea;
    const double zero[3] = {0, 0, 0};
    const int nP = static_cast<int>(M.patches.size());
    for (int pi = 0; pi < nP; ++pi)
    {
        const std::string& t = M.patches[static_cast<size_t>(pi)].type;
        if (pi == d.inlet)
        {
            setPatchBC('U', pi, CFG_BC_FIXED_VALUE, inletU);
            setPatchBC('p', pi, CFG_BC_ZERO_GRADIENT, zero);
        }
        else if (pi == d.outlet)
        {
            setPatchBC('U', pi, CFG_BC_ZERO_GRADIENT, zero);
            setPatchBC('p', pi, CFG_BC_FIXED_VALUE, zero);
        }
        else if (t == "wall")
        {
            setPatchBC('U', pi, CFG_BC_FIXED_VALUE, zero);
            setPatchBC('p', pi, CFG_BC_ZERO_GRADIENT, zero);
        }
        else
        {
            setPatchBC('U', pi, CFG_BC_ZERO_GRADIENT, zero);
            setPatchBC('p', pi, CFG_BC_ZERO_GRADIENT, zero);
        }
    }
    clearFaceValuesU();
    if (!d.inletWeights.empty())
    {
        std::vector<double> vals(3 * d.inletFaces.size());
        for (size_t j = 0; j < d.inletFaces.size(); ++j)
            for (int k = 0; k < 3; ++k) vals[3 * j + k] = inletU[k] * d.inletWeights[j];
        setFaceValuesU(static_cast<int64_t>(d.inletFaces.size()), d.inletFaces.data(), vals.data());
    }
    initFlux(nullptr);  // phi.correctBoundaryFlux(U)
    if (!turb_ && d.turbModel != "laminar")
        turbulenceSetup(d.turbModel, d.turbIntensity, d.turbLength, d.turbRelax, d.turbNu);
    prepareIterate(ctl);
}

/// The volume-weighted section pressures and the patch fluxes of measure
/// (coupledNetwork.cpp:1154-1195), and their copy to the host, enqueued.
void Ctx::detailEnqueueMeasure()
{
    DetailState& d = *detail_;
    const Mesh& M = mesh_;
    const auto& pin = M.patches[static_cast<size_t>(d.inlet)];
    const auto& pout = M.patches[static_cast<size_t>(d.outlet)];
    k_detail_measure<<<4, TPB, 0, stream_>>>(d.dFirst, static_cast<int>(d.first.size()), d.dLast,
                                             static_cast<int>(d.last.size()), static_cast<int>(pin.start),
                                             static_cast<int>(pin.size), static_cast<int>(pout.start),
                                             static_cast<int>(pout.size), dm_.V, p_, phi_, d.dOut);
    launchCheck("detail_measure");
    CFG_CUDA(cudaMemcpyAsync(d.hOut, d.dOut, 6 * sizeof(double), cudaMemcpyDeviceToHost, stream_));
}

/// The drop from the measured sums and lossAt's own checks of it
/// (coupledNetwork.cpp:1146-1151), once the device work is done.
void Ctx::detailFinish(double q, const cfg_simple_result& res, double deviceMs, cfg_detail_measure& out)
{
    DetailState& d = *detail_;
    const double* h = d.hOut;
    const double p0 = h[1] > 0 ? h[0] / h[1] : 0.0, p1 = h[3] > 0 ? h[2] / h[3] : 0.0;
    out = cfg_detail_measure{};
    out.cells = mesh_.nCells;
    out.sweeps = res.iterations;
    out.converged = res.converged;
    out.diverged = res.diverged;
    out.dp_pa = d.rho * p0 - d.rho * p1;
    out.imposed_q = q;
    out.flux_in = -h[4];
    out.flux_out = h[5];
    out.inlet_area = d.inletArea;
    out.plug_speed = q / d.inletArea;
    out.device_ms = deviceMs;
    out.u_inner_iterations = res.u_inner_iterations;
    out.p_inner_iterations = res.p_inner_iterations;
    if (!std::isfinite(out.dp_pa)) out.status = CFG_ENUMERIC;
    else if (out.dp_pa <= 0) out.status = CFG_ENUMERIC;
}

void Ctx::detailLoss(double q, const cfg_simple_controls& ctl, cfg_detail_measure& out)
{
    detailPrepare(q, ctl);
    cfg_simple_result res{};
    iterate(ctl, res);
    detailEnqueueMeasure();
    CFG_CUDA(cudaStreamSynchronize(stream_));
    detailFinish(q, res, lastMs[7], out);
}

void Ctx::detailTurbulence(const std::string& model, double intensity, double lengthScale, double relaxation,
                           double nu)
{
    if (!detail_) fail(CFG_EINVAL, "cfg_detail_turbulence: call cfg_detail_setup first");
    if (model != "laminar" && model != "kEpsilon" && model != "kOmegaSST" && model != "des" &&
        model != "gammaTransition")
        fail(CFG_ESETUP, "turbulence: model '" + model +
                             "' is not on the GPU path (laminar | kEpsilon | kOmegaSST | des | gammaTransition)");
    detail_->turbModel = model;
    detail_->turbIntensity = intensity;
    detail_->turbLength = lengthScale;
    detail_->turbRelax = relaxation;
    detail_->turbNu = nu;
    if (model == "laminar" && turb_) turbulenceSetup("laminar", 0, 0, 1, nu);
}

void Ctx::saveState()
{
    CFG_CUDA(cudaSetDevice(device_));
    const size_t nC = static_cast<size_t>(dm_.nC), nF = static_cast<size_t>(dm_.nF);
    if (!saved_) saved_ = alloc<double>(4 * nC + nF);
    for (int q = 0; q < 3; ++q)
        CFG_CUDA(cudaMemcpyAsync(saved_ + q * nC, U_.c[q], nC * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    CFG_CUDA(cudaMemcpyAsync(saved_ + 3 * nC, p_, nC * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    CFG_CUDA(cudaMemcpyAsync(saved_ + 4 * nC, phi_, nF * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    savedTurb_ = turb_ != nullptr;
    if (savedTurb_)
    {
        if (!savedT_) savedT_ = alloc<double>(4 * nC);
        turbCopy(savedT_, true);
    }
    CFG_CUDA(cudaStreamSynchronize(stream_));
}

void Ctx::restoreState()
{
    if (!saved_) fail(CFG_EINVAL, "restoreState: nothing saved");
    CFG_CUDA(cudaSetDevice(device_));
    const size_t nC = static_cast<size_t>(dm_.nC), nF = static_cast<size_t>(dm_.nF);
    for (int q = 0; q < 3; ++q)
        CFG_CUDA(cudaMemcpyAsync(U_.c[q], saved_ + q * nC, nC * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    CFG_CUDA(cudaMemcpyAsync(p_, saved_ + 3 * nC, nC * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    CFG_CUDA(cudaMemcpyAsync(phi_, saved_ + 4 * nC, nF * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    if (savedTurb_ && turb_) turbCopy(savedT_, false);
    CFG_CUDA(cudaStreamSynchronize(stream_));
}

void Ctx::setRowBlocks(int k)
{
    // the solver grid, for blocks that share the GPU: never larger than the
    // grid the partial buffers were sized for
    if (k <= 0) k = initRowBlocks_;
    if (k == rowBlocksPerSM_) return;
    const int keep = rowBlocksPerSM_;
    rowBlocksPerSM_ = k;
    int pOff = 0;
    for (const DicPhase& ph : dicPhase_) pOff += rowGrid(ph.cnt);
    if (rowGrid(dm_.nC) > initGS_ || pOff + 1 > initDicPartials_)
    {
        rowBlocksPerSM_ = keep;  // larger than the partial buffers allow
        return;
    }
    GS_ = rowGrid(dm_.nC);
    pOff = 0;
    for (DicPhase& ph : dicPhase_)
    {
        ph.partialOff = pOff;
        pOff += rowGrid(ph.cnt);
    }
    dicPartials_ = pOff + 1;
    for (auto& g : graphs_) cudaGraphExecDestroy(g.second);
    graphs_.clear();
}

}  // namespace cfg

// ---------------------------------------------------------------------------
// batches
// ---------------------------------------------------------------------------

namespace cfg
{

void DetailDeleter::operator()(DetailState* d) const
{
    if (d && d->hOut) cudaFreeHost(d->hOut);
    delete d;
}

/// The captured graph of a whole coupling pass (batch schedule with
/// workers == 0): every block's outer iteration and measure as parallel
/// branches, its solver loops as device-side while-nodes.
struct BatchGraph
{
    std::string key;
    cudaStream_t origin = nullptr;
    cudaEvent_t fork = nullptr;
    std::vector<cudaEvent_t> join;
    cudaGraphExec_t exec = nullptr;
    ~BatchGraph()
    {
        if (exec) cudaGraphExecDestroy(exec);
        for (cudaEvent_t e : join) cudaEventDestroy(e);
        if (fork) cudaEventDestroy(fork);
        if (origin) cudaStreamDestroy(origin);
    }
};

void BatchGraphDeleter::operator()(BatchGraph* g) const { delete g; }

namespace
{

/// Runs fn(i) for i in [0, n) on up to `threads` host threads; the error
/// of the lowest failing block is raised after all have run.
template <class F>
void forBlocks(int n, int threads, F&& fn)
{
    std::atomic<int> next{0};
    std::vector<std::string> errs(static_cast<size_t>(n));
    std::vector<int> codes(static_cast<size_t>(n), CFG_OK);
    auto work = [&]() {
        for (int i; (i = next.fetch_add(1)) < n;)
        {
            try
            {
                fn(i);
            }
            catch (const Error& e)
            {
                errs[static_cast<size_t>(i)] = e.what();
                codes[static_cast<size_t>(i)] = e.code;
            }
            catch (const std::exception& e)
            {
                errs[static_cast<size_t>(i)] = e.what();
                codes[static_cast<size_t>(i)] = CFG_EINVAL;
            }
        }
    };
    const int w = std::max(1, std::min(threads, n));
    if (w == 1) work();
    else
    {
        std::vector<std::thread> th;
        for (int t = 0; t < w; ++t) th.emplace_back(work);
        for (auto& t : th) t.join();
    }
    for (int i = 0; i < n; ++i)
        if (codes[static_cast<size_t>(i)] != CFG_OK)
            fail(codes[static_cast<size_t>(i)], "block " + std::to_string(i) + ": " + errs[static_cast<size_t>(i)]);
}

/// One coupling pass as a single CUDA-graph launch.  The host sets every
/// block's boundary values for its rate (on host threads), launches the
/// pass graph -- captured on the first pass of a schedule and set of
/// controls, replayed after -- and reads each block's scalars and sums.
void batchPassGraph(cfg_batch& b, const double* q, const cfg_simple_controls* ctl, cfg_detail_measure* out,
                    double* wallMs)
{
    const int n = static_cast<int>(b.blocks.size());
    for (cfg::Ctx* c : b.blocks)
        c->setRowBlocks(b.rowBlocks >= 0 ? b.rowBlocks
                                         : static_cast<int>(std::min<int64_t>(4, std::max<int64_t>(
                                                                                  1, c->mesh().nCells / 32768))));
    const auto t0 = std::chrono::steady_clock::now();
    const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
    forBlocks(n, static_cast<int>(std::min(hw, 16u)),
              [&](int i) { b.blocks[static_cast<size_t>(i)]->detailPrepare(q[i], ctl[i]); });
    std::string key = std::to_string(b.rowBlocks);
    for (int i = 0; i < n; ++i) key.append(reinterpret_cast<const char*>(&ctl[i]), sizeof(cfg_simple_controls));
    if (!b.graph || b.graph->key != key)
    {
        b.graph.reset(new BatchGraph());
        BatchGraph& g = *b.graph;
        g.key = key;
        CFG_CUDA(cudaStreamCreateWithFlags(&g.origin, cudaStreamNonBlocking));
        CFG_CUDA(cudaEventCreateWithFlags(&g.fork, cudaEventDisableTiming));
        g.join.resize(static_cast<size_t>(n));
        for (auto& e : g.join) CFG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        // every block's own set-up work is finished before its branch is
        // captured after it
        for (cfg::Ctx* c : b.blocks) CFG_CUDA(cudaStreamSynchronize(c->stream()));
        CFG_CUDA(cudaStreamBeginCapture(g.origin, cudaStreamCaptureModeThreadLocal));
        cudaGraph_t graph = nullptr;
        try
        {
            CFG_CUDA(cudaEventRecord(g.fork, g.origin));
            for (int i = 0; i < n; ++i)
            {
                cfg::Ctx& c = *b.blocks[static_cast<size_t>(i)];
                CFG_CUDA(cudaStreamWaitEvent(c.stream(), g.fork, 0));
                c.setDeviceLoops(true);
                int64_t u = 0, p = 0;
                try
                {
                    c.enqueueOuter(ctl[i], u, p);
                    c.detailEnqueueMeasure();
                }
                catch (...)
                {
                    c.setDeviceLoops(false);
                    throw;
                }
                c.setDeviceLoops(false);
                CFG_CUDA(cudaEventRecord(g.join[static_cast<size_t>(i)], c.stream()));
                CFG_CUDA(cudaStreamWaitEvent(g.origin, g.join[static_cast<size_t>(i)], 0));
            }
        }
        catch (...)
        {
            cudaStreamEndCapture(g.origin, &graph);
            if (graph) cudaGraphDestroy(graph);
            b.graph.reset();
            throw;
        }
        CFG_CUDA(cudaStreamEndCapture(g.origin, &graph));
        const cudaError_t e = cudaGraphInstantiate(&g.exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess)
        {
            b.graph.reset();
            fail(CFG_ECUDA, std::string("batch pass graph: cudaGraphInstantiate: ") + cudaGetErrorString(e));
        }
    }
    BatchGraph& g = *b.graph;
    for (cfg::Ctx* c : b.blocks) CFG_CUDA(cudaStreamSynchronize(c->stream()));
    CFG_CUDA(cudaGraphLaunch(g.exec, g.origin));
    CFG_CUDA(cudaStreamSynchronize(g.origin));
    const auto t1 = std::chrono::steady_clock::now();
    const double ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    if (wallMs) *wallMs = ms;
    for (int i = 0; i < n; ++i)
    {
        cfg::Ctx& c = *b.blocks[static_cast<size_t>(i)];
        cfg_simple_result res{};
        double lag1 = INFINITY, lag2 = INFINITY;
        c.finishOuter(ctl[i], 1, lag1, lag2, res);
        int64_t t = 0;
        c.deviceInner(res.u_inner_iterations, res.p_inner_iterations, t);
        c.detailFinish(q[i], res, ms, out[i]);
    }
}

}  // namespace

/// One coupling pass: every block's lossAt at its own rate.  With workers
/// == 0 the pass is one CUDA-graph launch (batchPassGraph); otherwise
/// blocks are taken largest first by `workers` host threads, each block on
/// its own context stream, so up to `workers` blocks run on the GPU at once.
void batchPass(cfg_batch& b, const double* q, const cfg_simple_controls* ctl, cfg_detail_measure* out,
               double* wallMs)
{
    if (b.workers == 0)
    {
        for (int i = 0; i < static_cast<int>(b.blocks.size()); ++i)
            if (ctl[i].max_iterations != 1 || ctl[i].p_precond == CFG_PRECOND_AMG ||
                ctl[i].p_precond == CFG_PRECOND_MPNN || ctl[i].p_precond == CFG_PRECOND_IR32 ||
                ctl[i].p_precond == CFG_PRECOND_AMG_MPNN || ctl[i].u_precond != CFG_PRECOND_JACOBI ||
                b.blocks[static_cast<size_t>(i)]->turbulenceModelName() == "gammaTransition")
                fail(CFG_EINVAL, "batch: the single-graph pass runs one outer iteration per block with Jacobi or DIC "
                                 "pressure, Jacobi momentum and no gammaTransition model");
        batchPassGraph(b, q, ctl, out, wallMs);
        return;
    }
    const int n = static_cast<int>(b.blocks.size());
    std::vector<int> order(static_cast<size_t>(n));
    for (int i = 0; i < n; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(),
                     [&](int x, int y) { return b.blocks[x]->mesh().nCells > b.blocks[y]->mesh().nCells; });
    // rowBlocks < 0: by size, so a large block on the critical path keeps a
    // wide grid while small ones share the SMs (1 block per SM per 32k cells,
    // at most 4)
    for (cfg::Ctx* c : b.blocks)
        c->setRowBlocks(b.rowBlocks >= 0 ? b.rowBlocks
                                         : static_cast<int>(std::min<int64_t>(4, std::max<int64_t>(
                                                                                  1, c->mesh().nCells / 32768))));
    std::atomic<int> next{0};
    std::vector<std::string> errs(static_cast<size_t>(n));
    std::vector<int> codes(static_cast<size_t>(n), CFG_OK);
    auto work = [&]() {
        for (;;)
        {
            const int k = next.fetch_add(1);
            if (k >= n) return;
            const int i = order[k];
            try
            {
                // a non-positive or non-finite drop is reported in
                // out[i].status; the pass goes on with the other blocks
                b.blocks[i]->detailLoss(q[i], ctl[i], out[i]);
            }
            catch (const Error& e)
            {
                errs[i] = e.what();
                codes[i] = e.code;
            }
            catch (const std::exception& e)
            {
                errs[i] = e.what();
                codes[i] = CFG_EINVAL;
            }
        }
    };
    const auto t0 = std::chrono::steady_clock::now();
    const int w = std::max(1, std::min(b.workers, n));
    if (w == 1)
    {
        work();
    }
    else
    {
        std::vector<std::thread> th;
        for (int t = 0; t < w; ++t) th.emplace_back(work);
        for (auto& t : th) t.join();
    }
    const auto t1 = std::chrono::steady_clock::now();
    if (wallMs) *wallMs = std::chrono::duration<double, std::milli>(t1 - t0).count();
    for (int i = 0; i < n; ++i)
        if (codes[i] != CFG_OK) fail(codes[i], "block " + std::to_string(i) + ": " + errs[i]);
}

}  // namespace cfg
