// The per-case device context (host declarations; kernels in simple.cu).
#pragma once

#include <cuda_runtime.h>

#include <functional>
#include <map>
#include <string>
#include <algorithm>
#include <memory>
#include <vector>

#include "cfg_internal.h"
#include "dev_types.h"

namespace cfg
{

struct Timing
{
    cudaEvent_t ev[16];
    double ms[8];
    int64_t launches;
};

struct DetailState;
struct DetailDeleter
{
    void operator()(DetailState* d) const;
};
struct MpnnState;
struct MpnnDeleter
{
    void operator()(MpnnState* m) const;
};
struct TurbState;
struct TurbDeleter
{
    void operator()(TurbState* t) const;
};
struct AmgState;
struct FcgState;
struct AmgDeleter
{
    void operator()(AmgState* a) const;
};

class Ctx
{
public:
    Ctx(const Mesh& mesh, int device, cudaStream_t stream, int order = -1);
    ~Ctx();

    // boundary conditions and schemes
    void setPatchBC(char field, int patch, int type, const double* value);
    void setFaceValuesU(int64_t n, const int64_t* faces, const double* values);
    void clearFaceValuesU();
    void setSchemes(const cfg_schemes& s) { schemes_ = s; }

    void upload(const double* U, const double* p, const double* phi);
    /// SimpleControls::uTimeOld (cfg_fields_upload_old)
    void uploadOld(const double* U);
    void download(double* U, double* p, double* phi);
    void initFlux(const double* u0);
    void iterate(const cfg_simple_controls& ctl, cfg_simple_result& res);
    /// The pieces of iterate: host set-up, one outer iteration enqueued
    /// (capturable with device loops on), and the host's reading of its
    /// scalars (1: stop).
    void prepareIterate(const cfg_simple_controls& ctl);
    void enqueueOuter(const cfg_simple_controls& ctl, int64_t& uInner, int64_t& pInner);
    int finishOuter(const cfg_simple_controls& ctl, int iter, double& contLag1, double& contLag2,
                    cfg_simple_result& res);
    /// Device-side solver loops (conditional while-nodes) instead of host
    /// polling, for enqueueOuter under stream capture.
    void setDeviceLoops(bool on) { devLoop_ = on; }
    cudaStream_t stream() const { return stream_; }
    /// the inner iteration counts a device-loop iteration left in the
    /// scalars: momentum, pressure, RANS model
    void deviceInner(int64_t& u, int64_t& p, int64_t& t) const;
    /// one transient PISO step (pisoSolver.cpp)
    void pisoStep(const cfg_piso_controls& ctl, cfg_piso_result& res);

    /// DetailBlock (src/coupling/src/coupledNetwork.cpp): inlet/outlet
    /// patches, cross-sections and the inlet profile, then lossAt(q).
    void detailSetup(const std::string& shape, double rho);
    void detailLoss(double q, const cfg_simple_controls& ctl, cfg_detail_measure& out);
    /// lossAt in pieces, for a pass captured as one graph: host set-up for
    /// rate q, the measure enqueued, the drop from the measured sums
    void detailPrepare(double q, const cfg_simple_controls& ctl);
    void detailEnqueueMeasure();
    void detailFinish(double q, const cfg_simple_result& res, double deviceMs, cfg_detail_measure& out);
    void detailTurbulence(const std::string& model, double intensity, double lengthScale, double relaxation,
                          double nu);
    /// Solver grid of at most k blocks per SM (0: the context's own).
    void setRowBlocks(int k);

    /// RANS model ("laminar" removes it), advanced once per SIMPLE outer
    /// iteration; the case's boundary conditions must be set first (the
    /// initial k and epsilon scale with the inlet velocity).
    void turbulenceSetup(const std::string& model, double intensity, double lengthScale, double relaxation,
                         double nu);
    void turbulenceFields(double* k, double* eps, double* nut, double* nuEffFace);
    void turbulenceParams(double cDES, double reOnset, double onsetWidth, double gammaRate);
    bool hasTurbulence() const { return static_cast<bool>(turb_); }
    std::string turbulenceModelName() const;

    /// The learned pressure preconditioner (mpnn.cu) on the context's
    /// pressure matrix (the Poisson system or the last SIMPLE equation).
    void mpnnCreate(int layers, uint64_t seed);
    void mpnnWeights(float* get, const float* set, int64_t n);
    int mpnnParams() const;
    double mpnnLossGradHost(const double* r, float* grad, const double* t = nullptr);
    void mpnnApplyHost(const double* r, double* z);
    void mpnnTrainHost(const double* samples, int nSamples, int epochs, float lr, double* losses,
                       const double* targets = nullptr);
    /// residuals the pressure solves start from, kept as training samples
    void mpnnCollect(int mode, int maxSamples);
    int mpnnCollected() const { return static_cast<int>(collected_.size()); }
    void mpnnTrainCollected(int epochs, float lr, double* losses);
    void poissonResidual(const double* b, const double* x, double* r);
    void refreshBcPublic() { refreshBc(); }
    int64_t lastTurbInner = 0;
    int64_t lastFallbackIters = 0;
    /// A device-side copy of U, p, phi, and its return (for schedule trials
    /// on identical work).
    void saveState();
    void restoreState();

    // diagnostics used by the parity tests
    void probeEquations(const cfg_simple_controls& ctl, const double* xprobe, double* out);
    void gradient(const double* data, const double* bvals, int scheme, int volQuirk, double* out);
    void probeDIC(const double* r, double* z, double* rDinv);
    int nColours() const { return nColours_; }

    /// solveCG / solveBiCGStab on a host CSR (Matrix.cpp:153-319)
    static void sparseSolve(int device, int64_t n, const int64_t* rs, const int64_t* cols, const double* vals,
                            const double* b, double* x, double tol, int maxIter, int method,
                            cfg_solver_report* rep);

    double lastMs[8] = {0};
    int64_t lastLaunches = 0;

    /// Per-kernel CUDA-event timing of the linear-solver kernels (opt-in):
    /// kstat[k] = {launches, total ms} for the slots KS_*.
    void setKernelTiming(bool on);
    enum
    {
        KS_CG_SPMV,
        KS_CG_UPDATE,
        KS_CG_P,
        KS_BI_P,
        KS_BI_SPMV1,
        KS_BI_SPMV2,
        KS_BI_X,
        KS_DIC_APPLY,
        // the momentum BiCGStab with the AMG V-cycle (u_precond AMG); the
        // two V-cycles of an iteration share the three V-cycle slots: the
        // finest pre-sweep and residual, everything coarser (restriction
        // to prolongation), the finest post-sweep
        KS_BIA_P,
        KS_AMGV_PRE0,
        KS_AMGV_COARSE,
        KS_AMGV_POST0,
        KS_BIA_SPMV1,
        KS_BIA_S,
        KS_BIA_SPMV2,
        KS_BIA_X,
        KS_COUNT
    };
    double kstat[KS_COUNT][2] = {};
    /// per slot, the launches weighted by the components still iterating
    /// (the fused BiCGStab kernels skip converged components; 1 per launch
    /// for the single-vector kernels)
    double kcomp[KS_COUNT] = {};

    const Mesh& mesh() const { return mesh_; }

private:
    template <class T>
    T* alloc(size_t n);
    template <class T>
    T* upload(const std::vector<T>& v);

    void buildDevice();
    void refreshBc();
    void gradCells(const double* const* x, int nComp, const BcTab& bc, int scheme, bool volQuirk, V3P* out);
    void solveMomentum(int nonOrth, int gradScheme, double tol, int maxIter, int64_t& inner);
    void solvePressure(int nonOrth, int gradScheme, double tol, int maxIter, int precond, int64_t& inner,
                       const double* x0 = nullptr);
    void runCG(const double* vals, const double* diag, const double* b, double* x, double tol, int maxIter,
               cfg_solver_report* rep, int normType = 0);
    void runBiCG3(const double* vals, const double* diag, V3P b, V3P x, int nComp, double tol, int maxIter,
                  cfg_solver_report* reps);
    void runBiCGAmg(const double* vals, const double* diag, V3P b, V3P x, double tol, int maxIter,
                    cfg_solver_report* reps);
    /// the momentum preconditioner of the outer iteration being enqueued
    /// (cfg_simple_controls.u_precond) and the FP32 copy of the momentum
    /// values the V-cycle's finest level reads
    int uPrecond_ = CFG_PRECOND_JACOBI;
    float* uVal32_ = nullptr;
    void launchCheck(const char* what, int kernels = 1);
    int linUpwindGrad(const BcTab& ub, int gradScheme);
    template <class F>
    void launchChunk(const std::string& key, int n, F&& body);
    /// While stream_ is being captured: a while-node whose body is what
    /// `body` enqueues, repeated until the solver state is done (at most
    /// maxBodies times).
    template <class F>
    void captureWhile(int maxBodies, F&& body);
    bool devLoop_ = false;
    double* tally_ = nullptr;  // {iterations, unconverged} of device-loop solves
    cudaStream_t bodyStream_ = nullptr;
    int* loopCount_ = nullptr;
    void dicSetup(const double* vals, const double* diag);
    void dicApply(const double* r, double* z);
    void runDICCG(const double* vals, const double* diag, const double* b, double* x, double tol, int maxIter,
                  cfg_solver_report* rep, int normType = 0);
    template <class T>
    void dicSetupT(DDicT<T>& D, const double* vals, const T* diag);
    template <class T>
    void dicApplyT(const DDicT<T>& D, const T* r, T* z);
    template <class T>
    void dicCGT(const DDicT<T>& D, const T* vals, const T* diag, const T* b, T* x, T* r, T* p, T* Ap, T* z, double tol,
                int maxIter, int normType, cfg_solver_report* rep);

public:
    /// The pressure-Poisson system of the mixed-precision study: the
    /// orthogonal part of laplacianFace with unit face coefficient, the
    /// patches' p conditions and an optional reference cell.
    void poissonSetup(int64_t refCell);
    void poissonSolve(const double* b, double* x, int method, double tol, int maxIter, int innerMax,
                      double innerTol, double* out);
    /// the AMG hierarchy for the Poisson system's current values
    void poissonAmg(double* out);
    void poissonAmgApply(const double* r, double* z);
    void poissonAmgApply3(const double* r, double* z, const int32_t done[3]);
    /// strength threshold of the pressure hierarchy's aggregation (0: plain);
    /// fixed once that hierarchy is built
    void setAmgStrength(double theta);
    double amgStrength() const { return amgTheta_; }

private:
    void setNu(double nu);
    void checkMomentumBcs() const;

    Mesh mesh_;
    int device_;
    cudaStream_t stream_;
    bool ownStream_ = false;
    int G_ = 0;        // grid of row kernels
    int GF_ = 0;       // grid of face kernels
    int GS_ = 0;       // grid of solver kernels (rowGrid(nC))
    int sms_ = 0;
    int rowBlocksPerSM_ = 4;  // 0: RPT rows per thread; k > 0: at most k blocks per SM
    int initRowBlocks_ = 4, initGS_ = 0, initDicPartials_ = 1;
    std::unique_ptr<DetailState, DetailDeleter> detail_;
    std::unique_ptr<TurbState, TurbDeleter> turb_;
    std::unique_ptr<MpnnState, MpnnDeleter> mpnn_;
    // aggregation AMG in FP32 (amg.cu): one hierarchy for the pressure (and
    // the Poisson system), aggregated by strength of connection when
    // amgTheta_ > 0, and one for the momentum matrix, aggregated plainly.
    // Each is built from its operator's pattern (and, for strength, values)
    // on its first amgValues.
    enum AmgUse { kAmgPressure = 0, kAmgMomentum = 1 };
    std::unique_ptr<AmgState, AmgDeleter> amg_, amgU_;
    std::unique_ptr<AmgState, AmgDeleter>& amgSlot(AmgUse use) { return use == kAmgMomentum ? amgU_ : amg_; }
    double amgTheta_ = 0.0;
    void amgSetup(AmgUse use, const double* vals, double theta);
    void amgValues(AmgUse use, const double* vals, const double* diag, const float* vals32);
    void amgApply(const double* r, double* z);
    void amgCycle(const double* r, double* z, const double* q, FcgState* st);
    /// mark(0) after the finest pre-sweep, mark(1) before the finest
    /// post-sweep (kernel timing), when given
    void amgCycle3(AmgUse use, CV3P b, V3P z, const int* done, float scale, const std::function<void(int)>& mark = {});
    void amgVectors3(AmgUse use);
    int amgCycleKernels(AmgUse use = kAmgPressure) const;
    void amgFcg(const double* vals, const double* b, double* x, double tol, int maxIter, int normType,
                cfg_solver_report* rep);
    void amgInfo(double* out);
    bool amgFresh_ = false;  // the hierarchy's values match the Poisson system
    void mpnnApply(const double* vals, const double* diag, const double* r, double* z);
    double mpnnLossGrad(const double* vals, const double* diag, const double* r, double* z,
                        const double* t = nullptr);
    void mpnnGuess(const double* vals, const double* diag, const double* b, double* x);
    bool mpnnTimeLayers_ = false;
    double mpnnLayerMs_ = 0;
    int64_t mpnnLayerLaunches_ = 0;

public:
    void mpnnTime(int reps, double* out);

private:
    double* trainBuf_ = nullptr;
    size_t trainCap_ = 0;
    void mpnnAdam(float lr);
    void mpnnMatrix(const double** vals, const double** diag) const;
    void mpnnTrain(const double* samples, int nSamples, int epochs, float lr, double* losses,
                   const double* targets = nullptr);
    void mpnnFcg(const double* vals, const double* diag, const double* b, double* x, double tol, int maxIter,
                 int window, int64_t* out, int normType, int pc = 0);
    double fcgNorm(const double* v, int normType);
    void mpnnResidualHost(const double* vals, const double* b, const double* x, double* rHost);
    bool collectOn_ = false;
    int collectMax_ = 0;
    std::vector<std::vector<double>> collected_;   // residual each collected solve started from
    std::vector<std::vector<double>> collectedT_;  // the correction it converged to
    void fcgSpmv(const double* vals, const double* x, double* y);
    void fcgDots(int np, const double* const* a, const double* const* b, double* out);
    const double** fcgPtrs_ = nullptr;
    double* fcgOut_ = nullptr;
    unsigned* fcgTicket_ = nullptr;
    void turbCorrect(int64_t& inner, double dt = 0.0);
    void turbRefreshNut();
    void turbSolveScalar(const double* bc, const double* bk, const double* sigCell, double sigma, bool wallOverride,
                         const double* src2, double* field, double floorV, bool clamp01, double dt,
                         int64_t& inner);
    double turbURef();
    // the model options of TurbulenceConfig beyond cfg_turbulence_setup's
    double turbCDES_ = 0.61, turbReOnset_ = 0.0, turbOnsetWidth_ = -1.0, turbGammaRate_ = 4.0;
    double* saved_ = nullptr;
    V3P uOld_{};
    bool oldUploaded_ = false;
    double* savedT_ = nullptr;
    bool savedTurb_ = false;
    void turbCopy(double* buf, bool save);
    int rowGrid(int rows) const;
    int maxW_ = 0;     // longest matrix row
    int nSlicesEntries_ = 0;  // matrix SELL entries
    int nSlices_ = 0;
    std::vector<void*> allocs_;
    DMesh dm_{};

    // boundary conditions (host)
    std::vector<int> uType_, pType_;
    // device numbering: slot i holds original cell perm_[i]; inv_ = perm_^-1
    int order_ = -1;
    std::vector<int> perm_, inv_;
    bool identityOrder_ = true;
    std::vector<double> hostTmp_;
    void toDevCells(double* dev, const double* host, int stride, int off);
    void fromDevCells(double* host, const double* dev, int stride, int off);
    // whole cell fields of nc = 1 or 3 interleaved components: one copy of the
    // host array through ioStage_, transposed and renumbered on the device
    void cellsToDev(double* const* dev, int nc, const double* host);
    void cellsFromDev(double* host, const double* const* dev, int nc);
    double* ioStage_ = nullptr;  // 3 nC doubles
    int* dPerm_ = nullptr;       // perm_ on the device; null for the identity
    int deviceCell(int64_t c) const;
    std::vector<Vec> uVal_;
    std::vector<double> pVal_;
    std::map<int64_t, Vec> uFace_;
    bool bcDirty_ = true;
    cfg_schemes schemes_{CFG_DIV_UPWIND, 1, CFG_GRAD_CORRECTED, 0.9};

    // device BC tables
    double *uc_[3], *uk_[3], *hc_[3], *hk_[3], *pc_, *pk_;
    int64_t nFreeUFaces_ = 0;  // faces of patches whose U is not fixedValue

    // fields
    V3P U_, gPn_, gPF_, Hf_, gA_, gB_, uBase_, uRhs_, ux_;
    double *p_, *phi_, *rAUr_, *rAUf_, *uDiag_, *pDiag_, *pBase_, *pRhs_, *px_, *mVal_, *pVal_d_;
    double* gU_ = nullptr;   // harmonic face viscosity for the current nu
    double* fScratch_ = nullptr;  // nFaces
    double* bScratch_ = nullptr;  // 2 nBoundary
    double lastNu_ = -1.0;
    // adjustPhi addressing (patch ranges, which patches have a free U)
    int *dpStart_, *dpSize_, *dpFree_, *dFreeFace_, *dEmptyFace_;
    bool needReference_ = true;
    // solver work
    double *cr_, *cp_, *cAp_, *cz_;
    // mixed-precision Poisson solves
    float *pVal32_ = nullptr, *pDiag32_ = nullptr, *r32_, *p32_, *Ap32_, *z32_, *e32_, *b32_;
    DDicT<float> dic32_{};
    double *pb64_ = nullptr, *px64_ = nullptr;
    bool poissonReady_ = false;
    bool mixedReady_ = false;
    void ensureMixed();
    void runIR32(const double* vals, const double* diag, const double* b, double* x, double tol, int maxIter,
                 double innerTol, cfg_solver_report* rep);
    // multicolour DIC
    DDic dic_{};
    std::vector<DicPhase> dicPhase_;
    int nColours_ = 0, nLo_ = 0, nUp_ = 0, dicPartials_ = 1;
    V3P br_, br0_, bp_, bv_, bs_, bsh_, bt_, bz_;
    double* bInvD_ = nullptr;  // BiCGStab's Jacobi inverse diagonal
    double* partials_;
    SolveState* st_;
    SolveState* stHost_;
    double* scal_;      // device scalars of one outer iteration
    double* scalHost_;  // pinned copy
    Timing tm_{};
    int64_t launches_ = 0;
    bool ktime_ = false;
    bool useGraphs_ = true;
    // CHUANFLOW_PDL=1: the host-driven solver loops (AMG V-cycles, the AMG
    // flexible CG, the AMG-preconditioned BiCGStab) launch their kernels as
    // programmatic dependents of the kernel before.  Off by default: on the
    // 2M-cell channel it shortened the eagerly launched V-cycle's coarse part
    // (108.6 -> 94.7 us) but lengthened the graph-replayed outer iteration
    // (265.5 -> 269.9 ms), with the same results
    bool pdl_ = false;
    std::map<std::string, cudaGraphExec_t> graphs_;
    static constexpr int kEvPerIter = 12;  // events per solver iteration of a chunk (timed segments + 1)
    std::vector<cudaEvent_t> kev_;
    void tmark(int k, int j);
    void harvest(int ran, const int* slots, int nSlots, int active = 1);
};

}  // namespace cfg

namespace cfg
{

/// device memory owned by the context (zeroed), released in its destructor
template <class T>
T* Ctx::alloc(size_t n)
{
    void* p = nullptr;
    CFG_CUDA(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
    allocs_.push_back(p);
    CFG_CUDA(cudaMemsetAsync(p, 0, std::max<size_t>(n, 1) * sizeof(T), stream_));
    return static_cast<T*>(p);
}

template <class T>
T* Ctx::upload(const std::vector<T>& v)
{
    T* p = alloc<T>(v.size());
    if (!v.empty()) CFG_CUDA(cudaMemcpyAsync(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, stream_));
    return p;
}

}  // namespace cfg

struct cfg_ctx
{
    std::unique_ptr<cfg::Ctx> c;
};

namespace cfg
{
struct BatchGraph;
struct BatchGraphDeleter
{
    void operator()(BatchGraph* g) const;
};
}  // namespace cfg

struct cfg_batch
{
    std::vector<cfg::Ctx*> blocks;
    int workers = 1;    // 0: the whole pass as one captured CUDA graph
    int rowBlocks = 0;  // 0: each block's own solver grid
    std::unique_ptr<cfg::BatchGraph, cfg::BatchGraphDeleter> graph;
};

namespace cfg
{
void batchPass(cfg_batch& b, const double* q, const cfg_simple_controls* ctl, cfg_detail_measure* out,
               double* wallMs);
}
