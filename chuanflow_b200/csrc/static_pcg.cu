// Jacobi-preconditioned CG on a caller's device CSR matrix, with every work
// vector in a fixed, file-scope device array instead of memory this library
// allocates.
//
// Who needs it: callers that must not allocate device memory while they run.
// A solver embedded in a larger simulation whose memory manager pre-reserves
// the whole GPU (a coupled 1D-3D network driver, a fixed-budget embedded
// deployment) cannot have a library call cudaMalloc behind its back, and
// cudaMalloc / cudaFree synchronise the device, which stalls every other
// stream of a caller that overlaps work.  cfg_pcg_solve_static runs the same
// algorithm as cfg_sparse_solve's CG (src/common/src/Matrix.cpp:153-222) on
// buffers the caller already owns, using only this file's static scratch.
//
// The scratch is a static __device__ array, so every GPU that loads the
// library holds it (about 8.5 MB) until the process exits.  On the host, the
// array's name is only a stand-in for the symbol, not a device address; the
// address is looked up once per device with cudaGetSymbolAddress and passed
// to the kernels.
#include <cstring>
#include <mutex>

#include "ctx.h"
#include "solvers.cuh"

namespace cfg
{
namespace
{

constexpr int kStaticMaxRows = 1 << 18;  // largest system the static scratch holds
constexpr int kStaticMaxBlocks = (kStaticMaxRows + RPT * TPB - 1) / (RPT * TPB);
constexpr size_t kVecBytes = sizeof(double) * kStaticMaxRows;
constexpr size_t kPartialBytes = sizeof(double) * 16 * kStaticMaxBlocks;
constexpr size_t kStateBytes = (sizeof(SolveState) + 255) / 256 * 256;
// layout: r, p, Ap, diag (one vector each), block partials, solver state
constexpr size_t kScratchBytes = 4 * kVecBytes + kPartialBytes + kStateBytes;

static __device__ __align__(256) unsigned char g_pcgScratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_setupMutex;
unsigned char* g_scratchAddr[kMaxDevices] = {};

/// The device address of g_pcgScratch on `device` (current), looked up on
/// the first call for that device and kept for the life of the process (a
/// cudaDeviceReset of the device would leave it stale; the header says so).
unsigned char* scratchOn(int device)
{
    std::lock_guard<std::mutex> lock(g_setupMutex);
    if (!g_scratchAddr[device])
    {
        void* ptr = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&ptr, g_pcgScratch);
        if (e != cudaSuccess)
            fail(CFG_ECUDA, std::string("cfg_pcg_solve_static: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_scratchAddr[device] = static_cast<unsigned char*>(ptr);
    }
    return g_scratchAddr[device];
}

/// Every field of the solver state cleared (tickets, flags, counters), then
/// the tolerance and iteration limit set: the array keeps the previous
/// call's contents.
__global__ void k_static_state_init(SolveState* st, double tol, int maxIter)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    unsigned char* b = reinterpret_cast<unsigned char*>(st);
    for (size_t i = 0; i < sizeof(SolveState); ++i) b[i] = 0;
    st->tol = tol;
    st->maxIter = maxIter;
    st->nComp = 1;
}

/// One CSR row of A x, columns in the row's order (SparseMatrix::product,
/// Matrix.cpp:119-133), and the row's diagonal (SparseMatrix::diagonal,
/// Matrix.cpp:135-151: the first entry in the diagonal column, else 0).
__device__ __forceinline__ double csr_row(const int* __restrict__ rs, const int* __restrict__ cols,
                                          const double* __restrict__ vals, const double* __restrict__ x, int r,
                                          double* diag)
{
    double s = 0.0;
    bool seen = false;
    const int k1 = rs[r + 1];
    for (int k = rs[r]; k < k1; ++k)
    {
        const int c = cols[k];
        const double v = vals[k];
        if (c == r && !seen && diag)
        {
            *diag = v;
            seen = true;
        }
        s += v * x[c];
    }
    if (diag && !seen) *diag = 0.0;
    return s;
}

__global__ void __launch_bounds__(TPB) k_static_cg_init(int n, const int* __restrict__ rs, const int* __restrict__ cols,
                                                        const double* __restrict__ vals, const double* __restrict__ b,
                                                        const double* __restrict__ x, double* __restrict__ r,
                                                        double* __restrict__ p, double* __restrict__ d,
                                                        double* partials, SolveState* st)
{
    double mx[3] = {0.0, 0.0, 0.0};
    double sm[1] = {0.0};
    FOR_ROWS(c, n)
    {
        double dc;
        const double y = csr_row(rs, cols, vals, x, c, &dc);
        d[c] = dc;
        const double bi = b[c];
        const double ri = bi - y;
        r[c] = ri;
        const double zi = inv_diag_cg(dc) * ri;
        p[c] = zi;
        if (isnan(ri) || isnan(bi)) mx[2] = 1.0;
        mx[0] = smax(mx[0], fabs(ri));
        mx[1] = smax(mx[1], fabs(bi));
        sm[0] += ri * zi;
    }
    block_max<3>(mx);
    __syncthreads();
    block_sum<1>(sm);
    const int G = gridDim.x;
    if (threadIdx.x == 0)
    {
        partials[blockIdx.x] = mx[0];
        partials[G + blockIdx.x] = mx[1];
        partials[2 * G + blockIdx.x] = mx[2];
        partials[3 * G + blockIdx.x] = sm[0];
    }
    if (!last_block(&st->ticket[0])) return;
    double fm[3], fs[1];
    final_max<3>(partials, G, fm);
    __syncthreads();
    final_sum<1>(partials + 3 * G, G, fs);
    if (threadIdx.x == 0)
    {
        st->ticket[0] = 0;
        const double init = fm[2] > 0 ? NAN : fm[0];
        const double bn = smax(fm[1], 1e-300);
        st->init[0] = init;
        st->bnorm[0] = bn;
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

__global__ void __launch_bounds__(TPB) k_static_cg_spmv(int n, const int* __restrict__ rs, const int* __restrict__ cols,
                                                        const double* __restrict__ vals, const double* __restrict__ p,
                                                        double* __restrict__ Ap, double* partials, SolveState* st)
{
    if (st->allDone) return;
    double sm[1] = {0.0};
    FOR_ROWS(c, n)
    {
        const double y = csr_row(rs, cols, vals, p, c, nullptr);
        Ap[c] = y;
        sm[0] += p[c] * y;
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
        st->pAp[0] = pAp;
        if (pAp <= 0 || fabs(st->rz[0]) < 1e-300)
        {
            st->done[0] = 1;
            st->allDone = 1;
        }
        else
        {
            st->alpha[0] = st->rz[0] / pAp;
        }
    }
}

}  // namespace
}  // namespace cfg

extern "C" int cfg_pcg_solve_static(int32_t device, int64_t n64, const int32_t* rowStart, const int32_t* cols,
                                    const double* vals, const double* b, double* x, double tol, int32_t maxIter,
                                    void* stream, cfg_solver_report* report)
{
    using namespace cfg;
    int prev = -1;
    bool switched = false;
    try
    {
        if (!rowStart || !cols || !vals || !b || !x || !report)
            fail(CFG_EINVAL, "cfg_pcg_solve_static: null argument");
        if (n64 <= 0 || n64 > kStaticMaxRows)
            fail(CFG_EINVAL, "cfg_pcg_solve_static: " + std::to_string(n64) + " rows; the static scratch holds 1.." +
                                 std::to_string(kStaticMaxRows));
        if (device < 0 || device >= kMaxDevices) fail(CFG_EINVAL, "cfg_pcg_solve_static: device out of range");
        if (maxIter < 0) fail(CFG_EINVAL, "cfg_pcg_solve_static: negative iteration limit");
        const int n = static_cast<int>(n64);
        CFG_CUDA(cudaGetDevice(&prev));
        if (prev != device)
        {
            CFG_CUDA(cudaSetDevice(device));
            switched = true;
        }
        unsigned char* base = scratchOn(device);
        double* r = reinterpret_cast<double*>(base);
        double* p = reinterpret_cast<double*>(base + kVecBytes);
        double* Ap = reinterpret_cast<double*>(base + 2 * kVecBytes);
        double* d = reinterpret_cast<double*>(base + 3 * kVecBytes);
        double* partials = reinterpret_cast<double*>(base + 4 * kVecBytes);
        SolveState* st = reinterpret_cast<SolveState*>(base + 4 * kVecBytes + kPartialBytes);
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        const int G = (n + RPT * TPB - 1) / (RPT * TPB);
        k_static_state_init<<<1, 1, 0, s>>>(st, tol, maxIter);
        k_static_cg_init<<<G, TPB, 0, s>>>(n, rowStart, cols, vals, b, x, r, p, d, partials, st);
        CFG_CUDA(cudaGetLastError());
        int allDone = 0;
        for (int launched = 0, chunk = 8;; chunk = std::min(2 * chunk, 64))
        {
            CFG_CUDA(cudaMemcpyAsync(&allDone, &st->allDone, sizeof(int), cudaMemcpyDeviceToHost, s));
            CFG_CUDA(cudaStreamSynchronize(s));
            if (allDone || launched >= maxIter) break;
            const int m = std::min(chunk, maxIter - launched);
            for (int k = 0; k < m; ++k)
            {
                k_static_cg_spmv<<<G, TPB, 0, s>>>(n, rowStart, cols, vals, p, Ap, partials, st);
                k_cg_update<double><<<G, TPB, 0, s>>>(n, d, p, Ap, x, r, partials, st);
                k_cg_p<double><<<G, TPB, 0, s>>>(n, d, r, p, st);
            }
            CFG_CUDA(cudaGetLastError());
            launched += m;
        }
        SolveState h;
        CFG_CUDA(cudaMemcpyAsync(&h, st, sizeof(SolveState), cudaMemcpyDeviceToHost, s));
        CFG_CUDA(cudaStreamSynchronize(s));
        report->iterations = h.it[0];
        report->converged = h.conv[0];
        report->initial_residual = h.init[0];
        report->final_residual = (h.conv[0] && h.it[0] == 0) ? h.init[0] : h.fin[0];
        if (switched) cudaSetDevice(prev);
        return CFG_OK;
    }
    catch (const Error& e)
    {
        if (switched) cudaSetDevice(prev);
        setLastError(e.what());
        return e.code;
    }
    catch (const std::exception& e)
    {
        if (switched) cudaSetDevice(prev);
        setLastError(e.what());
        return CFG_EINVAL;
    }
}
