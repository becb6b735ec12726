// solveCG / solveBiCGStab on a caller's CSR matrix (src/common/src/Matrix.cpp:153-319):
// the drop-in for the reference's linear-solver call surface.
#include <algorithm>
#include <type_traits>
#include <vector>

#include "ctx.h"
#include "solvers.cuh"

namespace cfg
{

namespace
{

struct DevBuf
{
    std::vector<void*> ptrs;
    cudaStream_t s;
    template <class T>
    T* get(size_t n)
    {
        void* p = nullptr;
        CFG_CUDA(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)));
        ptrs.push_back(p);
        CFG_CUDA(cudaMemsetAsync(p, 0, std::max<size_t>(n, 1) * sizeof(T), s));
        return static_cast<T*>(p);
    }
    ~DevBuf()
    {
        cudaStreamSynchronize(s);
        for (void* p : ptrs) cudaFree(p);
    }
};

__global__ void k_diag_from_sell(DMat A, const int* __restrict__ isDiag, const double* __restrict__ val, double* d)
{
    ROW_LOOP(c, A.n)
    {
        const int sl = c >> 5, lane = c & 31;
        double v = 0.0;
        for (int e = A.start[sl] + lane; e < A.start[sl + 1]; e += 32)
        {
            if (A.col[e] < 0) break;
            if (isDiag[e])
            {
                v = val[e];
                break;
            }
        }
        d[c] = v;
    }
}

}  // namespace

void Ctx::sparseSolve(int device, int64_t n64, const int64_t* rs, const int64_t* cols, const double* vals,
                      const double* b, double* x, double tol, int maxIter, int method, cfg_solver_report* rep)
{
    if (n64 <= 0 || n64 >= (1LL << 30)) fail(CFG_EINVAL, "sparse solve: matrix size out of range");
    const int n = static_cast<int>(n64);
    for (int r = 0; r < n; ++r)
    {
        if (rs[r + 1] < rs[r]) fail(CFG_EINVAL, "sparse solve: row offsets not ascending");
        for (int64_t k = rs[r]; k < rs[r + 1]; ++k)
            if (cols[k] < 0 || cols[k] >= n) fail(CFG_EINVAL, "sparse solve: column out of range");
    }
    CFG_CUDA(cudaSetDevice(device));
    cudaStream_t s;
    CFG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    struct StreamGuard
    {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } sg{s};
    DevBuf buf;
    buf.s = s;
    // SELL-32 with each row's entries in the caller's order
    const int nS = (n + 31) / 32;
    std::vector<int> start(nS + 1, 0);
    for (int sl = 0; sl < nS; ++sl)
    {
        int w = 0;
        for (int l = 0; l < 32 && 32 * sl + l < n; ++l) w = std::max<int>(w, static_cast<int>(rs[32 * sl + l + 1] - rs[32 * sl + l]));
        start[sl + 1] = start[sl] + 32 * w;
    }
    std::vector<int> col(start[nS], -1), isDiag(start[nS], 0);
    std::vector<double> val(start[nS], 0.0);
    std::vector<char> seenDiag(n, 0);
    for (int r = 0; r < n; ++r)
    {
        const int sl = r >> 5, l = r & 31;
        for (int64_t k = rs[r]; k < rs[r + 1]; ++k)
        {
            const int e = start[sl] + 32 * static_cast<int>(k - rs[r]) + l;
            col[e] = static_cast<int>(cols[k]);
            val[e] = vals[k];
            // SparseMatrix::diagonal takes the first entry in the diagonal column
            if (cols[k] == r && !seenDiag[r])
            {
                isDiag[e] = 1;
                seenDiag[r] = 1;
            }
        }
    }
    int sms = 0;
    CFG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device));
    const int G = std::max(1, std::min((n + TPB - 1) / TPB, sms * 8));
    const int GS = std::max(1, (n + RPT * TPB - 1) / (RPT * TPB));
    int maxW = 0;
    for (int sl = 0; sl < nS; ++sl) maxW = std::max(maxW, (start[sl + 1] - start[sl]) / 32);
    int* dStart = buf.get<int>(start.size());
    int* dCol = buf.get<int>(col.size());
    int* dIsDiag = buf.get<int>(isDiag.size());
    double* dVal = buf.get<double>(val.size());
    double* dDiag = buf.get<double>(n);
    double* db = buf.get<double>(n);
    double* dx = buf.get<double>(n);
    CFG_CUDA(cudaMemcpyAsync(dStart, start.data(), start.size() * sizeof(int), cudaMemcpyHostToDevice, s));
    CFG_CUDA(cudaMemcpyAsync(dCol, col.data(), col.size() * sizeof(int), cudaMemcpyHostToDevice, s));
    CFG_CUDA(cudaMemcpyAsync(dIsDiag, isDiag.data(), isDiag.size() * sizeof(int), cudaMemcpyHostToDevice, s));
    CFG_CUDA(cudaMemcpyAsync(dVal, val.data(), val.size() * sizeof(double), cudaMemcpyHostToDevice, s));
    CFG_CUDA(cudaMemcpyAsync(db, b, n * sizeof(double), cudaMemcpyHostToDevice, s));
    CFG_CUDA(cudaMemcpyAsync(dx, x, n * sizeof(double), cudaMemcpyHostToDevice, s));
    const DMat A{n, dStart, dCol};
    k_diag_from_sell<<<G, TPB, 0, s>>>(A, dIsDiag, dVal, dDiag);
    double* partials = buf.get<double>(16 * static_cast<size_t>(std::max(G, GS)));
    SolveState* st = buf.get<SolveState>(1);
    SolveState* hst = nullptr;
    CFG_CUDA(cudaMallocHost(&hst, sizeof(SolveState)));
    struct HostGuard
    {
        SolveState* p;
        ~HostGuard() { cudaFreeHost(p); }
    } hg{hst};
    SolveState init{};
    init.tol = tol;
    init.maxIter = maxIter;
    init.nComp = 1;
    CFG_CUDA(cudaMemcpyAsync(st, &init, sizeof(SolveState), cudaMemcpyHostToDevice, s));
    auto poll = [&]() {
        CFG_CUDA(cudaMemcpyAsync(hst, st, sizeof(SolveState), cudaMemcpyDeviceToHost, s));
        CFG_CUDA(cudaStreamSynchronize(s));
        return hst->allDone != 0;
    };
    auto run = [&](auto Wc) {
        constexpr int W = decltype(Wc)::value;
        if (method == CFG_SOLVE_CG)
        {
            double* r = buf.get<double>(n);
            double* p = buf.get<double>(n);
            double* Ap = buf.get<double>(n);
            k_cg_init<W><<<GS, TPB, 0, s>>>(A, dVal, dDiag, db, dx, r, p, partials, st);
            CFG_CUDA(cudaGetLastError());
            for (int launched = 0, chunk = 8; !poll() && launched < maxIter; chunk = std::min(2 * chunk, 64))
            {
                const int m = std::min(chunk, maxIter - launched);
                for (int k = 0; k < m; ++k)
                {
                    k_cg_spmv<W><<<GS, TPB, 0, s>>>(A, dVal, p, Ap, partials, st);
                    k_cg_update<double><<<GS, TPB, 0, s>>>(n, dDiag, p, Ap, dx, r, partials, st);
                    k_cg_p<double><<<GS, TPB, 0, s>>>(n, dDiag, r, p, st);
                }
                CFG_CUDA(cudaGetLastError());
                launched += m;
            }
        }
        else
        {
            V3P r{}, r0{}, p{}, v{}, t{}, z{}, bb{}, xx{};
            for (int q = 0; q < 3; ++q)
            {
                r.c[q] = buf.get<double>(n);
                r0.c[q] = buf.get<double>(n);
                p.c[q] = buf.get<double>(n);
                v.c[q] = buf.get<double>(n);
                t.c[q] = buf.get<double>(n);
                z.c[q] = buf.get<double>(n);
                bb.c[q] = db;
                xx.c[q] = dx;
            }
            double* invD = buf.get<double>(n);
            k_bi_init<W, 1><<<GS, TPB, 0, s>>>(A, dVal, dDiag, invD, bb, xx, r, r0, p, v, partials, st);
            CFG_CUDA(cudaGetLastError());
            for (int launched = 0, chunk = 4; !poll() && launched < maxIter; chunk = std::min(2 * chunk, 32))
            {
                const int m = std::min(chunk, maxIter - launched);
                for (int k = 0; k < m; ++k)
                {
                    k_bi_p<1><<<GS, TPB, 0, s>>>(n, invD, r, p, v, z, st);
                    k_bi_spmv1<W, 1><<<GS, TPB, 0, s>>>(A, dVal, z, v, r0, partials, st);
                    k_bi_spmv2<W, 1><<<GS, TPB, 0, s>>>(A, dVal, invD, r, v, t, partials, st);
                    k_bi_x<1><<<GS, TPB, 0, s>>>(n, invD, xx, z, v, t, r, r0, partials, st);
                }
                CFG_CUDA(cudaGetLastError());
                launched += m;
            }
        }
    };
    if (maxW <= 7) run(std::integral_constant<int, 7>{});
    else if (maxW <= 16) run(std::integral_constant<int, 16>{});
    else run(std::integral_constant<int, 0>{});
    CFG_CUDA(cudaMemcpyAsync(x, dx, n * sizeof(double), cudaMemcpyDeviceToHost, s));
    CFG_CUDA(cudaStreamSynchronize(s));
    rep->iterations = hst->it[0];
    rep->converged = hst->conv[0];
    rep->initial_residual = hst->init[0];
    rep->final_residual = (hst->conv[0] && hst->it[0] == 0) ? hst->init[0] : hst->fin[0];
}

}  // namespace cfg
