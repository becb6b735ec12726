// A message-passing network on the cell-face graph of the pressure matrix,
// trained on the device by this file's forward and backward kernels and
// used as the preconditioner of a flexible CG (no reference counterpart:
// the reference's pressure solve is Jacobi-PCG, Matrix.cpp:153-222).
//
// The network maps a residual r to a correction z = M(r):
//   s      = rms(r)                      (scale: M(a r) = a M(r))
//   h0_i   = relu(w0 (r_i / s) + b0)                           width H = 32
//   m_i    = sum_j c_ij h_j,   c_ij = -a_ij / a_ii             (one hop)
//   h_i   <- h_i + relu(A h_i + B m_i + b)                     L layers
//   z_i    = r_i / a_ii + s (wout . h_i)
// so an untrained network (wout = 0) is the Jacobi preconditioner.  Weights
// are kept in FP32 (the optimiser's master copy) and used rounded to BF16;
// activations and accumulations are FP32.  Training minimises
// |A M(r) - r|^2 / |r|^2 over residual samples with Adam; the gradient is
// with respect to the BF16 weights, applied to the FP32 master.
//
// Device layout: hidden states are FP32 rows of 32 (one 128-byte line per
// cell).  A layer's warp takes 16 cells at a time: lane k gathers channel k
// of each cell's state and message (one coalesced line per neighbour), the
// 16 x 64 block [h | m] is rounded to BF16 in shared memory, and the 32 x 64
// contraction with [A | B] runs on the tensor cores (mma.sync m16n8k16,
// BF16 operands, FP32 accumulation).  The backward kernels use the same
// BF16-rounded operands for the weight gradients and pass gradients through
// the rounding unchanged.
#include <cuda_bf16.h>

#include <cmath>
#include <cstring>

#include "ctx.h"
#include "kernels.cuh"

namespace cfg
{

namespace
{

constexpr int H = 32;           // hidden width
constexpr int WP = H + 1;       // padded shared-memory row
constexpr int kWarps = 8;       // warps per block
constexpr int kMaxRow = 64;     // row entries a warp walks (the SELL rows are far shorter)

/// parameter offsets (floats): w0[H], b0[H], then per layer A[H*H], B[H*H],
/// b[H], then wout[H]
__host__ __device__ constexpr int offLayer(int l) { return 2 * H + l * (2 * H * H + H); }
__host__ __device__ constexpr int nParams(int L) { return offLayer(L) + H; }

struct Row
{
    int e0, e1;  // slot range of the SELL row (stride 32)
};

__device__ __forceinline__ Row sell_row(const DMat& A, int i)
{
    const int sl = i >> 5, l = i & 31;
    return Row{A.start[sl] + l, A.start[sl + 1]};
}

/// The message coefficients c_ij = -a_ij / a_ii of every off-diagonal SELL
/// entry (row i), in FP32, once per matrix; 0 on the diagonal and the pads.
__global__ void __launch_bounds__(TPB) k_mpnn_coef(DMat A, const double* __restrict__ val,
                                                   const double* __restrict__ diag, float* __restrict__ coef)
{
    FOR_ROWS(i, A.n)
    {
        const int sl = i >> 5, l = i & 31;
        const double aii = diag[i];
        for (int e = A.start[sl] + l; e < A.start[sl + 1]; e += 32)
        {
            const int j = A.col[e];
            coef[e] = (j < 0 || j == i) ? 0.f : static_cast<float>(-val[e] / aii);
        }
    }
}

/// m_k = sum_j c_ij x[j*H + k] over the off-diagonal entries of row i
__device__ __forceinline__ float message(const DMat& A, const float* __restrict__ coef, const float* __restrict__ x,
                                         int i, int lane)
{
    const Row r = sell_row(A, i);
    float m = 0.f;
    for (int e = r.e0; e < r.e1; e += 32)
    {
        const int j = __ldg(A.col + e);
        if (j < 0) break;
        if (j == i) continue;
        m += __ldg(coef + e) * x[static_cast<size_t>(j) * H + lane];
    }
    return m;
}

__global__ void k_mpnn_round(int n, const float* __restrict__ w, __nv_bfloat16* __restrict__ wb)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) wb[i] = __float2bfloat16(w[i]);
}

/// h0 = relu(w0 x + b0), x_i = r_i / s
__global__ void __launch_bounds__(kWarps * 32) k_mpnn_enc(int n, const double* __restrict__ r, const double* sInv,
                                                          const __nv_bfloat16* __restrict__ wb, float* __restrict__ h0,
                                                          unsigned* __restrict__ mask)
{
    const int lane = threadIdx.x & 31;
    const float w = __bfloat162float(wb[lane]), b = __bfloat162float(wb[H + lane]);
    const double si = *sInv;
    const int warp = blockIdx.x * kWarps + (threadIdx.x >> 5), nw = gridDim.x * kWarps;
    for (int i = warp; i < n; i += nw)
    {
        const float x = static_cast<float>(r[i] * si);
        const float u = w * x + b;
        h0[static_cast<size_t>(i) * H + lane] = u > 0.f ? u : 0.f;
        const unsigned bits = __ballot_sync(0xffffffffu, u > 0.f);
        if (lane == 0) mask[i] = bits;
    }
}

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16(x)); }

__device__ __forceinline__ uint32_t ld_pair(const __nv_bfloat16* p)
{
    return *reinterpret_cast<const uint32_t*>(p);
}

/// D (16x8, FP32) += A (16x16, BF16, row) * B (16x8, BF16, col)
__device__ __forceinline__ void mma_bf16_16816(float (&d)[4], uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3,
                                               uint32_t b0, uint32_t b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

constexpr int XP = 2 * H + 8;  // padded BF16 row of [h | m] and of the weights (144 bytes)
constexpr int kSlots = 8;      // entry slots a SELL slice may have for the staged message path

/// one residual message-passing layer: hout = hin + relu(A h + B m + b) for
/// 16 cells per warp step, the contraction on the tensor cores.  The 16
/// cells of a step are consecutive rows of one SELL slice: their entries
/// (column, coefficient) are loaded two slots per warp-wide load into shared
/// memory first, so the neighbour-state gathers of all 16 cells are
/// independent of each other and issue back to back (lane k gathers
/// channel k of each neighbour: one 128-byte line per neighbour).
__global__ void __launch_bounds__(kWarps * 32) k_mpnn_layer(DMat A, const float* __restrict__ coef,
                                                            const __nv_bfloat16* __restrict__ wl,
                                                            const float* __restrict__ hin, float* __restrict__ hout,
                                                            unsigned* __restrict__ mask)
{
    // sW[o][k]: output unit o, input k (k < 32: A, k >= 32: B)
    __shared__ __align__(16) __nv_bfloat16 sW[H][XP];
    __shared__ float sb[H];
    __shared__ __align__(16) __nv_bfloat16 sX[kWarps][16][XP];
    __shared__ float sU[kWarps][16][H + 1];
    // the step's row entries: slot k of cell t at [k][t] (column; -1 for a
    // pad, the diagonal or a cell past the end), coefficient beside it
    __shared__ int2 sE[kWarps][kSlots][16];
    for (int t = threadIdx.x; t < H * H; t += blockDim.x)
    {
        const int o = t / H, k = t % H;
        sW[o][k] = wl[t];
        sW[o][H + k] = wl[H * H + t];
    }
    for (int t = threadIdx.x; t < H; t += blockDim.x) sb[t] = __bfloat162float(wl[2 * H * H + t]);
    __syncthreads();
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int gid = lane >> 2, tig = lane & 3;
    const int groups = (A.n + 15) / 16;
    for (int g = blockIdx.x * kWarps + w; g < groups; g += gridDim.x * kWarps)
    {
        const int c0 = g * 16;
        const int s0 = __ldg(A.start + (c0 >> 5)), nSlots = (__ldg(A.start + (c0 >> 5) + 1) - s0) >> 5;
        float hr[16];
        if (nSlots <= kSlots)
        {
            const int t = lane & 15, i = c0 + t;
            for (int k = lane >> 4; k < nSlots; k += 2)
            {
                const int e = s0 + (c0 & 31) + t + 32 * k;
                int j = __ldg(A.col + e);
                if (i >= A.n || j == i) j = -1;
                sE[w][k][t] = make_int2(j, __float_as_int(__ldg(coef + e)));
            }
            __syncwarp();
            float m[16];
#pragma unroll
            for (int t2 = 0; t2 < 16; ++t2)
            {
                hr[t2] = c0 + t2 < A.n ? hin[static_cast<size_t>(c0 + t2) * H + lane] : 0.f;
                m[t2] = 0.f;
            }
            // slot by slot, the same order as message(): the gathers of the
            // 16 cells in one slot are independent
            for (int k = 0; k < nSlots; ++k)
            {
#pragma unroll
                for (int t2 = 0; t2 < 16; ++t2)
                {
                    const int2 p = sE[w][k][t2];
                    if (p.x >= 0) m[t2] += __int_as_float(p.y) * hin[static_cast<size_t>(p.x) * H + lane];
                }
            }
#pragma unroll
            for (int t2 = 0; t2 < 16; ++t2)
            {
                sX[w][t2][lane] = __float2bfloat16(hr[t2]);
                sX[w][t2][H + lane] = __float2bfloat16(m[t2]);
            }
        }
        else
        {
#pragma unroll
            for (int t = 0; t < 16; ++t)
            {
                const int i = c0 + t;
                float h = 0.f, m = 0.f;
                if (i < A.n)
                {
                    h = hin[static_cast<size_t>(i) * H + lane];
                    m = message(A, coef, hin, i, lane);
                }
                hr[t] = h;
                sX[w][t][lane] = __float2bfloat16(h);
                sX[w][t][H + lane] = __float2bfloat16(m);
            }
        }
        __syncwarp();
        float d[4][4] = {};
#pragma unroll
        for (int ks = 0; ks < 4; ++ks)
        {
            const int k0 = ks * 16 + tig * 2;
            const uint32_t a0 = ld_pair(&sX[w][gid][k0]), a1 = ld_pair(&sX[w][gid + 8][k0]);
            const uint32_t a2 = ld_pair(&sX[w][gid][k0 + 8]), a3 = ld_pair(&sX[w][gid + 8][k0 + 8]);
#pragma unroll
            for (int nt = 0; nt < 4; ++nt)
            {
                const int o = nt * 8 + gid;
                mma_bf16_16816(d[nt], a0, a1, a2, a3, ld_pair(&sW[o][k0]), ld_pair(&sW[o][k0 + 8]));
            }
        }
#pragma unroll
        for (int nt = 0; nt < 4; ++nt)
#pragma unroll
            for (int j = 0; j < 4; ++j)
            {
                const int row = gid + (j >> 1) * 8, col = nt * 8 + tig * 2 + (j & 1);
                sU[w][row][col] = d[nt][j] + sb[col];
            }
        __syncwarp();
#pragma unroll
        for (int t = 0; t < 16; ++t)
        {
            const int i = c0 + t;
            const float u = sU[w][t][lane];
            const unsigned bits = __ballot_sync(0xffffffffu, u > 0.f);
            if (i < A.n)
            {
                hout[static_cast<size_t>(i) * H + lane] = hr[t] + (u > 0.f ? u : 0.f);
                if (lane == 0) mask[i] = bits;
            }
        }
        __syncwarp();
    }
}

/// z_i = r_i / a_ii + s (wout . h_i)
__global__ void __launch_bounds__(kWarps * 32) k_mpnn_out(int n, const double* __restrict__ r,
                                                          const double* __restrict__ diag, const double* s,
                                                          const __nv_bfloat16* __restrict__ wout,
                                                          const float* __restrict__ h, double* __restrict__ z)
{
    const int lane = threadIdx.x & 31;
    const float w = __bfloat162float(wout[lane]);
    const double sc = *s;
    const int warp = blockIdx.x * kWarps + (threadIdx.x >> 5), nw = gridDim.x * kWarps;
    for (int i = warp; i < n; i += nw)
    {
        float v = w * h[static_cast<size_t>(i) * H + lane];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) z[i] = r[i] / diag[i] + sc * static_cast<double>(v);
    }
}

/// s = sqrt(sum r^2 / n), 1/s and sum r^2: block partials, then the block
/// that finishes last sums them in a fixed order
__global__ void __launch_bounds__(TPB) k_mpnn_scale(int n, const double* __restrict__ r, double* partials,
                                                    unsigned* ticket, double* s)
{
    double v[1] = {0.0};
    FOR_ROWS(i, n) v[0] += r[i] * r[i];
    block_sum<1>(v);
    if (threadIdx.x == 0) partials[blockIdx.x] = v[0];
    if (!last_block(ticket)) return;
    double f[1];
    final_sum<1>(partials, gridDim.x, f);
    if (threadIdx.x == 0)
    {
        *ticket = 0;
        const double rms = sqrt(f[0] / n);
        s[0] = rms;
        s[1] = rms > 0 ? 1.0 / rms : 0.0;
        s[2] = f[0];
    }
}

/// res = A z - r (FP64), and |res|^2 into acc[0] (atomic, for the loss)
template <int W>
__global__ void __launch_bounds__(TPB) k_mpnn_resid(DMat A, const double* __restrict__ val,
                                                    const double* __restrict__ z, const double* __restrict__ r,
                                                    double* __restrict__ res, double* acc)
{
    double sm[1] = {0.0};
    const double* xs[1] = {z};
    FOR_ROWS(c, A.n)
    {
        double y[1];
        spmv_row<W, 1>(A, val, c, xs, y);
        const double v = y[0] - r[c];
        res[c] = v;
        sm[0] += v * v;
    }
    block_sum<1>(sm);
    if (threadIdx.x == 0) atomicAdd(acc, sm[0]);
}

/// the output gradient dL/dh_i = s g_i wout with g = 2 A res / rr (rr: |r|^2
/// for the residual loss, t.At for the energy-norm loss), and the wout
/// gradient sum_i s g_i h_i
template <int W>
__global__ void __launch_bounds__(kWarps * 32) k_mpnn_out_bwd(DMat A, const double* __restrict__ val,
                                                              const double* __restrict__ res, const double* s,
                                                              const double* rrp,
                                                              const __nv_bfloat16* __restrict__ wout,
                                                              const float* __restrict__ h, float* __restrict__ dh,
                                                              float* __restrict__ gwout)
{
    __shared__ float sg[H];
    if (threadIdx.x < H) sg[threadIdx.x] = 0.f;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const float w = __bfloat162float(wout[lane]);
    const double sc = s[0], rr = *rrp;
    const int warp = blockIdx.x * kWarps + (threadIdx.x >> 5), nw = gridDim.x * kWarps;
    float acc = 0.f;
    const double* xs[1] = {res};
    for (int i = warp; i < A.n; i += nw)
    {
        double y = 0.0;
        if (lane == 0)
        {
            double yy[1];
            spmv_row<W, 1>(A, val, i, xs, yy);
            y = yy[0];
        }
        y = __shfl_sync(0xffffffffu, y, 0);
        const float g = static_cast<float>(sc * 2.0 * y / rr);
        dh[static_cast<size_t>(i) * H + lane] = g * w;
        acc += g * h[static_cast<size_t>(i) * H + lane];
    }
    atomicAdd(&sg[lane], acc);
    __syncthreads();
    if (threadIdx.x < H) atomicAdd(&gwout[threadIdx.x], sg[threadIdx.x]);
}

/// backward of one layer, part 1: delta = dh (.) relu'(u); weight gradients;
/// dhin = dh + A^T delta (the residual path plus the self transform); v =
/// B^T delta for the transposed message of part 2
__global__ void __launch_bounds__(kWarps * 32) k_mpnn_layer_bwd(DMat A, const float* __restrict__ coef,
                                                                const __nv_bfloat16* __restrict__ wl,
                                                                const float* __restrict__ hin,
                                                                const unsigned* __restrict__ mask,
                                                                const float* __restrict__ dh, float* __restrict__ dhin,
                                                                float* __restrict__ v, float* __restrict__ gl)
{
    __shared__ float sA[H * WP], sB[H * WP];
    __shared__ float gA[H * WP], gB[H * WP], gb[H];
    for (int t = threadIdx.x; t < H * H; t += blockDim.x)
    {
        const int k = t / H, q = t % H;
        sA[k * WP + q] = __bfloat162float(wl[t]);
        sB[k * WP + q] = __bfloat162float(wl[H * H + t]);
        gA[k * WP + q] = 0.f;
        gB[k * WP + q] = 0.f;
    }
    if (threadIdx.x < H) gb[threadIdx.x] = 0.f;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int warp = blockIdx.x * kWarps + (threadIdx.x >> 5), nw = gridDim.x * kWarps;
    float rA[H], rB[H], rb = 0.f;  // lane k: row k of the weight gradients
#pragma unroll
    for (int q = 0; q < H; ++q) rA[q] = rB[q] = 0.f;
    for (int i = warp; i < A.n; i += nw)
    {
        const size_t o = static_cast<size_t>(i) * H + lane;
        // the operands the forward multiplied: h and m rounded to BF16
        const float h = bf16r(hin[o]);
        const float m = bf16r(message(A, coef, hin, i, lane));
        const float d = (mask[i] >> lane) & 1u ? dh[o] : 0.f;
        rb += d;
        float at = 0.f, bt = 0.f;
#pragma unroll
        for (int q = 0; q < H; ++q)
        {
            const float hq = __shfl_sync(0xffffffffu, h, q);
            const float mq = __shfl_sync(0xffffffffu, m, q);
            const float dq = __shfl_sync(0xffffffffu, d, q);
            rA[q] += d * hq;
            rB[q] += d * mq;
            at += sA[q * WP + lane] * dq;  // (A^T d)_lane
            bt += sB[q * WP + lane] * dq;  // (B^T d)_lane
        }
        dhin[o] = dh[o] + at;
        v[o] = bt;
    }
#pragma unroll
    for (int q = 0; q < H; ++q)
    {
        atomicAdd(&gA[lane * WP + q], rA[q]);
        atomicAdd(&gB[lane * WP + q], rB[q]);
    }
    atomicAdd(&gb[lane], rb);
    __syncthreads();
    for (int t = threadIdx.x; t < H * H; t += blockDim.x)
    {
        const int k = t / H, q = t % H;
        atomicAdd(&gl[t], gA[k * WP + q]);
        atomicAdd(&gl[H * H + t], gB[k * WP + q]);
    }
    if (threadIdx.x < H) atomicAdd(&gl[2 * H * H + threadIdx.x], gb[threadIdx.x]);
}

/// backward of one layer, part 2: dhin_j += sum_{i in N(j)} c_ij v_i with
/// c_ij = -a_ij / a_ii = -a_ji / a_ii (the pressure matrix is symmetric)
__global__ void __launch_bounds__(kWarps * 32) k_mpnn_msg_bwd(DMat A, const double* __restrict__ val,
                                                              const double* __restrict__ diag,
                                                              const float* __restrict__ v, float* __restrict__ dhin)
{
    const int lane = threadIdx.x & 31;
    const int warp = blockIdx.x * kWarps + (threadIdx.x >> 5), nw = gridDim.x * kWarps;
    for (int j = warp; j < A.n; j += nw)
    {
        const Row r = sell_row(A, j);
        float acc = 0.f;
        for (int e = r.e0; e < r.e1; e += 32)
        {
            const int i = A.col[e];
            if (i < 0) break;
            if (i == j) continue;
            const float c = static_cast<float>(-val[e] / diag[i]);
            acc += c * v[static_cast<size_t>(i) * H + lane];
        }
        dhin[static_cast<size_t>(j) * H + lane] += acc;
    }
}

/// the encoder's gradient: d = dh0 (.) relu'; gw0 += d x, gb0 += d
__global__ void __launch_bounds__(kWarps * 32) k_mpnn_enc_bwd(int n, const double* __restrict__ r, const double* sInv,
                                                              const unsigned* __restrict__ mask,
                                                              const float* __restrict__ dh, float* __restrict__ g)
{
    __shared__ float s0[H], s1[H];
    if (threadIdx.x < H) s0[threadIdx.x] = s1[threadIdx.x] = 0.f;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const double si = *sInv;
    const int warp = blockIdx.x * kWarps + (threadIdx.x >> 5), nw = gridDim.x * kWarps;
    float aw = 0.f, ab = 0.f;
    for (int i = warp; i < n; i += nw)
    {
        const float d = (mask[i] >> lane) & 1u ? dh[static_cast<size_t>(i) * H + lane] : 0.f;
        aw += d * static_cast<float>(r[i] * si);
        ab += d;
    }
    atomicAdd(&s0[lane], aw);
    atomicAdd(&s1[lane], ab);
    __syncthreads();
    if (threadIdx.x < H)
    {
        atomicAdd(&g[threadIdx.x], s0[threadIdx.x]);
        atomicAdd(&g[H + threadIdx.x], s1[threadIdx.x]);
    }
}

/// Adam (Kingma & Ba 2015) on the FP32 master weights, then their BF16 copy
__global__ void k_mpnn_adam(int n, float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m1,
                            float* __restrict__ m2, float lr, float c1, float c2, __nv_bfloat16* __restrict__ wb)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    {
        const float gi = g[i];
        const float a = 0.9f * m1[i] + 0.1f * gi;
        const float b = 0.999f * m2[i] + 0.001f * gi * gi;
        m1[i] = a;
        m2[i] = b;
        w[i] -= lr * (a / c1) / (sqrtf(b / c2) + 1e-8f);
        wb[i] = __float2bfloat16(w[i]);
    }
}

/// dot products of NP vector pairs: block partials, then a last-block sum
/// into out (fixed order)
template <int NP>
__global__ void __launch_bounds__(TPB) k_fcg_dots(int n, const double* const* a, const double* const* b,
                                                  double* partials, unsigned* ticket, double* out)
{
    double sm[NP];
#pragma unroll
    for (int q = 0; q < NP; ++q) sm[q] = 0.0;
    FOR_ROWS(c, n)
    {
#pragma unroll
        for (int q = 0; q < NP; ++q) sm[q] += a[q][c] * b[q][c];
    }
    block_sum<NP>(sm);
    const int G = gridDim.x;
    if (threadIdx.x == 0)
#pragma unroll
        for (int q = 0; q < NP; ++q) partials[q * G + blockIdx.x] = sm[q];
    if (!last_block(ticket)) return;
    double fs[NP];
    final_sum<NP>(partials, G, fs);
    if (threadIdx.x == 0)
    {
        *ticket = 0;
#pragma unroll
        for (int q = 0; q < NP; ++q) out[q] = fs[q];
    }
}

/// max |a| (non-negative, order-free) into out
__global__ void __launch_bounds__(TPB) k_fcg_absmax(int n, const double* __restrict__ a, double* out)
{
    double v[1] = {0.0};
    FOR_ROWS(c, n) v[0] = smax(v[0], fabs(a[c]));
    block_max<1>(v);
    if (threadIdx.x == 0) atomic_max_nonneg(out, v[0]);
}

/// y = x + a p (x may alias y)
__global__ void __launch_bounds__(TPB) k_fcg_axpy(int n, double a, const double* __restrict__ p, double* y)
{
    FOR_ROWS(c, n) y[c] = y[c] + a * p[c];
}

/// p = z + beta p
__global__ void __launch_bounds__(TPB) k_fcg_p(int n, const double* __restrict__ z, double beta, double* p)
{
    FOR_ROWS(c, n) p[c] = z[c] + beta * p[c];
}

/// y = A x
template <int W>
__global__ void __launch_bounds__(TPB) k_fcg_spmv(DMat A, const double* __restrict__ val, const double* __restrict__ x,
                                                  double* __restrict__ y)
{
    const double* xs[1] = {x};
    FOR_ROWS(c, A.n)
    {
        double v[1];
        spmv_row<W, 1>(A, val, c, xs, v);
        y[c] = v[0];
    }
}

uint64_t mix64(uint64_t x)
{
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}

}  // namespace

struct MpnnState
{
    int L = 4, P = 0, n = 0;
    float *w = nullptr, *g = nullptr, *m1 = nullptr, *m2 = nullptr;
    __nv_bfloat16* wb = nullptr;
    float *h = nullptr, *dh0 = nullptr, *dh1 = nullptr, *v = nullptr;  // h: (L+1) n H
    unsigned* mask = nullptr;                                         // (L+1) n
    double *s = nullptr, *res = nullptr, *acc = nullptr;
    double *ae = nullptr, *at = nullptr;  // A e and A t of the energy-norm loss
    unsigned* ticket = nullptr;
    float* coef = nullptr;  // message coefficients, one per SELL entry
    int step = 0;
};

void MpnnDeleter::operator()(MpnnState* m) const { delete m; }

void Ctx::mpnnCreate(int layers, uint64_t seed)
{
    CFG_CUDA(cudaSetDevice(device_));
    if (layers < 1 || layers > 16) fail(CFG_EINVAL, "mpnn: 1..16 layers");
    if (maxW_ > kMaxRow) fail(CFG_EINVAL, "mpnn: matrix rows too wide");
    std::unique_ptr<MpnnState> m(new MpnnState());
    m->L = layers;
    m->P = nParams(layers);
    m->n = dm_.nC;
    // He-style initial weights from a counter hash; wout = 0 (Jacobi)
    std::vector<float> w(static_cast<size_t>(m->P), 0.f);
    auto uni = [&](uint64_t k) { return static_cast<float>((mix64(seed * 0x100000001B3ULL + k) >> 11) * 0x1.0p-53) * 2.f - 1.f; };
    for (int k = 0; k < H; ++k) w[k] = uni(k) * 1.0f;
    for (int l = 0; l < layers; ++l)
    {
        const int o = offLayer(l);
        const float sc = std::sqrt(3.0f / H) * 0.5f;
        for (int t = 0; t < 2 * H * H; ++t) w[o + t] = uni(1000 + l * 10000 + t) * sc;
    }
    m->w = upload(w);
    m->g = alloc<float>(m->P);
    m->m1 = alloc<float>(m->P);
    m->m2 = alloc<float>(m->P);
    CFG_CUDA(cudaMemsetAsync(m->m1, 0, m->P * sizeof(float), stream_));
    CFG_CUDA(cudaMemsetAsync(m->m2, 0, m->P * sizeof(float), stream_));
    m->wb = alloc<__nv_bfloat16>(m->P);
    k_mpnn_round<<<32, 256, 0, stream_>>>(m->P, m->w, m->wb);
    const size_t nH = static_cast<size_t>(m->n) * H;
    m->h = alloc<float>((layers + 1) * nH);
    m->dh0 = alloc<float>(nH);
    m->dh1 = alloc<float>(nH);
    m->v = alloc<float>(nH);
    m->mask = alloc<unsigned>(static_cast<size_t>(layers + 1) * m->n);
    m->s = alloc<double>(4);
    m->res = alloc<double>(m->n);
    m->ticket = alloc<unsigned>(1);
    m->coef = alloc<float>(static_cast<size_t>(nSlicesEntries_));
    m->ae = alloc<double>(m->n);
    m->at = alloc<double>(m->n);
    m->acc = alloc<double>(1);
    launchCheck("mpnn_init");
    mpnn_.reset(m.release());
    CFG_CUDA(cudaStreamSynchronize(stream_));
}

void Ctx::mpnnWeights(float* get, const float* set, int64_t n)
{
    if (!mpnn_) fail(CFG_EINVAL, "mpnn: call cfg_mpnn_create first");
    MpnnState& m = *mpnn_;
    if (n != m.P) fail(CFG_EINVAL, "mpnn: " + std::to_string(m.P) + " parameters, not " + std::to_string(n));
    if (set)
    {
        CFG_CUDA(cudaMemcpyAsync(m.w, set, n * sizeof(float), cudaMemcpyHostToDevice, stream_));
        k_mpnn_round<<<32, 256, 0, stream_>>>(m.P, m.w, m.wb);
        launchCheck("mpnn_round");
    }
    if (get) CFG_CUDA(cudaMemcpyAsync(get, m.w, n * sizeof(float), cudaMemcpyDeviceToHost, stream_));
    CFG_CUDA(cudaStreamSynchronize(stream_));
}

int Ctx::mpnnParams() const { return mpnn_ ? mpnn_->P : 0; }

/// z = M(r) on the pressure matrix (vals, diag), all device vectors
void Ctx::mpnnApply(const double* vals, const double* diag, const double* r, double* z)
{
    MpnnState& m = *mpnn_;
    const DMat A{dm_.nC, dm_.mStart, dm_.mCol};
    const int n = dm_.nC;
    const size_t nH = static_cast<size_t>(n) * H;
    const int blocks = std::max(1, std::min((n + kWarps - 1) / kWarps, sms_ * 16));
    k_mpnn_coef<<<GS_, TPB, 0, stream_>>>(A, vals, diag, m.coef);
    k_mpnn_scale<<<GS_, TPB, 0, stream_>>>(n, r, partials_, m.ticket, m.s);
    k_mpnn_enc<<<blocks, kWarps * 32, 0, stream_>>>(n, r, m.s + 1, m.wb, m.h, m.mask);
    for (int l = 0; l < m.L; ++l)
    {
        if (mpnnTimeLayers_) CFG_CUDA(cudaEventRecord(tm_.ev[4 + 2 * (l % 4)], stream_));
        k_mpnn_layer<<<blocks, kWarps * 32, 0, stream_>>>(A, m.coef, m.wb + offLayer(l), m.h + l * nH,
                                                          m.h + (l + 1) * nH, m.mask + static_cast<size_t>(l + 1) * n);
        if (mpnnTimeLayers_)
        {
            CFG_CUDA(cudaEventRecord(tm_.ev[5 + 2 * (l % 4)], stream_));
            CFG_CUDA(cudaEventSynchronize(tm_.ev[5 + 2 * (l % 4)]));
            float ms = 0;
            CFG_CUDA(cudaEventElapsedTime(&ms, tm_.ev[4 + 2 * (l % 4)], tm_.ev[5 + 2 * (l % 4)]));
            mpnnLayerMs_ += ms;
            ++mpnnLayerLaunches_;
        }
    }
    k_mpnn_out<<<blocks, kWarps * 32, 0, stream_>>>(n, r, diag, m.s, m.wb + offLayer(m.L), m.h + m.L * nH, z);
    launchCheck("mpnn_apply", 4 + m.L);
}

/// One sample's loss and its gradient (into m.g).  Without a target t: the
/// residual loss |A M(r) - r|^2 / |r|^2.  With t, the converged correction
/// for the residual r (A t = r): the energy-norm loss e.Ae / t.At with
/// e = M(r) - t -- the error CG itself minimises.
double Ctx::mpnnLossGrad(const double* vals, const double* diag, const double* r, double* z, const double* t)
{
    MpnnState& m = *mpnn_;
    const DMat A{dm_.nC, dm_.mStart, dm_.mCol};
    const int n = dm_.nC;
    const size_t nH = static_cast<size_t>(n) * H;
    const int blocks = std::max(1, std::min((n + kWarps - 1) / kWarps, sms_ * 16));
    mpnnApply(vals, diag, r, z);
    CFG_CUDA(cudaMemsetAsync(m.acc, 0, sizeof(double), stream_));
    CFG_CUDA(cudaMemsetAsync(m.g, 0, m.P * sizeof(float), stream_));
    const double* rrp = m.s + 2;
    double eAe = 0, tAt = 0;
    if (t)
    {
        // e = z - t, Ae, At, e.Ae and t.At (on the device for the gradient)
        k_fcg_p<<<GS_, TPB, 0, stream_>>>(n, z, 0.0, m.res);
        k_fcg_axpy<<<GS_, TPB, 0, stream_>>>(n, -1.0, t, m.res);
        fcgSpmv(vals, m.res, m.ae);
        fcgSpmv(vals, t, m.at);
        const double* a[2] = {m.res, t};
        const double* b[2] = {m.ae, m.at};
        double d[3];
        fcgDots(2, a, b, d);
        eAe = d[0];
        tAt = d[1];
        rrp = fcgOut_ + 1;
    }
    {
        const int W = maxW_ <= 7 ? 7 : (maxW_ <= 16 ? 16 : 0);
        if (W == 7)
        {
            if (!t) k_mpnn_resid<7><<<GS_, TPB, 0, stream_>>>(A, vals, z, r, m.res, m.acc);
            k_mpnn_out_bwd<7><<<blocks, kWarps * 32, 0, stream_>>>(A, vals, m.res, m.s, rrp, m.wb + offLayer(m.L),
                                                                   m.h + m.L * nH, m.dh0, m.g + offLayer(m.L));
        }
        else if (W == 16)
        {
            if (!t) k_mpnn_resid<16><<<GS_, TPB, 0, stream_>>>(A, vals, z, r, m.res, m.acc);
            k_mpnn_out_bwd<16><<<blocks, kWarps * 32, 0, stream_>>>(A, vals, m.res, m.s, rrp, m.wb + offLayer(m.L),
                                                                    m.h + m.L * nH, m.dh0, m.g + offLayer(m.L));
        }
        else
        {
            if (!t) k_mpnn_resid<0><<<GS_, TPB, 0, stream_>>>(A, vals, z, r, m.res, m.acc);
            k_mpnn_out_bwd<0><<<blocks, kWarps * 32, 0, stream_>>>(A, vals, m.res, m.s, rrp, m.wb + offLayer(m.L),
                                                                   m.h + m.L * nH, m.dh0, m.g + offLayer(m.L));
        }
    }
    float* dh = m.dh0;
    float* dn = m.dh1;
    for (int l = m.L - 1; l >= 0; --l)
    {
        k_mpnn_layer_bwd<<<blocks, kWarps * 32, 0, stream_>>>(A, m.coef, m.wb + offLayer(l), m.h + l * nH,
                                                              m.mask + static_cast<size_t>(l + 1) * n, dh, dn, m.v,
                                                              m.g + offLayer(l));
        k_mpnn_msg_bwd<<<blocks, kWarps * 32, 0, stream_>>>(A, vals, diag, m.v, dn);
        std::swap(dh, dn);
    }
    k_mpnn_enc_bwd<<<blocks, kWarps * 32, 0, stream_>>>(n, r, m.s + 1, m.mask, dh, m.g);
    launchCheck("mpnn_backward", 3 + 2 * m.L);
    if (t) return tAt > 0 ? eAe / tAt : 0.0;
    double h[3];
    CFG_CUDA(cudaMemcpyAsync(h, m.acc, sizeof(double), cudaMemcpyDeviceToHost, stream_));
    CFG_CUDA(cudaMemcpyAsync(h + 1, m.s + 2, sizeof(double), cudaMemcpyDeviceToHost, stream_));
    CFG_CUDA(cudaStreamSynchronize(stream_));
    return h[1] > 0 ? h[0] / h[1] : 0.0;
}

void Ctx::mpnnAdam(float lr)
{
    MpnnState& m = *mpnn_;
    ++m.step;
    const float c1 = 1.f - std::pow(0.9f, static_cast<float>(m.step));
    const float c2 = 1.f - std::pow(0.999f, static_cast<float>(m.step));
    k_mpnn_adam<<<32, 256, 0, stream_>>>(m.P, m.w, m.g, m.m1, m.m2, lr, c1, c2, m.wb);
    launchCheck("mpnn_adam");
}

/// the pressure matrix the network works on: the Poisson system when set
/// up, else the last assembled SIMPLE pressure equation
void Ctx::mpnnMatrix(const double** vals, const double** diag) const
{
    *vals = pVal_d_;
    *diag = pDiag_;
}

double Ctx::mpnnLossGradHost(const double* r, float* grad, const double* t)
{
    if (!mpnn_) fail(CFG_EINVAL, "mpnn: call cfg_mpnn_create first");
    CFG_CUDA(cudaSetDevice(device_));
    const double *vals, *diag;
    mpnnMatrix(&vals, &diag);
    toDevCells(cr_, r, 1, 0);
    double* td = nullptr;
    if (t)
    {
        td = bt_.c[2];  // free outside the momentum solve
        toDevCells(td, t, 1, 0);
    }
    const double loss = mpnnLossGrad(vals, diag, cr_, cz_, td);
    if (grad)
    {
        CFG_CUDA(cudaMemcpyAsync(grad, mpnn_->g, mpnn_->P * sizeof(float), cudaMemcpyDeviceToHost, stream_));
        CFG_CUDA(cudaStreamSynchronize(stream_));
    }
    return loss;
}

/// Event-timed applications of the network on the current pressure matrix
/// (input: the residual buffer's contents): out = {ms per application, ms
/// per message-passing layer launch}.
void Ctx::mpnnTime(int reps, double* out)
{
    if (!mpnn_) fail(CFG_EINVAL, "mpnn: call cfg_mpnn_create first");
    CFG_CUDA(cudaSetDevice(device_));
    const double *vals, *diag;
    mpnnMatrix(&vals, &diag);
    mpnnApply(vals, diag, cr_, cz_);  // warm
    CFG_CUDA(cudaEventRecord(tm_.ev[2], stream_));
    for (int k = 0; k < reps; ++k) mpnnApply(vals, diag, cr_, cz_);
    CFG_CUDA(cudaEventRecord(tm_.ev[3], stream_));
    CFG_CUDA(cudaEventSynchronize(tm_.ev[3]));
    float ms = 0;
    CFG_CUDA(cudaEventElapsedTime(&ms, tm_.ev[2], tm_.ev[3]));
    out[0] = ms / std::max(1, reps);
    mpnnTimeLayers_ = true;
    mpnnLayerMs_ = 0;
    mpnnLayerLaunches_ = 0;
    for (int k = 0; k < reps; ++k) mpnnApply(vals, diag, cr_, cz_);
    mpnnTimeLayers_ = false;
    out[1] = mpnnLayerMs_ / std::max<int64_t>(1, mpnnLayerLaunches_);
}

void Ctx::mpnnApplyHost(const double* r, double* z)
{
    if (!mpnn_) fail(CFG_EINVAL, "mpnn: call cfg_mpnn_create first");
    CFG_CUDA(cudaSetDevice(device_));
    const double *vals, *diag;
    mpnnMatrix(&vals, &diag);
    toDevCells(cr_, r, 1, 0);
    mpnnApply(vals, diag, cr_, cz_);
    fromDevCells(z, cz_, 1, 0);
}

/// Adam over `nSamples` residual samples (device, nSamples x nC, device
/// numbering), with their converged corrections when `targets` is given,
/// for `epochs` passes; losses[e] = the epoch's mean loss
void Ctx::mpnnTrain(const double* samples, int nSamples, int epochs, float lr, double* losses,
                    const double* targets)
{
    if (!mpnn_) fail(CFG_EINVAL, "mpnn: call cfg_mpnn_create first");
    const double *vals, *diag;
    mpnnMatrix(&vals, &diag);
    const size_t n = static_cast<size_t>(dm_.nC);
    for (int e = 0; e < epochs; ++e)
    {
        double sum = 0;
        for (int k = 0; k < nSamples; ++k)
        {
            sum += mpnnLossGrad(vals, diag, samples + k * n, cz_, targets ? targets + k * n : nullptr);
            mpnnAdam(lr);
        }
        if (losses) losses[e] = sum / std::max(1, nSamples);
    }
    CFG_CUDA(cudaStreamSynchronize(stream_));
}

void Ctx::mpnnTrainHost(const double* samples, int nSamples, int epochs, float lr, double* losses,
                        const double* targets)
{
    if (!mpnn_) fail(CFG_EINVAL, "mpnn: call cfg_mpnn_create first");
    if (nSamples <= 0 || epochs <= 0) fail(CFG_EINVAL, "mpnn: no samples or epochs");
    CFG_CUDA(cudaSetDevice(device_));
    const size_t n = static_cast<size_t>(dm_.nC);
    // the training set on the device, kept across calls when it fits
    const size_t need = n * nSamples * (targets ? 2 : 1);
    if (need > trainCap_)
    {
        trainBuf_ = alloc<double>(need);  // released with the context
        trainCap_ = need;
    }
    double* d = trainBuf_;
    for (int k = 0; k < nSamples; ++k) toDevCells(d + k * n, samples + k * n, 1, 0);
    double* t = nullptr;
    if (targets)
    {
        t = d + n * nSamples;
        for (int k = 0; k < nSamples; ++k) toDevCells(t + k * n, targets + k * n, 1, 0);
    }
    mpnnTrain(d, nSamples, epochs, lr, losses, t);
}

void Ctx::mpnnCollect(int mode, int maxSamples)
{
    if (mode == 2)
    {
        collected_.clear();
        collectedT_.clear();
    }
    collectOn_ = mode != 0;
    collectMax_ = std::max(0, maxSamples);
}

/// Training on the collected pairs: the residual each pressure solve started
/// from and the correction the plain solver converged to from there.
void Ctx::mpnnTrainCollected(int epochs, float lr, double* losses)
{
    if (collected_.empty()) fail(CFG_EINVAL, "mpnn: no collected samples");
    const size_t n = static_cast<size_t>(dm_.nC);
    const size_t k = collected_.size();
    std::vector<double> all(k * n), tgt(k * n);
    for (size_t j = 0; j < k; ++j)
    {
        std::copy(collected_[j].begin(), collected_[j].end(), all.begin() + j * n);
        std::copy(collectedT_[j].begin(), collectedT_[j].end(), tgt.begin() + j * n);
    }
    mpnnTrainHost(all.data(), static_cast<int>(k), epochs, lr, losses, tgt.data());
}

/// The network's initial guess: x += M(b - A x).
void Ctx::mpnnGuess(const double* vals, const double* diag, const double* b, double* x)
{
    const int n = dm_.nC;
    fcgSpmv(vals, x, cAp_);
    CFG_CUDA(cudaMemcpyAsync(cr_, b, n * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    k_fcg_axpy<<<GS_, TPB, 0, stream_>>>(n, -1.0, cAp_, cr_);
    mpnnApply(vals, diag, cr_, cz_);
    k_fcg_axpy<<<GS_, TPB, 0, stream_>>>(n, 1.0, cz_, x);
    launchCheck("mpnn_guess", 2);
}

void Ctx::poissonResidual(const double* b, const double* x, double* r)
{
    if (!poissonReady_) fail(CFG_EINVAL, "cfg_poisson_residual: call cfg_poisson_setup first");
    CFG_CUDA(cudaSetDevice(device_));
    const int n = dm_.nC;
    toDevCells(pb64_, b, 1, 0);
    toDevCells(px64_, x, 1, 0);
    fcgSpmv(pVal_d_, px64_, cAp_);
    CFG_CUDA(cudaMemcpyAsync(cr_, pb64_, n * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    k_fcg_axpy<<<GS_, TPB, 0, stream_>>>(n, -1.0, cAp_, cr_);
    launchCheck("poisson_residual");
    fromDevCells(r, cr_, 1, 0);
}

void Ctx::fcgSpmv(const double* vals, const double* x, double* y)
{
    const DMat A{dm_.nC, dm_.mStart, dm_.mCol};
    const int W = maxW_ <= 7 ? 7 : (maxW_ <= 16 ? 16 : 0);
    if (W == 7) k_fcg_spmv<7><<<GS_, TPB, 0, stream_>>>(A, vals, x, y);
    else if (W == 16) k_fcg_spmv<16><<<GS_, TPB, 0, stream_>>>(A, vals, x, y);
    else k_fcg_spmv<0><<<GS_, TPB, 0, stream_>>>(A, vals, x, y);
    launchCheck("fcg_spmv");
}

/// up to 3 dot products a[q].b[q], returned on the host
void Ctx::fcgDots(int np, const double* const* a, const double* const* b, double* out)
{
    if (!fcgPtrs_)
    {
        fcgPtrs_ = alloc<const double*>(6);
        fcgOut_ = alloc<double>(8);
        fcgTicket_ = alloc<unsigned>(1);
        CFG_CUDA(cudaMemsetAsync(fcgTicket_, 0, sizeof(unsigned), stream_));
    }
    const double* h[6] = {a[0], np > 1 ? a[1] : a[0], np > 2 ? a[2] : a[0],
                          b[0], np > 1 ? b[1] : b[0], np > 2 ? b[2] : b[0]};
    CFG_CUDA(cudaMemcpyAsync(fcgPtrs_, h, sizeof h, cudaMemcpyHostToDevice, stream_));
    k_fcg_dots<3><<<GS_, TPB, 0, stream_>>>(dm_.nC, fcgPtrs_, fcgPtrs_ + 3, partials_, fcgTicket_, fcgOut_);
    launchCheck("fcg_dots");
    double o[3];
    CFG_CUDA(cudaMemcpyAsync(o, fcgOut_, sizeof o, cudaMemcpyDeviceToHost, stream_));
    CFG_CUDA(cudaStreamSynchronize(stream_));
    for (int q = 0; q < np; ++q) out[q] = o[q];
}

/// Flexible CG (Notay's FCG(1): alpha = p.r / p.Ap, beta = -z.Ap / p.Ap) with
/// z = M(r) from the network, to |b - A x|2 / |b|2 <= tol.  When the
/// residual has not fallen by 10% over the last `window` iterations the
/// solve continues from the current x with FP64 DIC-PCG (the fallback).
/// out: {network iterations, fallback iterations, fell back}
/// the stopping norm: |v|2 (normType 1) or |v|inf (0, the reference's test)
double Ctx::fcgNorm(const double* v, int normType)
{
    if (normType == 1)
    {
        double d[1];
        const double* a[1] = {v};
        fcgDots(1, a, a, d);
        return std::sqrt(d[0]);
    }
    CFG_CUDA(cudaMemsetAsync(fcgOut_ + 3, 0, sizeof(double), stream_));
    k_fcg_absmax<<<GS_, TPB, 0, stream_>>>(dm_.nC, v, fcgOut_ + 3);
    launchCheck("fcg_absmax");
    double h;
    CFG_CUDA(cudaMemcpyAsync(&h, fcgOut_ + 3, sizeof(double), cudaMemcpyDeviceToHost, stream_));
    CFG_CUDA(cudaStreamSynchronize(stream_));
    return h;
}

void Ctx::mpnnResidualHost(const double* vals, const double* b, const double* x, double* rHost)
{
    const int n = dm_.nC;
    fcgSpmv(vals, x, cAp_);
    CFG_CUDA(cudaMemcpyAsync(cz_, b, n * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    k_fcg_axpy<<<GS_, TPB, 0, stream_>>>(n, -1.0, cAp_, cz_);
    launchCheck("mpnn_residual");
    fromDevCells(rHost, cz_, 1, 0);
}

void Ctx::mpnnFcg(const double* vals, const double* diag, const double* b, double* x, double tol, int maxIter,
                  int window, int64_t* out, int normType, int pc)
{
    const int n = dm_.nC;
    double* r = cr_;
    double* z = cz_;
    double* p = cp_;
    double* q = cAp_;
    // the preconditioner: the network (pc 0), an AMG V-cycle (1), or the
    // V-cycle with the network applied to the residual it leaves (2)
    auto precond = [&](const double* rr, double* zz) {
        if (pc == 0)
        {
            mpnnApply(vals, diag, rr, zz);
            return;
        }
        amgApply(rr, zz);
        if (pc != 2) return;
        double* t = bt_.c[0];
        double* w = bt_.c[1];
        fcgSpmv(vals, zz, t);
        k_fcg_p<<<GS_, TPB, 0, stream_>>>(n, rr, -1.0, t);  // t = r - A z
        launchCheck("amg_mpnn_residual");
        mpnnApply(vals, diag, t, w);
        k_fcg_axpy<<<GS_, TPB, 0, stream_>>>(n, 1.0, w, zz);  // z += N(r - A z)
        launchCheck("amg_mpnn_correct");
    };
    fcgSpmv(vals, x, q);
    CFG_CUDA(cudaMemcpyAsync(r, b, n * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    k_fcg_axpy<<<GS_, TPB, 0, stream_>>>(n, -1.0, q, r);
    launchCheck("fcg_r0");
    double d3[3];
    if (!fcgPtrs_) fcgDots(1, &b, &b, d3);  // allocates the scalar buffers
    const double bn = std::max(fcgNorm(b, normType), normType == 1 ? 0.0 : 1e-300);
    double rn = fcgNorm(r, normType);
    std::vector<double> hist{rn};
    int it = 0;
    out[0] = out[1] = out[2] = 0;
    if (!(bn > 0) || rn / bn <= tol) return;
    precond(r, z);
    CFG_CUDA(cudaMemcpyAsync(p, z, n * sizeof(double), cudaMemcpyDeviceToDevice, stream_));
    bool fallback = false;
    while (it < maxIter)
    {
        fcgSpmv(vals, p, q);
        const double* a[2] = {p, p};
        const double* bb[2] = {r, q};
        fcgDots(2, a, bb, d3);
        const double pq = d3[1];
        if (!(pq > 0)) break;
        const double alpha = d3[0] / pq;
        k_fcg_axpy<<<GS_, TPB, 0, stream_>>>(n, alpha, p, x);
        k_fcg_axpy<<<GS_, TPB, 0, stream_>>>(n, -alpha, q, r);
        launchCheck("fcg_update", 2);
        ++it;
        rn = fcgNorm(r, normType);
        hist.push_back(rn);
        if (rn / bn <= tol) break;
        if (static_cast<int>(hist.size()) > window && rn > 0.9 * hist[hist.size() - 1 - window])
        {
            fallback = true;
            break;
        }
        precond(r, z);
        {
            const double* aa[1] = {z};
            const double* bq[1] = {q};
            fcgDots(1, aa, bq, d3);
        }
        k_fcg_p<<<GS_, TPB, 0, stream_>>>(n, z, -d3[0] / pq, p);
        launchCheck("fcg_p");
    }
    out[0] = it;
    if (fallback && it < maxIter)
    {
        cfg_solver_report rep{};
        if (normType == 0) dicSetup(vals, diag);  // the SIMPLE/PISO matrix of this solve
        dicCGT<double>(dic_, vals, diag, b, x, cr_, cp_, cAp_, cz_, tol, maxIter - it, normType, &rep);
        out[1] = rep.iterations;
        out[2] = 1;
    }
}

}  // namespace cfg
