// gnn.cu — learned warm start: a small two-layer message-passing network
// that predicts the PageRank vector from degree features.  Its normalised
// output only seeds the solver (prg_solve with a start vector), so the fixed
// point, the stop rule and every correctness check stay those of the plain
// method.
//
// Model (per vertex v, internal ids; s_u = 1/outdeg(u), 0 when dangling):
//   X0[v]  = degree features (16, BF16)
//   H0     = relu(X0 W1^T + b1)                 (32, BF16)   tensor cores
//   M0[u]  = s_u * (H0[u] Wm1^T)                (8, FP32)    tensor cores
//   S1[v]  = sum_{u->v} M0[u],  A1 = slog(S1)   (8 -> BF16)  in-CSR aggregation
//   H1     = relu([H0 | A1] W2^T + b2)          (32, BF16)   tensor cores
//   M1[u]  = s_u * (H1[u] Wm2^T)                (8, FP32)    tensor cores
//   S2[v]  = sum_{u->v} M1[u],  A2 = slog(S2)   (8 -> BF16)
//   y[v]   = [H1 | A2] w3 + b3                  (FP32)       tensor cores
//   start  = exp(y) / sum exp(y)                (FP64)
// The messages carry rank-like mass (scaled by 1/outdeg exactly like the
// power step), so two layers see two hops of the operator; the aggregated
// mass spans orders of magnitude (hubs), so it enters the next layer through
// slog(z) = sign(z) log(1 + |z|).  Dense layers run
// on the tensor cores (mma.sync m16n8k16, BF16 operands, FP32 accumulate).
// Training minimises sum_v w_v (y_v - log(n x*_v))^2 / n with w_v = n x*_v;
// the backward pass is hand-written (FP32 CUDA cores, deterministic block
// partials for the weight gradients, atomics only for the transposed
// aggregation), and Adam updates FP32 master weights, then refreshes the
// BF16 copies the forward pass reads.
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "gnn.cuh"
#include "prims.cuh"

namespace prg {
namespace gnn {

// ---- parameter layout (FP32 master, flat) --------------------------------
constexpr int kF = 16, kH = 32, kC = 8, kZ = 48;  // features, hidden, message channels, [H|A] width
constexpr int oW1 = 0;                       // [32 x 16]
constexpr int oB1 = oW1 + kH * kF;           // [32]
constexpr int oWm1 = oB1 + kH;               // [8 x 32]
constexpr int oW2 = oWm1 + kC * kH;          // [32 x 48]
constexpr int oB2 = oW2 + kH * kZ;           // [32]
constexpr int oWm2 = oB2 + kH;               // [8 x 32]
constexpr int oW3 = oWm2 + kC * kH;          // [8 x 48] (row 0 used)
constexpr int oB3 = oW3 + 8 * kZ;            // [8]      (entry 0 used)
constexpr int kParams = oB3 + 8;             // 3016

struct Ws {  // BF16 copies of the weight matrices
    __nv_bfloat16 W1[kH * kF], Wm1[kC * kH], W2[kH * kZ], Wm2[kC * kH], W3[8 * kZ];
};

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    const __nv_bfloat162 p = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<const uint32_t *>(&p);
}

// ---- features --------------------------------------------------------------
__global__ void features_kernel(uint32_t n, const uint32_t *row_ptr, const uint32_t *deg, __nv_bfloat16 *X0) {
    const float ln = logf((float)n) * 0.0625f;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const float li = log1pf((float)(row_ptr[v + 1] - row_ptr[v]));
        const float lo = log1pf((float)deg[v]);
        float f[kF];
#pragma unroll
        for (int i = 0; i < kF; i++) f[i] = 0.0f;
        f[0] = li * 0.125f;
        f[1] = lo * 0.125f;
        f[2] = deg[v] == 0 ? 1.0f : 0.0f;
        f[3] = 1.0f;
        f[4] = (li - lo) * 0.125f;
        f[5] = ln;
        uint4 *dst = reinterpret_cast<uint4 *>(X0 + (size_t)v * kF);
        dst[0] = make_uint4(pack_bf16(f[0], f[1]), pack_bf16(f[2], f[3]), pack_bf16(f[4], f[5]), pack_bf16(f[6], f[7]));
        dst[1] = make_uint4(pack_bf16(f[8], f[9]), pack_bf16(f[10], f[11]), pack_bf16(f[12], f[13]),
                            pack_bf16(f[14], f[15]));
    }
}

// ---- rowwise dense layer on the tensor cores --------------------------------
// Y[v][0..N) = sum_k A[v][k] W[j][k] for 16-row tiles per warp.  A is the
// concatenation [A0 (K0 cols) | A1 (K1 cols)] (BF16, row-major); W is
// [N x (K0+K1)] BF16 row-major (= the B operand in column-major k x n).
// Fragment layout of mma.m16n8k16 (PTX ISA): group g = lane/4, t = lane%4;
// A regs: (g, 2t..2t+1), (g+8, 2t..), (g, 2t+8..), (g+8, 2t+8..);
// B regs: (k=2t..2t+1, n=g), (k=2t+8.., n=g); C: (g, 2t..2t+1), (g+8, 2t..).
enum Epi { EPI_RELU_BF16 = 0, EPI_SCALE_F32 = 1, EPI_COL0_F32 = 2 };

template <int K0, int K1, int N, int EPI>
__global__ void __launch_bounds__(128) rowwise_kernel(uint32_t n, const __nv_bfloat16 *A0, const __nv_bfloat16 *A1,
                                                      const __nv_bfloat16 *W, const float *bias, const float *scale,
                                                      __nv_bfloat16 *out_bf, float *out_f) {
    constexpr int K = K0 + K1;
    static_assert(K % 16 == 0 && N % 8 == 0, "mma tile shape");
    __shared__ __align__(16) __nv_bfloat16 sW[N * K];
    for (int i = threadIdx.x; i < N * K; i += blockDim.x) sW[i] = W[i];
    __syncthreads();
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const uint32_t ntiles = (n + 15) / 16;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t tile = warp; tile < ntiles; tile += nwarps) {
        const uint32_t r0 = tile * 16 + g, r1 = r0 + 8;
        float acc[N / 8][4];
#pragma unroll
        for (int j = 0; j < N / 8; j++) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0f;
#pragma unroll
        for (int kt = 0; kt < K / 16; kt++) {
            // A fragment (rows beyond n read as zero)
            const int kb = kt * 16;
            uint32_t a[4];
            auto ldA = [&](uint32_t r, int k) -> uint32_t {
                if (r >= n) return 0u;
                if (k < K0) return *reinterpret_cast<const uint32_t *>(A0 + (size_t)r * K0 + k);
                return *reinterpret_cast<const uint32_t *>(A1 + (size_t)r * K1 + (k - K0));
            };
            a[0] = ldA(r0, kb + 2 * t);
            a[1] = ldA(r1, kb + 2 * t);
            a[2] = ldA(r0, kb + 2 * t + 8);
            a[3] = ldA(r1, kb + 2 * t + 8);
#pragma unroll
            for (int j = 0; j < N / 8; j++) {
                const int col = j * 8 + g;
                const uint32_t b0 = *reinterpret_cast<const uint32_t *>(sW + col * K + kb + 2 * t);
                const uint32_t b1 = *reinterpret_cast<const uint32_t *>(sW + col * K + kb + 2 * t + 8);
                asm volatile(
                    "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
                    "{%0,%1,%2,%3};"
                    : "+f"(acc[j][0]), "+f"(acc[j][1]), "+f"(acc[j][2]), "+f"(acc[j][3])
                    : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
            }
        }
        // epilogue: C(g, 2t..), C(g+8, 2t..) of each n-tile
#pragma unroll
        for (int j = 0; j < N / 8; j++) {
            const int c0 = j * 8 + 2 * t;
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const uint32_t r = h ? r1 : r0;
                if (r >= n) continue;
                float v0 = acc[j][2 * h], v1 = acc[j][2 * h + 1];
                if constexpr (EPI == EPI_RELU_BF16) {
                    v0 = fmaxf(v0 + bias[c0], 0.0f);
                    v1 = fmaxf(v1 + bias[c0 + 1], 0.0f);
                    *reinterpret_cast<uint32_t *>(out_bf + (size_t)r * N + c0) = pack_bf16(v0, v1);
                } else if constexpr (EPI == EPI_SCALE_F32) {
                    const float sc = scale[r];
                    out_f[(size_t)r * N + c0] = v0 * sc;
                    out_f[(size_t)r * N + c0 + 1] = v1 * sc;
                } else {
                    if (c0 == 0) out_f[r] = v0 + bias[0];
                }
            }
        }
    }
}

template <int K0, int K1, int N, int EPI>
static void rowwise(uint32_t n, const __nv_bfloat16 *A0, const __nv_bfloat16 *A1, const __nv_bfloat16 *W,
                    const float *bias, const float *scale, __nv_bfloat16 *out_bf, float *out_f, cudaStream_t s) {
    const uint32_t tiles = (n + 15) / 16;
    const unsigned grid = (unsigned)std::min<uint32_t>((tiles + 3) / 4, 148u * 16u);
    rowwise_kernel<K0, K1, N, EPI><<<std::max(grid, 1u), 128, 0, s>>>(n, A0, A1, W, bias, scale, out_bf, out_f);
    PRG_CUDA(cudaGetLastError());
}

// ---- aggregation A[v] = sum_{u->v} M[u] (8 channels) ------------------------
// Rows of up to kAggHeavy arcs: 8 lanes per row, each lane takes every 8th
// arc and gathers the source's 32-byte message; lanes combine with shuffles.
// Longer rows are queued and summed by a whole block each.
constexpr uint32_t kAggHeavy = 2048;

__device__ __forceinline__ float slog(float z) { return copysignf(log1pf(fabsf(z)), z); }

__global__ void aggregate_kernel(uint32_t n, const uint32_t *row_ptr, const uint32_t *col, const float *M,
                                 __nv_bfloat16 *out, float *out_f, uint32_t *heavy, uint32_t *nheavy) {
    const uint32_t gid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t sub = threadIdx.x & 7;
    const uint32_t group = gid >> 3, ngroups = (gridDim.x * blockDim.x) >> 3;
    const uint32_t rounds = (n + ngroups - 1) / ngroups;
    for (uint32_t rd = 0; rd < rounds; rd++) {
        const uint32_t v = rd * ngroups + group;
        float acc[kC];
#pragma unroll
        for (int c = 0; c < kC; c++) acc[c] = 0.0f;
        bool skip = v >= n;
        if (!skip) {
            const uint32_t p0 = row_ptr[v], p1 = row_ptr[v + 1];
            if (p1 - p0 > kAggHeavy) {
                if (sub == 0) heavy[atomicAdd(nheavy, 1u)] = v;
                skip = true;
            } else {
                for (uint32_t p = p0 + sub; p < p1; p += 8) {
                    const uint32_t u = __ldg(&col[p]);
                    const float4 q0 = __ldg(reinterpret_cast<const float4 *>(M + (size_t)u * kC));
                    const float4 q1 = __ldg(reinterpret_cast<const float4 *>(M + (size_t)u * kC) + 1);
                    acc[0] += q0.x; acc[1] += q0.y; acc[2] += q0.z; acc[3] += q0.w;
                    acc[4] += q1.x; acc[5] += q1.y; acc[6] += q1.z; acc[7] += q1.w;
                }
            }
        }
#pragma unroll
        for (int c = 0; c < kC; c++) {
            acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], 4);
            acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], 2);
            acc[c] += __shfl_xor_sync(0xffffffffu, acc[c], 1);
        }
        if (!skip && sub == 0) {
            uint4 *dst = reinterpret_cast<uint4 *>(out + (size_t)v * 16);
            dst[0] = make_uint4(pack_bf16(slog(acc[0]), slog(acc[1])), pack_bf16(slog(acc[2]), slog(acc[3])),
                                pack_bf16(slog(acc[4]), slog(acc[5])), pack_bf16(slog(acc[6]), slog(acc[7])));
            dst[1] = make_uint4(0u, 0u, 0u, 0u);
            for (int c = 0; c < kC; c++) out_f[(size_t)v * kC + c] = acc[c];
        }
    }
}

__global__ void aggregate_heavy_kernel(const uint32_t *row_ptr, const uint32_t *col, const float *M,
                                       __nv_bfloat16 *out, float *out_f, const uint32_t *heavy,
                                       const uint32_t *nheavy) {
    __shared__ float sh[kC][32];
    const uint32_t cnt = *nheavy;
    for (uint32_t i = blockIdx.x; i < cnt; i += gridDim.x) {
        const uint32_t v = heavy[i];
        const uint32_t p0 = row_ptr[v], p1 = row_ptr[v + 1];
        float acc[kC];
#pragma unroll
        for (int c = 0; c < kC; c++) acc[c] = 0.0f;
        for (uint32_t p = p0 + threadIdx.x; p < p1; p += blockDim.x) {
            const uint32_t u = __ldg(&col[p]);
            const float4 q0 = __ldg(reinterpret_cast<const float4 *>(M + (size_t)u * kC));
            const float4 q1 = __ldg(reinterpret_cast<const float4 *>(M + (size_t)u * kC) + 1);
            acc[0] += q0.x; acc[1] += q0.y; acc[2] += q0.z; acc[3] += q0.w;
            acc[4] += q1.x; acc[5] += q1.y; acc[6] += q1.z; acc[7] += q1.w;
        }
        const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
        for (int c = 0; c < kC; c++) acc[c] = warp_sum(acc[c]);
        __syncthreads();
        if (l == 0)
            for (int c = 0; c < kC; c++) sh[c][w] = acc[c];
        __syncthreads();
        if (threadIdx.x < kC) {
            float tot = 0.0f;
            for (int k = 0; k < (int)(blockDim.x >> 5); k++) tot += sh[threadIdx.x][k];
            out[(size_t)v * 16 + threadIdx.x] = __float2bfloat16_rn(slog(tot));
            out[(size_t)v * 16 + 8 + threadIdx.x] = __float2bfloat16_rn(0.0f);
            out_f[(size_t)v * kC + threadIdx.x] = tot;
        }
    }
}

// ---- prediction --------------------------------------------------------------
__global__ void max_kernel(const float *y, uint32_t n, float *part) {
    float m = -INFINITY;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) m = fmaxf(m, y[v]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    __shared__ float sh[32];
    if ((threadIdx.x & 31) == 0) sh[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 1; i < (int)(blockDim.x >> 5); i++) m = fmaxf(m, sh[i]);
        m = fmaxf(m, sh[0]);
        part[blockIdx.x] = m;
    }
}

__global__ void expsum_kernel(const float *y, uint32_t n, const float *mpart, unsigned nm, double *x, double *part) {
    float m = -INFINITY;
    for (unsigned i = 0; i < nm; i++) m = fmaxf(m, mpart[i]);
    double s = 0.0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const double e = exp((double)(y[v] - m));
        x[v] = e;
        s += e;
    }
    __shared__ double sh[32];
    s = block_sum<double>(s, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = s;
}

__global__ void normalise_kernel(double *x, uint32_t n, const double *part, unsigned np) {
    double s = 0.0;
    for (unsigned i = 0; i < np; i++) s += part[i];
    const double inv = 1.0 / s;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) x[v] *= inv;
}

__global__ void scale_kernel(const uint32_t *deg, uint32_t n, float *s) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        s[v] = deg[v] ? 1.0f / (float)deg[v] : 0.0f;
}

// ---- loss ------------------------------------------------------------------
// target x* in internal ids; L = sum_v w_v (y_v - t_v)^2 / n, w_v = n x*_v.
__global__ void loss_kernel(const float *y, const double *xs, uint32_t n, float *dy, double *part) {
    double l = 0.0;
    const double nn = (double)n;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const double xv = xs[v] > 1e-300 ? xs[v] : 1e-300;
        const double w = nn * xv, tv = log(nn * xv);
        const double e = (double)y[v] - tv;
        l += w * e * e;
        dy[v] = (float)(2.0 * w * e / nn);
    }
    __shared__ double sh[32];
    l = block_sum<double>(l, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = l / nn;
}

// ---- backward (FP32 CUDA cores) -----------------------------------------------
__device__ __forceinline__ float bf(const __nv_bfloat16 &x) { return __bfloat162float(x); }

// dy -> dH1 (32) and dA2 (8) through y = [H1 | A2] w3 + b3
__global__ void bwd_out_kernel(uint32_t n, const float *dy, const float *P, float *dH1, float *dA2) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const float g = dy[v];
        for (int k = 0; k < kH; k++) dH1[(size_t)v * kH + k] = g * P[oW3 + k];
        for (int c = 0; c < kC; c++) dA2[(size_t)v * kC + c] = g * P[oW3 + kH + c];
    }
}

// dM[u] += dS[v] over every in-arc u -> v (transposed aggregation), where
// dS = dA / (1 + |S|) is the gradient through A = slog(S)
__global__ void scatter_kernel(uint32_t n, const uint32_t *row_ptr, const uint32_t *col, const float *dA,
                               const float *S, float *dM) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        float g[kC];
        for (int c = 0; c < kC; c++) g[c] = dA[(size_t)v * kC + c] / (1.0f + fabsf(S[(size_t)v * kC + c]));
        for (uint32_t p = row_ptr[v]; p < row_ptr[v + 1]; p++) {
            const uint32_t u = col[p];
            for (int c = 0; c < kC; c++) atomicAdd(&dM[(size_t)u * kC + c], g[c]);
        }
    }
}

// message layer: G = dM * s; dH += G Wm; then relu mask -> dPre (in place in dH)
__global__ void bwd_msg_kernel(uint32_t n, const float *dM, const float *s, const float *P, int oWm,
                               const __nv_bfloat16 *H, float *G, float *dH) {
    for (uint32_t u = blockIdx.x * blockDim.x + threadIdx.x; u < n; u += gridDim.x * blockDim.x) {
        float g[kC];
        for (int c = 0; c < kC; c++) {
            g[c] = dM[(size_t)u * kC + c] * s[u];
            G[(size_t)u * kC + c] = g[c];
        }
        for (int k = 0; k < kH; k++) {
            float d = dH[(size_t)u * kH + k];
            for (int c = 0; c < kC; c++) d += g[c] * P[oWm + c * kH + k];
            dH[(size_t)u * kH + k] = bf(H[(size_t)u * kH + k]) > 0.0f ? d : 0.0f;
        }
    }
}

// dZ1 = dPre1 W2 -> dH0 (first 32), dA1 (next 8)
__global__ void bwd_z1_kernel(uint32_t n, const float *dPre1, const float *P, float *dH0, float *dA1) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        float d[kH];
        for (int j = 0; j < kH; j++) d[j] = dPre1[(size_t)v * kH + j];
        for (int k = 0; k < kH + kC; k++) {
            float z = 0.0f;
            for (int j = 0; j < kH; j++) z += d[j] * P[oW2 + j * kZ + k];
            if (k < kH) dH0[(size_t)v * kH + k] = z;
            else dA1[(size_t)v * kC + (k - kH)] = z;
        }
    }
}

// Weight-gradient partials: part[block][o][i] = sum_v A[v][o] * B[v][i], with
// B = [B0 (I0 cols, BF16) | B1 (I1 cols, BF16)] and optional column sums of A
// (bias gradients) in part[block][O*I + o].  Fixed vertex ranges per block.
template <int O, int I0, int I1>
__global__ void __launch_bounds__(256) outer_kernel(uint32_t n, const float *A, const __nv_bfloat16 *B0, int ld0,
                                                    const __nv_bfloat16 *B1, int ld1, float *part, int stride) {
    constexpr int I = I0 + I1, OI = O * I, TV = 64;
    __shared__ float sA[TV][O];
    __shared__ float sB[TV][I];
    constexpr int PER = (OI + O + 255) / 256;
    float acc[PER];
#pragma unroll
    for (int k = 0; k < PER; k++) acc[k] = 0.0f;
    const uint64_t per_blk = ((uint64_t)n + gridDim.x - 1) / gridDim.x;
    const uint64_t lo = per_blk * blockIdx.x, hi = std::min<uint64_t>(lo + per_blk, n);
    for (uint64_t v0 = lo; v0 < hi; v0 += TV) {
        const int cnt = (int)std::min<uint64_t>(TV, hi - v0);
        __syncthreads();
        for (int i = threadIdx.x; i < TV * O; i += blockDim.x) {
            const int r = i / O, c = i % O;
            sA[r][c] = r < cnt ? A[(v0 + r) * O + c] : 0.0f;
        }
        for (int i = threadIdx.x; i < TV * I; i += blockDim.x) {
            const int r = i / I, c = i % I;
            float b = 0.0f;
            if (r < cnt) b = c < I0 ? bf(B0[(v0 + r) * ld0 + c]) : bf(B1[(v0 + r) * ld1 + (c - I0)]);
            sB[r][c] = b;
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < PER; k++) {
            const int idx = threadIdx.x + k * 256;
            if (idx < OI) {
                const int o = idx / I, i = idx % I;
                float a = acc[k];
                for (int r = 0; r < cnt; r++) a += sA[r][o] * sB[r][i];
                acc[k] = a;
            } else if (idx < OI + O) {
                const int o = idx - OI;
                float a = acc[k];
                for (int r = 0; r < cnt; r++) a += sA[r][o];
                acc[k] = a;
            }
        }
    }
#pragma unroll
    for (int k = 0; k < PER; k++) {
        const int idx = threadIdx.x + k * 256;
        if (idx < OI + O) part[(size_t)blockIdx.x * stride + idx] = acc[k];
    }
}

// grad[off + i] = sum over blocks of part[b][i]  (fixed order)
__global__ void reduce_part_kernel(const float *part, unsigned nb, int stride, int count, float *grad, int off) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (unsigned b = 0; b < nb; b++) s += part[(size_t)b * stride + i];
        grad[off + i] = (float)s;
    }
}

// dy-weighted outer products for the output layer (O = 1)
__global__ void __launch_bounds__(256) outer_out_kernel(uint32_t n, const float *dy, const __nv_bfloat16 *H1,
                                                        const __nv_bfloat16 *A2, float *part, int stride) {
    // threads 0..47: w3 row-0 entries; thread 48: b3
    float acc = 0.0f;
    const uint64_t per_blk = ((uint64_t)n + gridDim.x - 1) / gridDim.x;
    const uint64_t lo = per_blk * blockIdx.x, hi = std::min<uint64_t>(lo + per_blk, n);
    const int k = threadIdx.x;
    if (k <= kZ) {
        for (uint64_t v = lo; v < hi; v++) {
            float z = 1.0f;
            if (k < kH) z = bf(H1[v * kH + k]);
            else if (k < kZ) z = bf(A2[v * 16 + (k - kH)]);
            acc += dy[v] * z;
        }
        part[(size_t)blockIdx.x * stride + k] = acc;
    }
}

__global__ void adam_kernel(float *P, const float *G, float *m, float *v, int count, float lr, float b1, float b2,
                            float eps, float c1, float c2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const float g = G[i];
        const float mi = b1 * m[i] + (1.0f - b1) * g;
        const float vi = b2 * v[i] + (1.0f - b2) * g * g;
        m[i] = mi;
        v[i] = vi;
        P[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

__global__ void to_bf16_kernel(const float *P, Ws *w) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < kH * kF) w->W1[i] = __float2bfloat16_rn(P[oW1 + i]);
    if (i < kC * kH) w->Wm1[i] = __float2bfloat16_rn(P[oWm1 + i]);
    if (i < kH * kZ) w->W2[i] = __float2bfloat16_rn(P[oW2 + i]);
    if (i < kC * kH) w->Wm2[i] = __float2bfloat16_rn(P[oWm2 + i]);
    if (i < 8 * kZ) w->W3[i] = __float2bfloat16_rn(P[oW3 + i]);
}


// ---- fused inference path ---------------------------------------------------
// The same layer chain as the forward pass above, with the hidden layers kept
// in registers: the FP32 accumulator fragments of one mma.m16n8k16 are the
// BF16 A-operand fragments of the next layer once packed (C tile 2k / 2k+1
// of n-columns 16k..16k+15 -> A registers {0,1} / {2,3} of k-tile k), so H0
// and H1 never reach memory (they are recomputed where needed).  The
// rounding points and the mma sequence are those of rowwise_kernel, so the
// prediction is that of the training forward pass.

__device__ __forceinline__ float feat(uint32_t r, int c, uint32_t n, float ln, const uint32_t *row_ptr,
                                      const uint32_t *deg) {
    if (r >= n || c > 5) return 0.0f;
    const float li = log1pf((float)(row_ptr[r + 1] - row_ptr[r]));
    const float lo = log1pf((float)deg[r]);
    switch (c) {
        case 0: return li * 0.125f;
        case 1: return lo * 0.125f;
        case 2: return deg[r] == 0 ? 1.0f : 0.0f;
        case 3: return 1.0f;
        case 4: return (li - lo) * 0.125f;
        default: return ln;
    }
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};"
        : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// acc[j] += A(k-tiles) x W^T for n-tiles j < NT; W row-major [N x K] in smem
template <int NT, int KT>
__device__ __forceinline__ void layer(float (&acc)[NT][4], const uint32_t (&a)[KT][4], const __nv_bfloat16 *sW,
                                      int K, int g, int t) {
#pragma unroll
    for (int j = 0; j < NT; j++) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0f;
#pragma unroll
    for (int kt = 0; kt < KT; kt++) {
#pragma unroll
        for (int j = 0; j < NT; j++) {
            const int col = j * 8 + g;
            const uint32_t b0 = *reinterpret_cast<const uint32_t *>(sW + col * K + kt * 16 + 2 * t);
            const uint32_t b1 = *reinterpret_cast<const uint32_t *>(sW + col * K + kt * 16 + 2 * t + 8);
            mma_bf16(acc[j], a[kt], b0, b1);
        }
    }
}

// relu(acc + bias) -> BF16 A fragments of the next layer (32 columns = 2 k-tiles)
__device__ __forceinline__ void to_afrag(const float (&acc)[4][4], const float *bias, int t, uint32_t (&a)[2][4]) {
#pragma unroll
    for (int kt = 0; kt < 2; kt++) {
        float v[2][4];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int j = 2 * kt + h, c0 = j * 8 + 2 * t;
            v[h][0] = fmaxf(acc[j][0] + bias[c0], 0.0f);
            v[h][1] = fmaxf(acc[j][1] + bias[c0 + 1], 0.0f);
            v[h][2] = fmaxf(acc[j][2] + bias[c0], 0.0f);
            v[h][3] = fmaxf(acc[j][3] + bias[c0 + 1], 0.0f);
        }
        a[kt][0] = pack_bf16(v[0][0], v[0][1]);
        a[kt][1] = pack_bf16(v[0][2], v[0][3]);
        a[kt][2] = pack_bf16(v[1][0], v[1][1]);
        a[kt][3] = pack_bf16(v[1][2], v[1][3]);
    }
}

__device__ __forceinline__ uint32_t ld_pair(const __nv_bfloat16 *A, uint32_t r, uint32_t n, int k) {
    return r < n ? *reinterpret_cast<const uint32_t *>(A + (size_t)r * 16 + k) : 0u;
}

// STAGE 0: write M0 = s * (H0 Wm1^T); 1: write M1; 2: write y
template <int STAGE>
__global__ void __launch_bounds__(128) fused_kernel(uint32_t n, const uint32_t *row_ptr, const uint32_t *deg,
                                                    const __nv_bfloat16 *A1, const __nv_bfloat16 *A2, const Ws *Wg,
                                                    const float *P, const float *scale, float *out) {
    __shared__ __align__(16) __nv_bfloat16 sW1[kH * kF], sWm[kC * kH], sW2[kH * kZ], sW3[8 * kZ];
    __shared__ float sb1[kH], sb2[kH];
    for (int i = threadIdx.x; i < kH * kF; i += blockDim.x) sW1[i] = Wg->W1[i];
    for (int i = threadIdx.x; i < kC * kH; i += blockDim.x) sWm[i] = STAGE == 0 ? Wg->Wm1[i] : Wg->Wm2[i];
    for (int i = threadIdx.x; i < kH * kZ; i += blockDim.x) sW2[i] = Wg->W2[i];
    for (int i = threadIdx.x; i < 8 * kZ; i += blockDim.x) sW3[i] = Wg->W3[i];
    for (int i = threadIdx.x; i < kH; i += blockDim.x) {
        sb1[i] = P[oB1 + i];
        sb2[i] = P[oB2 + i];
    }
    __syncthreads();
    const float ln = logf((float)n) * 0.0625f;
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const uint32_t ntiles = (n + 15) / 16;
    const uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nwarps = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t tile = warp; tile < ntiles; tile += nwarps) {
        const uint32_t r0 = tile * 16 + g, r1 = r0 + 8;
        uint32_t ax[1][4];
        ax[0][0] = pack_bf16(feat(r0, 2 * t, n, ln, row_ptr, deg), feat(r0, 2 * t + 1, n, ln, row_ptr, deg));
        ax[0][1] = pack_bf16(feat(r1, 2 * t, n, ln, row_ptr, deg), feat(r1, 2 * t + 1, n, ln, row_ptr, deg));
        ax[0][2] = pack_bf16(feat(r0, 2 * t + 8, n, ln, row_ptr, deg), feat(r0, 2 * t + 9, n, ln, row_ptr, deg));
        ax[0][3] = pack_bf16(feat(r1, 2 * t + 8, n, ln, row_ptr, deg), feat(r1, 2 * t + 9, n, ln, row_ptr, deg));
        float acc[4][4];
        layer<4, 1>(acc, ax, sW1, kF, g, t);
        uint32_t ah[3][4];
        {
            uint32_t h0[2][4];
            to_afrag(acc, sb1, t, h0);
#pragma unroll
            for (int q = 0; q < 4; q++) {
                ah[0][q] = h0[0][q];
                ah[1][q] = h0[1][q];
            }
        }
        if constexpr (STAGE >= 1) {
            // k-tile 2 of [H0 | A1]
            ah[2][0] = ld_pair(A1, r0, n, 2 * t);
            ah[2][1] = ld_pair(A1, r1, n, 2 * t);
            ah[2][2] = ld_pair(A1, r0, n, 2 * t + 8);
            ah[2][3] = ld_pair(A1, r1, n, 2 * t + 8);
            layer<4, 3>(acc, ah, sW2, kZ, g, t);
            uint32_t h1[2][4];
            to_afrag(acc, sb2, t, h1);
#pragma unroll
            for (int q = 0; q < 4; q++) {
                ah[0][q] = h1[0][q];
                ah[1][q] = h1[1][q];
            }
        }
        if constexpr (STAGE <= 1) {
            float m[1][4];
            uint32_t a2[2][4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                a2[0][q] = ah[0][q];
                a2[1][q] = ah[1][q];
            }
            layer<1, 2>(m, a2, sWm, kH, g, t);
            const int c0 = 2 * t;
            if (r0 < n) {
                const float sc = scale[r0];
                out[(size_t)r0 * kC + c0] = m[0][0] * sc;
                out[(size_t)r0 * kC + c0 + 1] = m[0][1] * sc;
            }
            if (r1 < n) {
                const float sc = scale[r1];
                out[(size_t)r1 * kC + c0] = m[0][2] * sc;
                out[(size_t)r1 * kC + c0 + 1] = m[0][3] * sc;
            }
        } else {
            ah[2][0] = ld_pair(A2, r0, n, 2 * t);
            ah[2][1] = ld_pair(A2, r1, n, 2 * t);
            ah[2][2] = ld_pair(A2, r0, n, 2 * t + 8);
            ah[2][3] = ld_pair(A2, r1, n, 2 * t + 8);
            float yv[1][4];
            layer<1, 3>(yv, ah, sW3, kZ, g, t);
            if (t == 0) {
                if (r0 < n) out[r0] = yv[0][0] + P[oB3];
                if (r1 < n) out[r1] = yv[0][2] + P[oB3];
            }
        }
    }
}

template <int STAGE>
static void fused(uint32_t n, const DeviceGraph &g, const __nv_bfloat16 *A1, const __nv_bfloat16 *A2, const Ws *W,
                  const float *P, const float *scale, float *out, cudaStream_t s) {
    const uint32_t tiles = (n + 15) / 16;
    const unsigned grid = (unsigned)std::max<uint32_t>(1, std::min<uint32_t>((tiles + 3) / 4, 148u * 16u));
    fused_kernel<STAGE><<<grid, 128, 0, s>>>(n, g.row_ptr, g.deg, A1, A2, W, P, scale, out);
    PRG_CUDA(cudaGetLastError());
}

// ---- host side -------------------------------------------------------------

int param_count() { return kParams; }

void Net::init(uint64_t seed, cudaStream_t s) {
    std::vector<float> p(kParams, 0.0f);
    uint64_t st = seed;
    auto unit = [&]() {
        st += 0x9E3779B97F4A7C15ULL;
        uint64_t z = st;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        z ^= z >> 31;
        return (double)(z >> 11) * (1.0 / 9007199254740992.0);
    };
    auto fill = [&](int off, int rows, int cols) {
        const double a = std::sqrt(6.0 / (double)cols);
        for (int i = 0; i < rows * cols; i++) p[off + i] = (float)((2.0 * unit() - 1.0) * a);
    };
    fill(oW1, kH, kF);
    fill(oWm1, kC, kH);
    fill(oW2, kH, kZ);
    fill(oWm2, kC, kH);
    fill(oW3, 1, kZ);  // rows 1..7 of W3 stay zero
    for (int i = 0; i < kH; i++) p[oB1 + i] = 0.05f;
    for (int i = 0; i < kH; i++) p[oB2 + i] = 0.05f;
    set_params(p.data(), s);
}

void Net::alloc(cudaStream_t s) {
    if (P) return;
    PRG_CUDA(cudaMallocAsync((void **)&P, kParams * 4, s));
    PRG_CUDA(cudaMallocAsync((void **)&G, kParams * 4, s));
    PRG_CUDA(cudaMallocAsync((void **)&m, kParams * 4, s));
    PRG_CUDA(cudaMallocAsync((void **)&v, kParams * 4, s));
    PRG_CUDA(cudaMallocAsync((void **)&w, sizeof(Ws), s));
    // loss_grad writes only the used rows of W3 / entries of B3, so the
    // gradient's other slots must start (and stay) zero
    PRG_CUDA(cudaMemsetAsync(G, 0, kParams * 4, s));
    PRG_CUDA(cudaMemsetAsync(m, 0, kParams * 4, s));
    PRG_CUDA(cudaMemsetAsync(v, 0, kParams * 4, s));
    PRG_CUDA(cudaMemsetAsync(w, 0, sizeof(Ws), s));
}

void Net::set_params(const float *host, cudaStream_t s) {
    alloc(s);
    PRG_CUDA(cudaMemcpyAsync(P, host, kParams * 4, cudaMemcpyHostToDevice, s));
    to_bf16_kernel<<<(kH * kZ + 255) / 256, 256, 0, s>>>(P, (Ws *)w);
    PRG_CUDA(cudaGetLastError());
    PRG_CUDA(cudaStreamSynchronize(s));
}

void Net::get_params(float *host, cudaStream_t s) const {
    PRG_CUDA(cudaMemcpyAsync(host, P, kParams * 4, cudaMemcpyDeviceToHost, s));
    PRG_CUDA(cudaStreamSynchronize(s));
}

void Net::free(cudaStream_t s) {
    for (void *p : {(void *)P, (void *)G, (void *)m, (void *)v, (void *)w, (void *)buf})
        if (p) cudaFreeAsync(p, s);
    P = G = m = v = nullptr;
    w = nullptr;
    buf = nullptr;
    buf_n = 0;
}

// scratch layout per vertex (bytes): X0 32, H0 64, M0 32, A1 32, H1 64, M1 32,
// A2 32, y 4, s 4, dy 4, dH1 128, dA2 32, dM1 32, G1 32, dH0 128, dA1 32,
// dM0 32, G0 32, S1 32, S2 32  -> 832 bytes per vertex, plus partials.
constexpr size_t kPerVertex = 832;
constexpr unsigned kRedBlocks = 512;
constexpr int kPartStride = 2048;

void Net::ensure(uint32_t n, cudaStream_t s) {
    if (buf && buf_n >= n) return;
    if (buf) cudaFreeAsync(buf, s);
    buf_n = n;
    const size_t bytes = (size_t)n * kPerVertex + (size_t)kRedBlocks * kPartStride * 4 + 64 * 1024 +
                         (size_t)n * 4 + 8192;
    PRG_CUDA(cudaMallocAsync((void **)&buf, bytes, s));
}

struct Views {
    __nv_bfloat16 *X0, *H0, *A1, *H1, *A2;
    float *M0, *M1, *y, *s, *dy, *dH1, *dA2, *dM1, *G1, *dH0, *dA1, *dM0, *G0, *S1, *S2, *part, *fpart;
    double *dpart;
    uint32_t *heavy, *nheavy;
};

static Views views(unsigned char *b, uint32_t n) {
    Views V;
    size_t o = 0;
    auto take = [&](size_t bytes) {
        unsigned char *p = b + o;
        o += (bytes + 255) & ~(size_t)255;
        return p;
    };
    V.X0 = (__nv_bfloat16 *)take((size_t)n * 32);
    V.H0 = (__nv_bfloat16 *)take((size_t)n * 64);
    V.M0 = (float *)take((size_t)n * 32);
    V.A1 = (__nv_bfloat16 *)take((size_t)n * 32);
    V.H1 = (__nv_bfloat16 *)take((size_t)n * 64);
    V.M1 = (float *)take((size_t)n * 32);
    V.A2 = (__nv_bfloat16 *)take((size_t)n * 32);
    V.y = (float *)take((size_t)n * 4);
    V.s = (float *)take((size_t)n * 4);
    V.dy = (float *)take((size_t)n * 4);
    V.dH1 = (float *)take((size_t)n * 128);
    V.dA2 = (float *)take((size_t)n * 32);
    V.dM1 = (float *)take((size_t)n * 32);
    V.G1 = (float *)take((size_t)n * 32);
    V.dH0 = (float *)take((size_t)n * 128);
    V.dA1 = (float *)take((size_t)n * 32);
    V.dM0 = (float *)take((size_t)n * 32);
    V.G0 = (float *)take((size_t)n * 32);
    V.S1 = (float *)take((size_t)n * 32);
    V.S2 = (float *)take((size_t)n * 32);
    V.heavy = (uint32_t *)take((size_t)n * 4);
    V.part = (float *)take((size_t)kRedBlocks * kPartStride * 4);
    V.fpart = (float *)take(4096 * 4);
    V.dpart = (double *)take(4096 * 8);
    V.nheavy = (uint32_t *)take(256);
    return V;
}

static unsigned grid_n(uint32_t n) { return (unsigned)std::max<uint32_t>(1, std::min<uint32_t>((n + 255) / 256, 148 * 16)); }

void Net::forward(const DeviceGraph &g, cudaStream_t s) {
    ensure(g.n, s);
    Views V = views(buf, g.n);
    const Ws *W = (const Ws *)w;
    const uint32_t n = g.n;
    const unsigned gn = grid_n(n);
    features_kernel<<<gn, 256, 0, s>>>(n, g.row_ptr, g.deg, V.X0);
    scale_kernel<<<gn, 256, 0, s>>>(g.deg, n, V.s);
    PRG_CUDA(cudaGetLastError());
    rowwise<kF, 0, kH, EPI_RELU_BF16>(n, V.X0, nullptr, W->W1, P + oB1, nullptr, V.H0, nullptr, s);
    rowwise<kH, 0, kC, EPI_SCALE_F32>(n, V.H0, nullptr, W->Wm1, nullptr, V.s, nullptr, V.M0, s);
    for (int layer = 0; layer < 2; layer++) {
        const float *M = layer ? V.M1 : V.M0;
        __nv_bfloat16 *A = layer ? V.A2 : V.A1;
        float *S = layer ? V.S2 : V.S1;
        PRG_CUDA(cudaMemsetAsync(V.nheavy, 0, 4, s));
        aggregate_kernel<<<148 * 16, 256, 0, s>>>(n, g.row_ptr, g.col, M, A, S, V.heavy, V.nheavy);
        aggregate_heavy_kernel<<<148 * 4, 256, 0, s>>>(g.row_ptr, g.col, M, A, S, V.heavy, V.nheavy);
        PRG_CUDA(cudaGetLastError());
        if (layer == 0) {
            rowwise<kH, 16, kH, EPI_RELU_BF16>(n, V.H0, V.A1, W->W2, P + oB2, nullptr, V.H1, nullptr, s);
            rowwise<kH, 0, kC, EPI_SCALE_F32>(n, V.H1, nullptr, W->Wm2, nullptr, V.s, nullptr, V.M1, s);
        }
    }
    rowwise<kH, 16, 8, EPI_COL0_F32>(n, V.H1, V.A2, W->W3, P + oB3, nullptr, nullptr, V.y, s);
}

void Net::predict(const DeviceGraph &g, double *x_internal, cudaStream_t s) {
    // fused inference: M0, A1, M1, A2, y without materialising H0 / H1
    ensure(g.n, s);
    Views V = views(buf, g.n);
    const Ws *W = (const Ws *)w;
    const uint32_t n = g.n;
    scale_kernel<<<grid_n(n), 256, 0, s>>>(g.deg, n, V.s);
    fused<0>(n, g, nullptr, nullptr, W, P, V.s, V.M0, s);
    for (int layer = 0; layer < 2; layer++) {
        const float *M = layer ? V.M1 : V.M0;
        __nv_bfloat16 *A = layer ? V.A2 : V.A1;
        float *S = layer ? V.S2 : V.S1;
        PRG_CUDA(cudaMemsetAsync(V.nheavy, 0, 4, s));
        aggregate_kernel<<<148 * 16, 256, 0, s>>>(n, g.row_ptr, g.col, M, A, S, V.heavy, V.nheavy);
        aggregate_heavy_kernel<<<148 * 4, 256, 0, s>>>(g.row_ptr, g.col, M, A, S, V.heavy, V.nheavy);
        PRG_CUDA(cudaGetLastError());
        if (layer == 0) fused<1>(n, g, V.A1, nullptr, W, P, V.s, V.M1, s);
    }
    fused<2>(n, g, V.A1, V.A2, W, P, V.s, V.y, s);
    const unsigned gb = 296;
    max_kernel<<<gb, 256, 0, s>>>(V.y, g.n, V.fpart);
    expsum_kernel<<<gb, 256, 0, s>>>(V.y, g.n, V.fpart, gb, x_internal, V.dpart);
    normalise_kernel<<<gb, 256, 0, s>>>(x_internal, g.n, V.dpart, gb);
    PRG_CUDA(cudaGetLastError());
}

double Net::loss_grad(const DeviceGraph &g, const double *target_internal, cudaStream_t s) {
    forward(g, s);
    Views V = views(buf, g.n);
    const uint32_t n = g.n;
    const unsigned gn = grid_n(n);
    const unsigned gb = 296;
    loss_kernel<<<gb, 256, 0, s>>>(V.y, target_internal, n, V.dy, V.dpart);
    // output layer
    const unsigned nb = std::min<unsigned>(kRedBlocks, std::max<uint32_t>(1, (n + 1023) / 1024));
    outer_out_kernel<<<nb, 256, 0, s>>>(n, V.dy, V.H1, V.A2, V.part, kPartStride);
    reduce_part_kernel<<<1, 64, 0, s>>>(V.part, nb, kPartStride, kZ, G, oW3);
    reduce_part_kernel<<<1, 64, 0, s>>>(V.part + kZ, nb, kPartStride, 1, G, oB3);
    bwd_out_kernel<<<gn, 256, 0, s>>>(n, V.dy, P, V.dH1, V.dA2);
    // second aggregation (transposed) and message layer
    PRG_CUDA(cudaMemsetAsync(V.dM1, 0, (size_t)n * 32, s));
    scatter_kernel<<<gn, 256, 0, s>>>(n, g.row_ptr, g.col, V.dA2, V.S2, V.dM1);
    bwd_msg_kernel<<<gn, 256, 0, s>>>(n, V.dM1, V.s, P, oWm2, V.H1, V.G1, V.dH1);
    outer_kernel<kC, kH, 0><<<nb, 256, 0, s>>>(n, V.G1, V.H1, kH, nullptr, 0, V.part, kPartStride);
    reduce_part_kernel<<<4, 256, 0, s>>>(V.part, nb, kPartStride, kC * kH, G, oWm2);
    // layer 2 (dH1 now holds dPre1): dW2 over [H0 | A1 (16 incl. zero pad)] = 48
    // columns, i.e. W2's row layout, followed by b2 = column sums of dPre1
    outer_kernel<kH, kH, 16><<<nb, 256, 0, s>>>(n, V.dH1, V.H0, kH, V.A1, 16, V.part, kPartStride);
    reduce_part_kernel<<<8, 256, 0, s>>>(V.part, nb, kPartStride, kH * kZ + kH, G, oW2);
    bwd_z1_kernel<<<gn, 256, 0, s>>>(n, V.dH1, P, V.dH0, V.dA1);
    PRG_CUDA(cudaMemsetAsync(V.dM0, 0, (size_t)n * 32, s));
    scatter_kernel<<<gn, 256, 0, s>>>(n, g.row_ptr, g.col, V.dA1, V.S1, V.dM0);
    bwd_msg_kernel<<<gn, 256, 0, s>>>(n, V.dM0, V.s, P, oWm1, V.H0, V.G0, V.dH0);
    outer_kernel<kC, kH, 0><<<nb, 256, 0, s>>>(n, V.G0, V.H0, kH, nullptr, 0, V.part, kPartStride);
    reduce_part_kernel<<<4, 256, 0, s>>>(V.part, nb, kPartStride, kC * kH, G, oWm1);
    outer_kernel<kH, kF, 0><<<nb, 256, 0, s>>>(n, V.dH0, V.X0, kF, nullptr, 0, V.part, kPartStride);
    reduce_part_kernel<<<4, 256, 0, s>>>(V.part, nb, kPartStride, kH * kF + kH, G, oW1);
    PRG_CUDA(cudaGetLastError());
    std::vector<double> lp(gb);
    PRG_CUDA(cudaMemcpyAsync(lp.data(), V.dpart, gb * 8, cudaMemcpyDeviceToHost, s));
    PRG_CUDA(cudaStreamSynchronize(s));
    double l = 0.0;
    for (double x : lp) l += x;
    return l;
}

void Net::adam(float lr, cudaStream_t s) {
    step += 1;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - std::pow(b1, (float)step), c2 = 1.0f - std::pow(b2, (float)step);
    adam_kernel<<<(kParams + 255) / 256, 256, 0, s>>>(P, G, m, v, kParams, lr, b1, b2, 1e-8f, c1, c2);
    to_bf16_kernel<<<(kH * kZ + 255) / 256, 256, 0, s>>>(P, (Ws *)w);
    PRG_CUDA(cudaGetLastError());
}

}  // namespace gnn
}  // namespace prg
