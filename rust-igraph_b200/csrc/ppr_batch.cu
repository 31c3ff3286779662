// ppr_batch.cu — batched personalized PageRank: K reset vectors solved
// together as an FP32 SpMM over the resident in-CSR.
//
// Column k follows rust-igraph personalized_pagerank() semantics
// (personalized_pagerank.rs:65-182; the reset of column k is uniform over
// its seed list with duplicates adding weight, as personalized_pagerank_vs
// builds it at :241-268): start from the reset r_k, then
//     x'[v] = (1-d) r_k[v] + d (sum_{u->v} x[u]/outdeg[u] + dsum_k r_k[v])
// until the successive L1 change of that column is < tol.  Columns freeze
// individually: a converged column keeps its last iterate and is no longer
// written.
//
// Layout: columns are processed in tiles of W = 32*VEC.  A tile's iterate X
// and scaled iterate XT = X / outdeg live vertex-major (row v = W floats), so
// the gather of one source vertex is one coalesced 128*VEC-byte load of a
// warp: lane l owns columns [l*VEC, l*VEC+VEC).  One warp handles one
// destination row at a time.  Reset vectors are sparse: a per-vertex seed
// list (vertex-sorted CSR of (column, weight) entries).
//
// Undirected graphs can take Chebyshev semi-iteration in place of the plain
// step (tuning batch_cheb = 1; plain steps by default, because a tile runs
// until its slowest column freezes and a Chebyshev step reads one more
// iterate, so the fewer column-iterations did not shorten the batch).  The
// iteration x -> G(x) = d P^T(x/s) + d (dangling mass) r + (1-d) r has a real
// spectrum in [-d, d] there: P = D^-1 A is similar to
// the symmetric D^-1/2 A D^-1/2, and the dangling term only adds a block
// that is triangular to it.  Once the column's own contraction ratio
// (successive changes of its plain steps) has settled, it gives an interval
// [-beta, beta] (beta <= d), and each later step is
//     x_{k+1} = w_{k+1} (G(x_k) - x_{k-1}) + x_{k-1},
//     w_2 = 2 / (2 - beta^2),  w_{k+1} = 1 / (1 - beta^2 w_k / 4)
// (Golub & Varga's recurrence).  For a symmetric interval the iteration
// converges for every eigenvalue of modulus < 1, so a low estimate of beta
// only slows it.  The stop test is the reference's: the change a power step
// makes, ||G(x_k) - x_k||_1 < tol.  A column freezes only on a plain step,
// whose iterate is that G(x_k) (one that meets the test on a Chebyshev step
// takes one plain step more), so its answer lies within d/(1-d) tol of the
// fixed point, as the reference's answer does.  Directed graphs (complex
// spectra) always take the plain step.
//
// One cooperative persistent launch runs all iterations of a tile.  Phases
// are separated by a grid barrier whose spin is bounded: if a barrier does
// not complete within ~1.5 s the kernel records PRG_ERR_TIMEOUT in its status
// word and every block returns, so the host gets an error, not a hang.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "graph.cuh"
#include "prims.cuh"
#include "ppr_batch.cuh"

namespace prg {

constexpr int kBThreads = 256;
constexpr int kBWarps = kBThreads / 32;

struct ColState {
    double diff;      // last successive L1 change
    double dsum;      // dangling mass of the column's current iterate
    uint32_t iters;
    uint32_t active;  // 1 until the column converged or hit max_iter
    uint32_t final_buf;
    uint32_t cheb_steps;  // Chebyshev steps taken (0 = still in the plain phase, kChebOff = left for good)
    double prev_diff;     // the change before `diff`
    double prev_ratio;    // the contraction ratio before the last one
    double beta;          // Chebyshev interval half-width
    double omega;         // weight of the next step (0 = plain step)
    double best_diff;     // smallest change seen during the Chebyshev steps
    uint32_t stall;       // Chebyshev steps since best_diff last fell
    uint32_t pad2;
};

// A column leaves its plain steps once its contraction ratio diff/prev_diff
// has settled (two successive ratios within kChebSettle, at least
// kChebMinPower steps) or after kChebMaxPower steps; the ratio, which by
// then follows the slowest modes, times kChebMargin is the half-width beta.
constexpr uint32_t kChebMinPower = 6, kChebMaxPower = 24;
constexpr double kChebSettle = 0.01, kChebMargin = 1.05;
// FP32 rounding sets a floor under ||G(x) - x||_1 (about n ulp of the
// column's mass, which at n = 2 M sits near the 1e-8 tolerance): a weighted
// combination of iterates never becomes an exact FP32 fixed point, and plain
// FP32 steps started from a Chebyshev iterate at that floor can settle into a
// cycle of a few ulp flips.  So a Chebyshev column hands over to plain steps
// once its change is below kChebHandoff x tol (or has not reached a new
// minimum for kChebStall steps); the plain steps then converge as the
// reference's do, to the FP32 fixed point where the change is 0.  As a last
// guard, a plain column that makes no new minimum for kChebStall steps with
// its change within kChebFloor x tol freezes there (its answer G(x) is then
// within d/(1-d) of that change of the fixed point).
constexpr uint32_t kChebStall = 6, kChebOff = 0xFFFFFFFFu;
constexpr double kChebHandoff = 100.0, kChebFloor = 10.0;

struct TileArgs {
    const uint32_t *row_ptr;
    const uint32_t *col;
    const float *inv32;  // 1/outdeg (0 for dangling)
    uint32_t n;
    uint32_t tile_base;  // first global column of the tile
    uint32_t tile_w;     // live columns in this tile (<= W)
    uint32_t max_iter;
    const uint32_t *seed_ptr;  // n+1, vertex-sorted seed entries
    const uint32_t *seed_col;  // global column of each entry
    const float *seed_w;       // weight of each entry
    float *X[3];        // iterates; X[2] only with Chebyshev steps (x_{k-1})
    float *XT[2];
    int cheb;           // 1: Chebyshev semi-iteration (undirected graphs)
    ColState *cs;       // tile_w entries
    double *bpart;      // [gridDim][W][2] per-block (diff, dsum) partials
    uint32_t *bar;      // [0] arrivals, [1] generation
    int32_t *status;
    double damping;
    double tol;
    uint32_t bar_extra;  // arrivals a barrier waits for beyond the grid (0; >0 only to exercise the timeout)
};

// Grid barrier with a bounded spin (co-residency is guaranteed by the
// cooperative launch).  Returns false when it timed out or another block
// reported an error; callers then return.
__device__ __forceinline__ bool grid_sync(const TileArgs &a) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile uint32_t *gen = a.bar + 1;
        const uint32_t g0 = *gen;
        __threadfence();
        const uint32_t arrived = atomicAdd(a.bar, 1u);
        int ok = 1;
        if (arrived == gridDim.x - 1 + a.bar_extra) {
            a.bar[0] = 0u;
            __threadfence();
            atomicAdd(a.bar + 1, 1u);
        } else {
            uint32_t spins = 0;
            while (*gen == g0) {
                __nanosleep(64);
                if (++spins > (1u << 22)) {  // ~1.5 s (a phase takes milliseconds)
                    atomicExch(a.status, 7);  // PRG_ERR_TIMEOUT
                    ok = 0;
                    break;
                }
                if (*(volatile int32_t *)a.status != 0) {
                    ok = 0;
                    break;
                }
            }
        }
        __threadfence();
        if (*(volatile int32_t *)a.status != 0) ok = 0;
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

__device__ __forceinline__ void kahan_add(float &acc, float &c, float x) {
    const float y = __fsub_rn(x, c);
    const float t = __fadd_rn(acc, y);
    c = __fsub_rn(__fsub_rn(t, acc), y);
    acc = t;
}

template <int VEC>
struct Vec {
    float v[VEC];
};

// Iterates are rewritten every iteration of the persistent launch by other
// SMs, so they are read L2-coherently (ld.global.cg), never through L1 or the
// read-only path.
template <int VEC>
__device__ __forceinline__ Vec<VEC> ldv_cg(const float *p) {
    Vec<VEC> r;
    if constexpr (VEC == 4) {
        const float4 q = __ldcg(reinterpret_cast<const float4 *>(p));
        r.v[0] = q.x; r.v[1] = q.y; r.v[2] = q.z; r.v[3] = q.w;
    } else if constexpr (VEC == 2) {
        const float2 q = __ldcg(reinterpret_cast<const float2 *>(p));
        r.v[0] = q.x; r.v[1] = q.y;
    } else {
        r.v[0] = __ldcg(p);
    }
    return r;
}

template <int VEC>
__device__ __forceinline__ void stv(float *p, const Vec<VEC> &x) {
    if constexpr (VEC == 4) *reinterpret_cast<float4 *>(p) = make_float4(x.v[0], x.v[1], x.v[2], x.v[3]);
    else if constexpr (VEC == 2) *reinterpret_cast<float2 *>(p) = make_float2(x.v[0], x.v[1]);
    else *p = x.v[0];
}

// Reduces per-lane (diff, dsum) of the block's warps into bpart[block][col].
template <int VEC>
__device__ __forceinline__ void block_columns(const TileArgs &a, const double (&pd)[VEC], const double (&pds)[VEC],
                                              double *sh) {
    constexpr int W = 32 * VEC;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
#pragma unroll
    for (int j = 0; j < VEC; j++) {
        sh[(warp * W + lane * VEC + j) * 2] = pd[j];
        sh[(warp * W + lane * VEC + j) * 2 + 1] = pds[j];
    }
    __syncthreads();
    for (int c = threadIdx.x; c < W; c += blockDim.x) {
        double x = 0.0, y = 0.0;
        for (int w = 0; w < kBWarps; w++) {
            x += sh[(w * W + c) * 2];
            y += sh[(w * W + c) * 2 + 1];
        }
        a.bpart[((size_t)blockIdx.x * W + c) * 2] = x;
        a.bpart[((size_t)blockIdx.x * W + c) * 2 + 1] = y;
    }
}

// Column totals over blocks (fixed order) -> column state.  Block b handles
// columns b, b + gridDim.x, ...  `init`: only record the dangling mass.
template <int VEC>
__device__ __forceinline__ void reduce_columns(const TileArgs &a, int parity_new, bool init, double *sh) {
    constexpr int W = 32 * VEC;
    for (uint32_t c = blockIdx.x; c < a.tile_w; c += gridDim.x) {
        double x = 0.0, y = 0.0;
        for (uint32_t b = threadIdx.x; b < gridDim.x; b += blockDim.x) {
            x += __ldcg(&a.bpart[((size_t)b * W + c) * 2]);
            y += __ldcg(&a.bpart[((size_t)b * W + c) * 2 + 1]);
        }
        x = warp_sum(x);
        y = warp_sum(y);
        const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
        __syncthreads();
        if (l == 0) {
            sh[w * 2] = x;
            sh[w * 2 + 1] = y;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double tx = 0.0, ty = 0.0;
            for (int k = 0; k < kBWarps; k++) {
                tx += sh[k * 2];
                ty += sh[k * 2 + 1];
            }
            ColState &s = a.cs[c];
            if (init) {
                s.dsum = ty;
            } else if (s.active) {
                s.prev_diff = s.diff;
                s.diff = tx;
                s.dsum = ty;
                s.iters += 1u;
                const bool cheb_step = a.cheb && s.cheb_steps != 0u && s.cheb_steps != kChebOff;
                if (tx < a.tol && cheb_step && s.iters < a.max_iter) {
                    // met the test on a Chebyshev step, whose iterate is not
                    // G(x): one plain step more, and the column freezes on it
                    s.omega = 0.0;
                    s.cheb_steps = kChebOff;
                    s.stall = 0u;
                } else if (tx < a.tol || s.iters >= a.max_iter) {
                    s.active = 0u;
                    s.final_buf = (uint32_t)parity_new;
                } else if (a.cheb) {
                    const double ratio = s.prev_diff > 0.0 ? tx / s.prev_diff : a.damping;
                    if (s.cheb_steps == 0u && s.iters >= kChebMinPower &&
                        (fabs(ratio - s.prev_ratio) <= kChebSettle || s.iters >= kChebMaxPower)) {
                        // settled contraction ratio of the plain steps -> interval
                        double b = kChebMargin * ratio;
                        if (!(b > 0.05)) b = 0.05;
                        if (!(b < a.damping)) b = a.damping;
                        s.beta = b;
                        s.omega = 2.0 / (2.0 - b * b);
                        s.cheb_steps = 1u;
                        s.best_diff = tx;
                        s.stall = 0u;
                    } else if (s.cheb_steps > 0u) {
                        if (tx < s.best_diff) {
                            s.best_diff = tx;
                            s.stall = 0u;
                        } else {
                            s.stall += 1u;
                        }
                        if (s.cheb_steps != kChebOff) {
                            if (tx < kChebHandoff * a.tol || s.stall >= kChebStall) {
                                s.omega = 0.0;  // plain steps from here on
                                s.cheb_steps = kChebOff;
                                s.stall = 0u;
                            } else {
                                s.omega = 1.0 / (1.0 - 0.25 * s.beta * s.beta * s.omega);
                                s.cheb_steps += 1u;
                            }
                        } else if (s.stall >= kChebStall && tx < kChebFloor * a.tol) {
                            // plain steps caught in a rounding cycle at the
                            // FP32 floor: freeze with this step's G(x)
                            s.active = 0u;
                            s.final_buf = (uint32_t)parity_new;
                        }
                    }
                    s.prev_ratio = ratio;
                }
            }
        }
    }
}

template <int VEC>
__global__ void __launch_bounds__(kBThreads) ppr_tile_kernel(const TileArgs a) {
    constexpr int W = 32 * VEC;
    __shared__ double sh[kBWarps * W * 2];
    __shared__ int s_any;
    const int lane = threadIdx.x & 31;
    const uint32_t gw = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    const float d = (float)a.damping;

    // dangling mass of the start vectors (the resets)
    {
        double pd[VEC], pds[VEC];
#pragma unroll
        for (int j = 0; j < VEC; j++) pd[j] = pds[j] = 0.0;
        for (uint32_t v = gw; v < a.n; v += nw) {
            if (a.inv32[v] != 0.0f) continue;
            const Vec<VEC> x = ldv_cg<VEC>(a.X[0] + (size_t)v * W + lane * VEC);
#pragma unroll
            for (int j = 0; j < VEC; j++) pds[j] += (double)x.v[j];
        }
        block_columns<VEC>(a, pd, pds, sh);
        if (!grid_sync(a)) return;
        reduce_columns<VEC>(a, 0, true, sh);
        if (!grid_sync(a)) return;
    }

    for (uint32_t it = 0;; it++) {
        const int cur = it & 1, nxt = cur ^ 1;
        // iterate buffers: two in rotation, three with Chebyshev steps
        const int xc = a.cheb ? (int)(it % 3u) : cur;
        const int xn_ = a.cheb ? (int)((it + 1u) % 3u) : nxt;
        const int xp = (int)((it + 2u) % 3u);
        // column flags, dangling shares and step weights for this iteration
        // (column state was written by other blocks before the last barrier)
        bool act[VEC];
        float dsh[VEC], om[VEC];
        bool any_om = false;
#pragma unroll
        for (int j = 0; j < VEC; j++) {
            const uint32_t c = lane * VEC + j;
            act[j] = c < a.tile_w && __ldcg(&a.cs[c].active) != 0u;
            dsh[j] = act[j] ? (float)__ldcg(&a.cs[c].dsum) : 0.0f;
            om[j] = act[j] && a.cheb ? (float)__ldcg(&a.cs[c].omega) : 0.0f;
            any_om |= om[j] != 0.0f;
        }
        if (threadIdx.x < 32) {
            int anyc = 0;
            for (uint32_t c = threadIdx.x; c < a.tile_w; c += 32) anyc |= __ldcg(&a.cs[c].active) != 0u ? 1 : 0;
            anyc = __any_sync(0xffffffffu, anyc);
            if (threadIdx.x == 0) s_any = anyc;
        }
        __syncthreads();
        if (!s_any) break;

        double pd[VEC], pds[VEC];
#pragma unroll
        for (int j = 0; j < VEC; j++) pd[j] = pds[j] = 0.0;
        const float *XT = a.XT[cur];
        for (uint32_t v = gw; v < a.n; v += nw) {
            const uint32_t p0 = __ldg(&a.row_ptr[v]), p1 = __ldg(&a.row_ptr[v + 1]);
            // compensated (Kahan) FP32 accumulation: the error of a row sum
            // stays ~1 ulp however many in-arcs the row has
            float acc[VEC], cmp[VEC];
#pragma unroll
            for (int j = 0; j < VEC; j++) acc[j] = cmp[j] = 0.0f;
            for (uint32_t base = p0; base < p1; base += 32) {
                const uint32_t cnt = min(32u, p1 - base);
                const uint32_t mine = lane < cnt ? __ldg(&a.col[base + lane]) : 0u;
                uint32_t k = 0;
                for (; k + 4 <= cnt; k += 4) {
                    const uint32_t u0 = __shfl_sync(0xffffffffu, mine, k);
                    const uint32_t u1 = __shfl_sync(0xffffffffu, mine, k + 1);
                    const uint32_t u2 = __shfl_sync(0xffffffffu, mine, k + 2);
                    const uint32_t u3 = __shfl_sync(0xffffffffu, mine, k + 3);
                    const Vec<VEC> g0 = ldv_cg<VEC>(XT + (size_t)u0 * W + lane * VEC);
                    const Vec<VEC> g1 = ldv_cg<VEC>(XT + (size_t)u1 * W + lane * VEC);
                    const Vec<VEC> g2 = ldv_cg<VEC>(XT + (size_t)u2 * W + lane * VEC);
                    const Vec<VEC> g3 = ldv_cg<VEC>(XT + (size_t)u3 * W + lane * VEC);
#pragma unroll
                    for (int j = 0; j < VEC; j++) kahan_add(acc[j], cmp[j], (g0.v[j] + g1.v[j]) + (g2.v[j] + g3.v[j]));
                }
                for (; k < cnt; k++) {
                    const uint32_t u = __shfl_sync(0xffffffffu, mine, k);
                    const Vec<VEC> g = ldv_cg<VEC>(XT + (size_t)u * W + lane * VEC);
#pragma unroll
                    for (int j = 0; j < VEC; j++) kahan_add(acc[j], cmp[j], g.v[j]);
                }
            }
            // reset entries of this row (usually none)
            float r[VEC];
#pragma unroll
            for (int j = 0; j < VEC; j++) r[j] = 0.0f;
            const uint32_t s0 = __ldg(&a.seed_ptr[v]), s1 = __ldg(&a.seed_ptr[v + 1]);
            for (uint32_t e = s0; e < s1; e++) {
                const uint32_t c = __ldg(&a.seed_col[e]);
                const float w = __ldg(&a.seed_w[e]);
#pragma unroll
                for (int j = 0; j < VEC; j++)
                    if (c == a.tile_base + lane * VEC + j) r[j] += w;
            }
            const float iv = __ldg(&a.inv32[v]);
            const Vec<VEC> old = ldv_cg<VEC>(a.X[xc] + (size_t)v * W + lane * VEC);
            Vec<VEC> prev{};
            if (any_om) prev = ldv_cg<VEC>(a.X[xp] + (size_t)v * W + lane * VEC);
            Vec<VEC> xn, xtn;
#pragma unroll
            for (int j = 0; j < VEC; j++) {
                // personalized_pagerank.rs:169-170 in FP32: g = G(x_k)
                const float val = (1.0f - d) * r[j] + d * (acc[j] + dsh[j] * r[j]);
                // Chebyshev step, or the plain step when om == 0
                const float step = om[j] != 0.0f ? __fmaf_rn(om[j], val - prev.v[j], prev.v[j]) : val;
                xn.v[j] = act[j] ? step : old.v[j];
                xtn.v[j] = xn.v[j] * iv;
                if (act[j]) {
                    pd[j] += fabs((double)val - (double)old.v[j]);
                    if (iv == 0.0f) pds[j] += (double)xn.v[j];
                }
            }
            stv<VEC>(a.X[xn_] + (size_t)v * W + lane * VEC, xn);
            stv<VEC>(a.XT[nxt] + (size_t)v * W + lane * VEC, xtn);
        }
        block_columns<VEC>(a, pd, pds, sh);
        if (!grid_sync(a)) return;
        reduce_columns<VEC>(a, xn_, false, sh);
        if (!grid_sync(a)) return;
    }
}

// ---- host side -----------------------------------------------------------

__global__ void seeds_to_internal(uint32_t *v, uint32_t cnt, const uint32_t *iperm) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) v[i] = iperm[v[i]];
}

// X0 = reset (tile columns), XT0 = X0 / outdeg; X0 must be zeroed.
__global__ void seed_fill(const uint32_t *ent_v, const uint32_t *ent_col, const float *ent_w, uint32_t cnt,
                          uint32_t tile_base, uint32_t W, float *X0) {
    // one thread per (vertex run); duplicates of the same (v, col) add up in order
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
        if (i > 0 && ent_v[i - 1] == ent_v[i]) continue;  // first entry of its vertex run handles the run
        const uint32_t v = ent_v[i];
        for (uint32_t j = i; j < cnt && ent_v[j] == v; j++) {
            const uint32_t c = ent_col[j];
            if (c >= tile_base && c < tile_base + W) X0[(size_t)v * W + (c - tile_base)] += ent_w[j];
        }
    }
}

__global__ void scale_rows(const float *X, float *XT, const float *inv32, uint32_t n, uint32_t W) {
    const size_t total = (size_t)n * W;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x)
        XT[i] = X[i] * inv32[i / W];
}

// out[caller_row * K + tile_base + c] = X_final(c)[internal_row][c]
__global__ void tile_writeback(const float *X0, const float *X1, const float *X2, const ColState *cs, uint32_t n,
                               uint32_t W, uint32_t tile_w, uint32_t tile_base, uint32_t K, const uint32_t *perm,
                               float *out) {
    const size_t total = (size_t)n * tile_w;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (size_t)gridDim.x * blockDim.x) {
        const uint32_t v = (uint32_t)(i / tile_w), c = (uint32_t)(i % tile_w);
        const uint32_t fb = cs[c].final_buf;
        const float *X = fb == 2u ? X2 : fb == 1u ? X1 : X0;
        const uint32_t ov = perm ? perm[v] : v;
        out[(size_t)ov * K + tile_base + c] = X[(size_t)v * W + c];
    }
}

template <int VEC>
static void run_tile(const TileArgs &a, int grid, cudaStream_t s) {
    void *args[] = {(void *)&a};
    PRG_CUDA(cudaLaunchCooperativeKernel((const void *)ppr_tile_kernel<VEC>, dim3(grid), dim3(kBThreads), args, 0, s));
}

template <int VEC>
static int tile_grid() {
    int dev = 0, sms = 0, occ = 0;
    PRG_CUDA(cudaGetDevice(&dev));
    PRG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    PRG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, ppr_tile_kernel<VEC>, kBThreads, 0));
    return sms * std::max(occ, 1);
}

int ppr_batch(const DeviceGraph &g, uint32_t K, const uint64_t *seed_offsets, const uint32_t *seeds,
              double damping, double tol, uint32_t max_iter, uint32_t vec, float *d_out, BatchStats &st,
              cudaStream_t s) {
    st = BatchStats{};
    const uint32_t n = g.n;
    if (vec != 1 && vec != 2 && vec != 4) vec = 1;
    const uint32_t W = 32 * vec;
    // the persistent launch keeps every block resident: lane-per-row gathers
    // need the graph's ids < n and the column tiles below
    // seed entries (vertex, column, weight), weight 1/len like
    // personalized_pagerank_vs; vertex ids mapped to internal ids, then a
    // vertex-sorted CSR built on the host (a few hundred thousand entries)
    const uint64_t S = seed_offsets[K];
    std::vector<uint32_t> hv(S);
    std::memcpy(hv.data(), seeds, S * 4);
    auto A = [&](void **p, size_t bytes) { PRG_CUDA(cudaMallocAsync(p, std::max<size_t>(bytes, 16), s)); };
    uint32_t *ev = nullptr, *ecs = nullptr, *sptr = nullptr;
    float *ews = nullptr;
    A((void **)&ev, S * 4);
    A((void **)&ecs, S * 4);
    A((void **)&ews, S * 4);
    A((void **)&sptr, ((size_t)n + 1) * 4);
    if (g.iperm && S) {
        PRG_CUDA(cudaMemcpyAsync(ev, hv.data(), S * 4, cudaMemcpyHostToDevice, s));
        seeds_to_internal<<<64, 256, 0, s>>>(ev, (uint32_t)S, g.iperm);
        PRG_CUDA(cudaMemcpyAsync(hv.data(), ev, S * 4, cudaMemcpyDeviceToHost, s));
        PRG_CUDA(cudaStreamSynchronize(s));
    }
    std::vector<uint32_t> hptr((size_t)n + 1, 0), fill((size_t)n, 0);
    for (uint64_t i = 0; i < S; i++) hptr[hv[i] + 1]++;
    for (uint32_t v = 0; v < n; v++) hptr[v + 1] += hptr[v];
    std::vector<uint32_t> sv(S), sc(S);
    std::vector<float> sw(S);
    for (uint32_t k = 0; k < K; k++) {  // columns in order: stable within a vertex
        const uint64_t b = seed_offsets[k], e = seed_offsets[k + 1];
        const float w = (float)(1.0 / (double)(e - b));
        for (uint64_t i = b; i < e; i++) {
            const uint32_t v = hv[i];
            const uint32_t pos = hptr[v] + fill[v]++;
            sv[pos] = v;
            sc[pos] = k;
            sw[pos] = w;
        }
    }
    PRG_CUDA(cudaMemcpyAsync(ev, sv.data(), S * 4, cudaMemcpyHostToDevice, s));
    PRG_CUDA(cudaMemcpyAsync(ecs, sc.data(), S * 4, cudaMemcpyHostToDevice, s));
    PRG_CUDA(cudaMemcpyAsync(ews, sw.data(), S * 4, cudaMemcpyHostToDevice, s));
    PRG_CUDA(cudaMemcpyAsync(sptr, hptr.data(), ((size_t)n + 1) * 4, cudaMemcpyHostToDevice, s));
    uint32_t *kk = ev;

    // tile buffers (Chebyshev steps need a third iterate)
    const bool cheb = !g.directed && tuning().batch_cheb != 0;
    float *X[3] = {nullptr, nullptr, nullptr}, *XT[2];
    for (int i = 0; i < 2; i++) {
        A((void **)&X[i], (size_t)n * W * 4);
        A((void **)&XT[i], (size_t)n * W * 4);
    }
    if (cheb) {
        A((void **)&X[2], (size_t)n * W * 4);
    }
    const int grid = vec == 4 ? tile_grid<4>() : vec == 2 ? tile_grid<2>() : tile_grid<1>();
    ColState *cs = nullptr;
    double *bpart = nullptr;
    uint32_t *bar = nullptr;
    int32_t *status = nullptr;
    A((void **)&cs, (size_t)W * sizeof(ColState));
    A((void **)&bpart, (size_t)grid * W * 2 * sizeof(double));
    A((void **)&bar, 16);
    A((void **)&status, 16);
    cudaEvent_t e0, e1;
    PRG_CUDA(cudaEventCreate(&e0));
    PRG_CUDA(cudaEventCreate(&e1));
    PRG_CUDA(cudaEventRecord(e0, s));
    int rc = 0;
    std::vector<ColState> hcs(W);
    for (uint32_t tb = 0; tb < K && rc == 0; tb += W) {
        const uint32_t tw = std::min(W, K - tb);
        PRG_CUDA(cudaMemsetAsync(X[0], 0, (size_t)n * W * 4, s));
        seed_fill<<<std::max<uint32_t>(1, (uint32_t)std::min<uint64_t>((S + 255) / 256, 4096)), 256, 0, s>>>(
            kk, ecs, ews, (uint32_t)S, tb, W, X[0]);
        scale_rows<<<148 * 8, 256, 0, s>>>(X[0], XT[0], g.inv32, n, W);
        std::vector<ColState> init(W);
        for (uint32_t c = 0; c < W; c++) {
            std::memset(&init[c], 0, sizeof(ColState));
            init[c].active = c < tw ? 1u : 0u;
        }
        PRG_CUDA(cudaMemcpyAsync(cs, init.data(), W * sizeof(ColState), cudaMemcpyHostToDevice, s));
        PRG_CUDA(cudaMemsetAsync(bar, 0, 16, s));
        PRG_CUDA(cudaMemsetAsync(status, 0, 16, s));
        TileArgs a;
        std::memset(&a, 0, sizeof(a));
        a.row_ptr = g.row_ptr;
        a.col = g.col;
        a.inv32 = g.inv32;
        a.n = n;
        a.tile_base = tb;
        a.tile_w = tw;
        a.max_iter = max_iter;
        a.seed_ptr = sptr;
        a.seed_col = ecs;
        a.seed_w = ews;
        a.X[0] = X[0];
        a.X[1] = X[1];
        a.X[2] = X[2];
        a.XT[0] = XT[0];
        a.XT[1] = XT[1];
        a.cheb = cheb ? 1 : 0;
        a.cs = cs;
        a.bpart = bpart;
        a.bar = bar;
        a.status = status;
        a.damping = damping;
        a.tol = tol;
        a.bar_extra = tuning().batch_barrier_extra;
        if (vec == 4) run_tile<4>(a, grid, s);
        else if (vec == 2) run_tile<2>(a, grid, s);
        else run_tile<1>(a, grid, s);
        tile_writeback<<<148 * 8, 256, 0, s>>>(X[0], X[1], X[2], cs, n, W, tw, tb, K, g.perm, d_out);
        PRG_CUDA(cudaGetLastError());
        int32_t hs = 0;
        PRG_CUDA(cudaMemcpyAsync(&hs, status, 4, cudaMemcpyDeviceToHost, s));
        PRG_CUDA(cudaMemcpyAsync(hcs.data(), cs, W * sizeof(ColState), cudaMemcpyDeviceToHost, s));
        PRG_CUDA(cudaStreamSynchronize(s));
        if (hs != 0) rc = hs;
        for (uint32_t c = 0; c < tw; c++) {
            st.column_iters.push_back(hcs[c].iters);
            st.column_diff.push_back(hcs[c].diff);
            st.column_iterations += hcs[c].iters;
            st.max_iters = std::max(st.max_iters, hcs[c].iters);
        }
        st.tiles += 1;
        st.kernel_launches += 4;
    }
    PRG_CUDA(cudaEventRecord(e1, s));
    PRG_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    PRG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    st.ms = ms;
    st.vec = vec;
    st.grid = (uint32_t)grid;
    st.chebyshev = cheb ? 1u : 0u;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    for (void *p : {(void *)ev, (void *)ews, (void *)ecs, (void *)sptr, (void *)X[0], (void *)X[1], (void *)X[2],
                    (void *)XT[0], (void *)XT[1], (void *)cs, (void *)bpart, (void *)bar, (void *)status})
        if (p) cudaFreeAsync(p, s);
    PRG_CUDA(cudaStreamSynchronize(s));
    return rc;
}

}  // namespace prg
