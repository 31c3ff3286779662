// spmv.cu — the fused PageRank iteration: one kernel per power step.
//
// Work unit: a row-block (csr_build.cu) of the pull CSR.  One CUDA block of
// 256 threads handles one row-block:
//   stream  — a run of short rows: the block streams the rows' contiguous arc
//             range with 16-byte evict-first index loads, gathers the scaled
//             rank vector xt = x / outdeg through the read-only path
//             (evict-last in L2), stages the products in shared memory and
//             reduces each row with a power-of-two thread group;
//   long    — one row with cap < deg <= split: whole block, strided, tree sum;
//   chunk   — a slice of a hub row (deg > split); slices write partial sums
//             and the last slice to finish (atomic ticket) combines them in
//             slice order and finishes the row.
// The epilogue of every row is fused: teleport + dangling share + damping,
// the row's L1 change |x'[v]-x[v]|, the next dangling mass and the next
// scaled vector xt'[v] = x'[v] / outdeg[v].  Per-row-block partial sums are
// reduced in two fixed-order levels (groups of 256 row-blocks, then groups);
// the last group's block writes the iteration's scalars into Ctl and raises
// `done` when the stop rule holds, so later launches in the same CUDA graph
// return immediately.  No floating-point atomics: results are
// bit-reproducible run to run.
//
// Semantics mirror rust-igraph's loop body (pagerank.rs:107-140,
// pagerank_weighted.rs:129-159, personalized_pagerank.rs:149-182).
#include <cuda_runtime.h>
#include <stdint.h>

#include "prims.cuh"
#include "spmv.cuh"

namespace prg {

template <int MODE>
struct ModeT {
    using A = double;  // gather / accumulate type
};
template <>
struct ModeT<MODE_CORR32> {
    using A = float;
};

__device__ __forceinline__ void block_sum3(double &a, double &b, double &c, double *sh) {
    a = warp_sum(a);
    b = warp_sum(b);
    c = warp_sum(c);
    int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
    __syncthreads();
    if (l == 0) {
        sh[w] = a;
        sh[32 + w] = b;
        sh[64 + w] = c;
    }
    __syncthreads();
    if (w == 0) {
        a = l < nw ? sh[l] : 0.0;
        b = l < nw ? sh[32 + l] : 0.0;
        c = l < nw ? sh[64 + l] : 0.0;
        a = warp_sum(a);
        b = warp_sum(b);
        c = warp_sum(c);
    }
}

template <class A>
__device__ __forceinline__ A block_sum_t(A v, A *sh) {
    v = warp_sum(v);
    int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    A r = A(0);
    if (w == 0) {
        r = l < nw ? sh[l] : A(0);
        r = warp_sum(r);
    }
    return r;
}

__device__ __forceinline__ double4 ldcg4(const double4 *p) {
    const double2 a = __ldcg(reinterpret_cast<const double2 *>(p));
    const double2 b = __ldcg(reinterpret_cast<const double2 *>(p) + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}

// Scalars every row of a launch shares.
struct Uni {
    double d, dsum, tele, dshare;
};

template <int MODE>
__device__ __forceinline__ void epilogue(const IterArgs &a, const Uni &u, uint32_t v, typename ModeT<MODE>::A y,
                                         double &pd, double &pds, double &ps) {
    if constexpr (MODE == MODE_CORR32) {
        const float df = (float)u.d;
        const float t = a.t32 ? a.t32[v] : (float)a.inv_n;
        const float out = df * y + ((float)(u.d * u.dsum)) * t + a.b32[v];
        const float old = a.x32_in[v];
        a.x32_out[v] = out;
        pd += fabs((double)out - (double)old);
        const float iv = a.inv32[v];
        a.xt32_out[v] = out * iv;
        if (iv == 0.0f) pds += (double)out;
    } else {
        double out;
        if (a.t64) {
            // personalized_pagerank.rs:169-170
            const double t = a.t64[v];
            out = __dadd_rn(__dmul_rn(1.0 - u.d, t), __dmul_rn(u.d, __dadd_rn(y, __dmul_rn(u.dsum, t))));
        } else {
            // pagerank.rs:129: teleport + dangling_share + d * incoming
            out = __dadd_rn(__dadd_rn(u.tele, u.dshare), __dmul_rn(u.d, y));
        }
        const double old = a.x64_in[v];
        const double dv = a.dval[v];
        a.x64_out[v] = out;
        if constexpr (MODE == MODE_RESID64) {
            const double r = out - old;
            pd += fabs(r);
            ps += out;
            const float r32 = (float)r;
            a.b32_out[v] = r32;
            a.x32_out[v] = r32;  // the correction iteration starts from e0 = r
            a.xt32_out[v] = r32 * a.inv32[v];
            if (dv == 0.0) pds += (double)r32;
        } else {
            pd += fabs(out - old);
            if (dv == 0.0) {
                pds += out;
                a.xt64_out[v] = 0.0;
            } else {
                a.xt64_out[v] = out / dv;  // the reference's pr[u] / out_deg(u)
            }
        }
    }
}

template <int MODE>
__device__ __forceinline__ const typename ModeT<MODE>::A *gather_src(const IterArgs &a) {
    if constexpr (MODE == MODE_CORR32) return a.xt32_in;
    else return a.xt64_in;
}

// Accumulates (or stores) w * xt[col] for arcs [p_lo, p_hi) using aligned
// 16-byte index loads.  STORE: s_prod[p - p_lo] = product; else acc += product.
template <int MODE, bool W, bool STORE>
__device__ __forceinline__ void arc_products(const IterArgs &a, uint32_t p_lo, uint32_t p_hi,
                                             typename ModeT<MODE>::A *s_prod, typename ModeT<MODE>::A &acc) {
    using A = typename ModeT<MODE>::A;
    const A *xt = gather_src<MODE>(a);
    const uint32_t a0 = p_lo & ~3u;
    const uint32_t nvec = (p_hi - a0 + 3u) >> 2;
    const uint64_t pol_s = policy_evict_first(), pol_g = policy_evict_last();
    for (uint32_t vi = threadIdx.x; vi < nvec; vi += blockDim.x) {
        const uint32_t base = a0 + 4u * vi;
        const uint4 c = ld_stream_u4(reinterpret_cast<const uint4 *>(a.col + base), pol_s);
        const uint32_t cc[4] = {c.x, c.y, c.z, c.w};
        A wv[4] = {A(1), A(1), A(1), A(1)};
        if constexpr (W) {
            if constexpr (MODE == MODE_CORR32) {
                const float4 q = ld_stream_f4(reinterpret_cast<const float4 *>(a.w32 + base), pol_s);
                wv[0] = q.x; wv[1] = q.y; wv[2] = q.z; wv[3] = q.w;
            } else {
                const double2 q0 = ld_stream_d2(reinterpret_cast<const double2 *>(a.w64 + base), pol_s);
                const double2 q1 = ld_stream_d2(reinterpret_cast<const double2 *>(a.w64 + base + 2), pol_s);
                wv[0] = q0.x; wv[1] = q0.y; wv[2] = q1.x; wv[3] = q1.y;
            }
        }
        A g[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const uint32_t p = base + k;
            g[k] = (p >= p_lo && p < p_hi) ? ld_gather(xt + cc[k], pol_g) : A(0);
        }
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const uint32_t p = base + k;
            if (p >= p_lo && p < p_hi) {
                const A prod = W ? wv[k] * g[k] : g[k];
                if constexpr (STORE) s_prod[p - p_lo] = prod;
                else acc += prod;
            }
        }
    }
}

template <int MODE, bool W>
__global__ void __launch_bounds__(kThreads) iter_kernel(const IterArgs a) {
    using A = typename ModeT<MODE>::A;
    __shared__ A s_prod[2 * kCap];
    __shared__ uint32_t s_rp[kRowCap + 1];
    __shared__ double s_red[96];
    __shared__ A s_redA[32];
    __shared__ int s_flag;

    Ctl *ctl = a.ctl;
    if constexpr (MODE != MODE_RESID64) {
        if (*(volatile int32_t *)&ctl->done) return;
    }
    const uint32_t rb = blockIdx.x;
    const uint4 d = a.rb[rb];
    const uint32_t kind = d.z & 3u;
    const uint32_t tid = threadIdx.x;

    Uni u;
    u.d = a.damping;
    u.dsum = *(volatile double *)&ctl->dsum[a.parity];
    {
        const double nf = (double)a.n;
        u.tele = __ddiv_rn(1.0 - u.d, nf);
        u.dshare = __ddiv_rn(__dmul_rn(u.d, u.dsum), nf);
    }
    double pd = 0.0, pds = 0.0, ps = 0.0;

    if (kind == RB_STREAM) {
        const uint32_t r0 = d.x, r1 = d.y, nrows = r1 - r0;
        const uint32_t p0 = __ldg(&a.row_ptr[r0]);
        for (uint32_t i = tid; i <= nrows; i += blockDim.x) s_rp[i] = __ldg(&a.row_ptr[r0 + i]) - p0;
        __syncthreads();
        const uint32_t cnt = s_rp[nrows];
        A dummy = A(0);
        arc_products<MODE, W, true>(a, p0, p0 + cnt, s_prod, dummy);
        __syncthreads();
        uint32_t tpr = 32;
        while (tpr > 1 && tpr * nrows > blockDim.x) tpr >>= 1;
        const uint32_t ngrp = blockDim.x / tpr, grp = tid / tpr, gl = tid % tpr;
        const uint32_t rounds = (nrows + ngrp - 1) / ngrp;
        for (uint32_t rd = 0; rd < rounds; rd++) {
            const uint32_t row = rd * ngrp + grp;
            const bool valid = row < nrows;
            A acc = A(0);
            if (valid)
                for (uint32_t j = s_rp[row] + gl; j < s_rp[row + 1]; j += tpr) acc += s_prod[j];
            for (uint32_t o = tpr >> 1; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (valid && gl == 0) epilogue<MODE>(a, u, r0 + row, acc, pd, pds, ps);
        }
    } else {
        const uint32_t r = d.x;
        const uint32_t p0 = __ldg(&a.row_ptr[r]), p1 = __ldg(&a.row_ptr[r + 1]);
        uint32_t lo = p0, hi = p1;
        if (kind == RB_CHUNK) {
            const uint32_t c = d.z >> 2;
            lo = p0 + c * a.split;
            hi = min(p1, lo + a.split);
        }
        A acc = A(0);
        arc_products<MODE, W, false>(a, lo, hi, nullptr, acc);
        const A tot = block_sum_t<A>(acc, s_redA);
        if (tid == 0) {
            if (kind == RB_LONG) {
                epilogue<MODE>(a, u, r, tot, pd, pds, ps);
            } else {
                const Hub h = a.hubs[d.w];
                a.chunk_part[rb] = (double)tot;
                __threadfence();
                const uint32_t t = atomicAdd(&a.hub_ticket[d.w], 1u);
                if (t == h.nchunks - 1) {
                    __threadfence();
                    double y = 0.0;
                    for (uint32_t j = 0; j < h.nchunks; j++) y += __ldcg(&a.chunk_part[h.first_rb + j]);
                    double hd = 0.0, hds = 0.0, hs = 0.0;
                    epilogue<MODE>(a, u, r, (A)y, hd, hds, hs);
                    a.hub_rec[d.w] = make_double4(hd, hds, hs, 0.0);
                    a.hub_ticket[d.w] = 0u;
                }
            }
        }
    }

    // ---- deterministic two-level reduction of (diff, dangling, sum)
    block_sum3(pd, pds, ps, s_red);
    const uint32_t g = rb / kGroup;
    if (tid == 0) {
        a.rb_part[rb] = make_double4(pd, pds, ps, 0.0);
        __threadfence();
        const uint32_t gsize = min(kGroup, a.nrb - g * kGroup);
        const uint32_t t = atomicAdd(&a.grp_ticket[g], 1u);
        s_flag = (t == gsize - 1);
    }
    __syncthreads();
    if (!s_flag) return;
    __threadfence();
    {
        const uint32_t gsize = min(kGroup, a.nrb - g * kGroup);
        double x = 0.0, y = 0.0, z = 0.0;
        if (tid < gsize) {
            const double4 q = ldcg4(&a.rb_part[g * kGroup + tid]);
            x = q.x; y = q.y; z = q.z;
        }
        block_sum3(x, y, z, s_red);
        if (tid == 0) {
            a.grp_part[g] = make_double4(x, y, z, 0.0);
            a.grp_ticket[g] = 0u;
            __threadfence();
            const uint32_t t = atomicAdd(&ctl->groups_done, 1u);
            s_flag = (t == a.ngroups - 1);
        }
    }
    __syncthreads();
    if (!s_flag) return;
    __threadfence();
    {
        double x = 0.0, y = 0.0, z = 0.0;
        for (uint32_t i = tid; i < a.ngroups; i += blockDim.x) {
            const double4 q = ldcg4(&a.grp_part[i]);
            x += q.x; y += q.y; z += q.z;
        }
        block_sum3(x, y, z, s_red);
        double hx = 0.0, hy = 0.0, hz = 0.0;
        for (uint32_t i = tid; i < a.nhub; i += blockDim.x) {
            const double4 q = ldcg4(&a.hub_rec[i]);
            hx += q.x; hy += q.y; hz += q.z;
        }
        block_sum3(hx, hy, hz, s_red);
        if (tid == 0) {
            const double diff = x + hx, dsn = y + hy, sum = z + hz;
            ctl->groups_done = 0u;
            ctl->dsum[a.parity ^ 1] = dsn;
            if constexpr (MODE == MODE_RESID64) {
                ctl->rnorm = diff;
                ctl->gsum = sum;
                ctl->resid_passes += 1u;
                const double t = ctl->rho * diff;
                ctl->thr = t > ctl->floor_abs ? t : ctl->floor_abs;
                ctl->iters = 0u;
                ctl->done = 0;
                ctl->parity_last = a.parity;
            } else {
                ctl->diff = diff;
                ctl->iters += 1u;
                ctl->total_iters += 1u;
                ctl->parity_last = a.parity;
                if (diff < ctl->thr || ctl->iters >= ctl->max_iter) ctl->done = 1;
            }
            __threadfence();
        }
    }
}

void launch_iteration(int mode, bool weighted, const IterArgs &a, cudaStream_t s) {
    const dim3 grid(a.nrb), block(kThreads);
#define PRG_LAUNCH(M)                                                           \
    if (weighted) iter_kernel<M, true><<<grid, block, 0, s>>>(a);               \
    else iter_kernel<M, false><<<grid, block, 0, s>>>(a);
    switch (mode) {
        case MODE_PLAIN64: PRG_LAUNCH(MODE_PLAIN64); break;
        case MODE_PPR64: PRG_LAUNCH(MODE_PPR64); break;
        case MODE_RESID64: PRG_LAUNCH(MODE_RESID64); break;
        case MODE_CORR32: PRG_LAUNCH(MODE_CORR32); break;
        default: break;
    }
#undef PRG_LAUNCH
    PRG_CUDA(cudaGetLastError());
}

// ------------------------------------------------------------------ elementwise

constexpr unsigned kPrepBlocks = 148u * 4u;

__global__ void __launch_bounds__(kThreads) prepare64_kernel(uint32_t n, double *x, const float *e, double *xt,
                                                             const double *dval, double4 *part) {
    __shared__ double sh[96];
    double ds = 0.0, sm = 0.0, unused = 0.0;
    const uint64_t per = ((uint64_t)n + gridDim.x - 1) / gridDim.x;
    const uint64_t lo = per * blockIdx.x, hi = lo + per < n ? lo + per : n;
    for (uint64_t v = lo + threadIdx.x; v < hi; v += blockDim.x) {
        double xv = x[v];
        if (e) {
            xv += (double)e[v];
            x[v] = xv;
        }
        const double dv = dval[v];
        if (dv == 0.0) {
            ds += xv;
            xt[v] = 0.0;
        } else {
            xt[v] = xv / dv;
        }
        sm += xv;
    }
    block_sum3(ds, sm, unused, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = make_double4(ds, sm, 0.0, 0.0);
}

__global__ void __launch_bounds__(kThreads) prepare64_final(const double4 *part, unsigned nb, Ctl *ctl, int parity) {
    __shared__ double sh[96];
    double a = 0.0, b = 0.0, c = 0.0;
    for (unsigned i = threadIdx.x; i < nb; i += blockDim.x) {
        a += part[i].x;
        b += part[i].y;
    }
    block_sum3(a, b, c, sh);
    if (threadIdx.x == 0) {
        ctl->dsum[parity] = a;
        ctl->gsum = b;
    }
}

void launch_prepare64(const DeviceGraph &g, double *x, const float *e, double *xt, Ctl *ctl, int parity,
                      double4 *part, cudaStream_t s) {
    prepare64_kernel<<<kPrepBlocks, kThreads, 0, s>>>(g.n, x, e, xt, g.dval, part);
    prepare64_final<<<1, kThreads, 0, s>>>(part, kPrepBlocks, ctl, parity);
    PRG_CUDA(cudaGetLastError());
}

__global__ void normalise_kernel(double *x, uint32_t n, const Ctl *ctl) {
    const double s = ctl->gsum;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) x[v] = x[v] / s;
}

void launch_normalise(double *x, uint32_t n, const Ctl *ctl, cudaStream_t s) {
    normalise_kernel<<<kPrepBlocks, kThreads, 0, s>>>(x, n, ctl);
    PRG_CUDA(cudaGetLastError());
}

__global__ void fill_start_kernel(double *x, const double *t, uint32_t n) {
    const double u = 1.0 / (double)n;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        x[v] = t ? t[v] : u;
}

void launch_fill_start(double *x, const double *t, uint32_t n, cudaStream_t s) {
    fill_start_kernel<<<kPrepBlocks, kThreads, 0, s>>>(x, t, n);
    PRG_CUDA(cudaGetLastError());
}

}  // namespace prg
