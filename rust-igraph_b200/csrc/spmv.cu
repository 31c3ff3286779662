// spmv.cu — the fused PageRank iteration: one kernel launch per power step.
//
// Persistent grid (SMs x resident blocks) of 256-thread blocks; every warp
// walks the row-block list (csr_build.cu) with a static round-robin stride,
// prefetching its next descriptor.  Per row-block:
//   stream — <= 32 consecutive short rows with < kWarpBuf arcs: the warp
//            streams the contiguous arc range with 16-byte evict-first index
//            loads, gathers the scaled rank vector xt = x / outdeg through the
//            read-only path (evict-last in L2), stages the products in its
//            shared-memory buffer, then lane i sums row r0+i and runs its
//            epilogue (32 consecutive rows -> coalesced stores);
//   long   — one row: warp-strided accumulation, shuffle reduction;
//   chunk  — a slice of a hub row: the slice sum goes to chunk_part, and the
//            last slice to finish (atomic ticket) adds the slices in order
//            and runs the row's epilogue.
// The epilogue is fused: teleport + dangling share + damping, the row's L1
// change |x'[v]-x[v]|, the next dangling mass and the next scaled vector
// xt'[v] = x'[v] / outdeg[v].  Lanes accumulate (diff, dangling, sum) in
// FP64 registers; blocks reduce them with a fixed tree, and the last block to
// finish (atomic ticket) adds the block records and hub records in index
// order, writes the iteration's scalars into Ctl and raises `done` when the
// stop rule holds, so later launches in the same CUDA graph return at once.
// The schedule is static and no floating-point atomics are used, so results
// are bit-reproducible run to run on a given GPU model.
//
// Semantics mirror rust-igraph's loop body (pagerank.rs:107-140,
// pagerank_weighted.rs:129-159, personalized_pagerank.rs:149-182).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

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
template <>
struct ModeT<MODE_KRY32> {
    using A = float;
};

template <int MODE>
constexpr bool kIs32 = MODE == MODE_CORR32 || MODE == MODE_KRY32;
template <int MODE>
constexpr bool kIsKry = MODE == MODE_KRY32 || MODE == MODE_KRY64;

__device__ __forceinline__ void block_sum3(double &a, double &b, double &c, double *sh) {
    a = warp_sum(a);
    b = warp_sum(b);
    c = warp_sum(c);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
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

__device__ __forceinline__ double4 ldcg4(const double4 *p) {
    const double2 a = __ldcg(reinterpret_cast<const double2 *>(p));
    const double2 b = __ldcg(reinterpret_cast<const double2 *>(p) + 1);
    return make_double4(a.x, a.y, b.x, b.y);
}

// Scalars every row of a launch shares.
struct Uni {
    double d, dsum, tele, dshare;
};

// Epilogue operands of one row, loaded before the row's gathers so their
// latency overlaps them.
template <int MODE>
struct Pre {
    double old, dv, t;
    float iv;
};
template <>
struct Pre<MODE_CORR32> {
    float old, t, iv, b;
};
template <>
struct Pre<MODE_KRY32> {
    float in, rh, t;
};
template <>
struct Pre<MODE_KRY64> {
    double in, rh, t;
};
template <>
struct Pre<MODE_KRES64> {
    double old, t;
};
template <>
struct Pre<MODE_EIG64> {
    double in;
};

template <int MODE>
__device__ __forceinline__ Pre<MODE> epi_load(const IterArgs &a, uint32_t v) {
    Pre<MODE> p;
    if constexpr (MODE == MODE_KRY32) {
        p.in = __ldcs(a.x32_in + v);
        p.rh = a.rh32 ? __ldcs(a.rh32 + v) : 0.0f;
        p.t = a.t32 ? a.t32[v] : (float)a.inv_n;
    } else if constexpr (MODE == MODE_KRY64) {
        p.in = __ldcs(a.x64_in + v);
        p.rh = a.rh64 ? __ldcs(a.rh64 + v) : 0.0;
        p.t = a.t64 ? a.t64[v] : a.inv_n;
    } else if constexpr (MODE == MODE_KRES64) {
        p.old = __ldcs(a.x64_in + v);
        p.t = a.t64 ? a.t64[v] : 0.0;
    } else if constexpr (MODE == MODE_EIG64) {
        p.in = a.x64_in[v];
    } else if constexpr (MODE == MODE_CORR32) {
        p.old = a.x32_in[v];
        p.b = a.b32[v];
        p.iv = a.inv32[v];
        p.t = a.t32 ? a.t32[v] : (float)a.inv_n;
    } else {
        p.old = a.x64_in[v];
        p.dv = a.dval[v];
        p.t = a.t64 ? a.t64[v] : 0.0;
        if constexpr (MODE == MODE_RESID64) p.iv = a.inv32[v];
        else p.iv = 0.0f;
    }
    return p;
}

template <int MODE>
__device__ __forceinline__ void epilogue(const IterArgs &a, const Uni &u, uint32_t v, typename ModeT<MODE>::A y,
                                         const Pre<MODE> &p, double &pd, double &pds, double &ps) {
    if constexpr (MODE == MODE_EIG64) {
        const double out = a.shift * p.in + y;
        a.x64_out[v] = out;
        pd = fmax(pd, fabs(out));
        pds += p.in * out;
        ps += p.in * p.in;
    } else if constexpr (kIsKry<MODE>) {
        // y = p - d*sum - d*dsum_p*t; Uni::dshare holds d*dsum_p
        using A = typename ModeT<MODE>::A;
        const A out = p.in - ((A)u.d * y + (A)u.dshare * p.t);
        if constexpr (MODE == MODE_KRY32) __stcs(a.x32_out + v, out);
        else __stcs(a.x64_out + v, out);
        pd += (double)p.rh * (double)out;
        pds += (double)out * (double)p.in;
        ps += (double)out * (double)out;
    } else if constexpr (MODE == MODE_CORR32) {
        const float df = (float)u.d;
        const float out = df * y + ((float)(u.d * u.dsum)) * p.t + p.b;
        a.x32_out[v] = out;
        pd += fabs((double)out - (double)p.old);
        a.xt32_out[v] = out * p.iv;
        if (p.iv == 0.0f) pds += (double)out;
    } else {
        double out;
        if (a.t64) {
            // personalized_pagerank.rs:169-170
            out = __dadd_rn(__dmul_rn(1.0 - u.d, p.t), __dmul_rn(u.d, __dadd_rn(y, __dmul_rn(u.dsum, p.t))));
        } else {
            // pagerank.rs:129: teleport + dangling_share + d * incoming
            out = __dadd_rn(__dadd_rn(u.tele, u.dshare), __dmul_rn(u.d, y));
        }
        a.x64_out[v] = out;
        if constexpr (MODE == MODE_KRES64) {
            const double r = out - p.old;
            pd += fabs(r);
            ps += out;
            if (a.b64_out) __stcs(a.b64_out + v, r);
            else __stcs(a.b32_out + v, (float)r);
        } else if constexpr (MODE == MODE_RESID64) {
            const double r = out - p.old;
            pd += fabs(r);
            ps += out;
            const float r32 = (float)r;
            if (a.b64_out) a.b64_out[v] = r;
            if (a.b32_out) a.b32_out[v] = r32;
            if (a.x32_out) {
                a.x32_out[v] = r32;  // the correction iteration starts from e0 = r
                a.xt32_out[v] = r32 * p.iv;
            }
            if (p.dv == 0.0) pds += (double)r32;
        } else {
            pd += fabs(out - p.old);
            if (p.dv == 0.0) {
                pds += out;
                a.xt64_out[v] = 0.0;
            } else {
                a.xt64_out[v] = out / p.dv;  // the reference's pr[u] / out_deg(u)
            }
        }
    }
}

template <int MODE>
__device__ __forceinline__ const typename ModeT<MODE>::A *gather_src(const IterArgs &a) {
    if constexpr (kIs32<MODE>) return a.xt32_in;
    else return a.xt64_in;
}

// Products w * xt[col] of the 4 arcs at aligned position `base`; lanes outside
// [lo, hi) get 0 and issue no gather.  Sources below `hot` are read from the
// block's shared-memory copy of the rank vector's hot prefix (degree-sorted
// ids put the most-gathered vertices there): a warp's random shared-memory
// reads cost a few bank wavefronts where the same global gathers cost about
// one L1 wavefront per lane.
template <int MODE, bool W, bool HOT>
__device__ __forceinline__ void quad(const IterArgs &a, uint32_t base, uint32_t lo, uint32_t hi, uint64_t pol_s,
                                     uint64_t pol_g, const typename ModeT<MODE>::A *s_hot, uint32_t hot,
                                     typename ModeT<MODE>::A (&out)[4]) {
    using A = typename ModeT<MODE>::A;
    const A *xt = gather_src<MODE>(a);
    pol_s = policy_evict_first();
    pol_g = policy_evict_last();
    const uint4 c = ld_stream_u4(reinterpret_cast<const uint4 *>(a.col + base), pol_s);
    const uint32_t cc[4] = {c.x, c.y, c.z, c.w};
    A wv[4] = {A(1), A(1), A(1), A(1)};
    if constexpr (W) {
        if constexpr (kIs32<MODE>) {
            const float4 q = ld_stream_f4(reinterpret_cast<const float4 *>(a.w32 + base), pol_s);
            wv[0] = q.x; wv[1] = q.y; wv[2] = q.z; wv[3] = q.w;
        } else {
            const double2 q0 = ld_stream_d2(reinterpret_cast<const double2 *>(a.w64 + base), pol_s);
            const double2 q1 = ld_stream_d2(reinterpret_cast<const double2 *>(a.w64 + base + 2), pol_s);
            wv[0] = q0.x; wv[1] = q0.y; wv[2] = q1.x; wv[3] = q1.y;
        }
    }
#pragma unroll
    for (int k = 0; k < 4; k++) {
        const uint32_t p = base + k;
        A g = A(0);
        if (p >= lo && p < hi) {
            if constexpr (HOT) g = cc[k] < hot ? s_hot[cc[k]] : ld_gather(xt + cc[k], pol_g);
            else g = cc[k] < a.l1hot ? ld_gather(xt + cc[k], pol_g) : ld_gather_na(xt + cc[k], pol_g);
        }
        out[k] = W ? wv[k] * g : g;
    }
}

// Quads each lane has in flight per step of `stage`: 32-bit passes take four
// (16 gathers per lane outstanding), FP64 passes two (register budget).
template <int MODE>
constexpr int kStageQuads = kIs32<MODE> ? 4 : 2;

// Warp: stage products of arcs [lo, hi) (hi - lo <= kWarpBuf) into buf[p - lo].
// Each step issues the index loads and gathers of kStageQuads quads per lane
// before storing any product, so a stream row-block of <= kWarpBuf arcs takes
// one or two round trips to memory, not four.
template <int MODE, bool W, bool HOT>
__device__ __forceinline__ void stage(const IterArgs &a, uint32_t lo, uint32_t hi, typename ModeT<MODE>::A *buf,
                                      uint32_t lane, uint64_t pol_s, uint64_t pol_g,
                                      const typename ModeT<MODE>::A *s_hot, uint32_t hot) {
    using A = typename ModeT<MODE>::A;
    constexpr int QN = kStageQuads<MODE>;
    const uint32_t a0 = lo & ~3u;
    const uint32_t nvec = (hi - a0 + 3u) >> 2;
    for (uint32_t vi = lane; vi < nvec; vi += 32u * QN) {
        A g[QN][4];
#pragma unroll
        for (int j = 0; j < QN; j++) {
            const uint32_t q = vi + 32u * j;
            if (q < nvec) {
                quad<MODE, W, HOT>(a, a0 + 4u * q, lo, hi, pol_s, pol_g, s_hot, hot, g[j]);
            } else {
#pragma unroll
                for (int k = 0; k < 4; k++) g[j][k] = A(0);
            }
        }
#pragma unroll
        for (int j = 0; j < QN; j++) {
            const uint32_t q = vi + 32u * j;
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const uint32_t p = a0 + 4u * q + k;
                if (q < nvec && p >= lo && p < hi) buf[p - lo] = g[j][k];
            }
        }
    }
}

__device__ __forceinline__ void comp_add(float &acc, float &c, float x) {
    const float y = __fsub_rn(x, c);
    const float t = __fadd_rn(acc, y);
    c = __fsub_rn(__fsub_rn(t, acc), y);
    acc = t;
}
__device__ __forceinline__ void comp_add(double &acc, double &, double x) { acc += x; }

// Warp: sum of products of arcs [lo, hi) (any length), result in every lane.
// FP32 lanes accumulate with Kahan compensation so long (hub) rows keep
// ~1-ulp sums; FP64 lanes add plainly.
template <int MODE, bool W, bool HOT>
__device__ __forceinline__ typename ModeT<MODE>::A warp_row_sum(const IterArgs &a, uint32_t lo, uint32_t hi,
                                                                 uint32_t lane, uint64_t pol_s, uint64_t pol_g,
                                                                 const typename ModeT<MODE>::A *s_hot,
                                                                 uint32_t hot) {
    using A = typename ModeT<MODE>::A;
    const uint32_t a0 = lo & ~3u;
    const uint32_t nvec = (hi - a0 + 3u) >> 2;
    A acc0 = A(0), acc1 = A(0), c0 = A(0), c1 = A(0);
    uint32_t vi = lane;
    for (; vi + 32 < nvec; vi += 64) {
        A g0[4], g1[4];
        quad<MODE, W, HOT>(a, a0 + 4u * vi, lo, hi, pol_s, pol_g, s_hot, hot, g0);
        quad<MODE, W, HOT>(a, a0 + 4u * (vi + 32), lo, hi, pol_s, pol_g, s_hot, hot, g1);
        comp_add(acc0, c0, (g0[0] + g0[1]) + (g0[2] + g0[3]));
        comp_add(acc1, c1, (g1[0] + g1[1]) + (g1[2] + g1[3]));
    }
    if (vi < nvec) {
        A g0[4];
        quad<MODE, W, HOT>(a, a0 + 4u * vi, lo, hi, pol_s, pol_g, s_hot, hot, g0);
        comp_add(acc0, c0, (g0[0] + g0[1]) + (g0[2] + g0[3]));
    }
    return warp_sum((acc0 - c0) + (acc1 - c1));
}

// Dynamic shared memory layout: [NT/32 warp buffers of kWarpBuf][hot prefix].
// NT = kThreads: several blocks per SM, each with its own (small) hot prefix.
// NT = 512 / 1024 (hot variants only): one block per SM whose hot prefix takes
// the shared memory the warp buffers leave, up to ~48 K FP32 entries.
template <int MODE, bool W, bool HOT, int NT>
__global__ void __launch_bounds__(NT, NT != kThreads ? 1 : HOT ? (kIs32<MODE> ? 4 : 3) : 4)
    iter_kernel(const IterArgs a) {
    using A = typename ModeT<MODE>::A;
    constexpr int kW = NT / 32;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    A *s_buf = reinterpret_cast<A *>(smem_raw);
    A *s_hot = s_buf + kW * kWarpBuf;
    __shared__ double s_red[96];
    __shared__ int s_flag;

    Ctl *ctl = a.ctl;
    if constexpr (MODE == MODE_EIG64) {
        if (a.kdone && *(volatile const int32_t *)a.kdone) return;
    } else if constexpr (kIsKry<MODE>) {
        if (*(volatile const int32_t *)a.kdone) return;
    } else if constexpr (MODE != MODE_RESID64 && MODE != MODE_KRES64) {
        if (*(volatile int32_t *)&ctl->done) return;
    }
    const uint32_t hot = HOT ? a.hot : 0u;
    if (HOT && hot) {
        // hot prefix of the gathered vector -> shared memory (16-byte loads;
        // hot is a multiple of 4 and the vector is 256-byte aligned)
        const A *xt = gather_src<MODE>(a);
        constexpr int kPer = 16 / sizeof(A);
        for (uint32_t i = threadIdx.x * kPer; i < hot; i += NT * kPer)
            *reinterpret_cast<uint4 *>(s_hot + i) = __ldcg(reinterpret_cast<const uint4 *>(xt + i));
        __syncthreads();
    }
    const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    Uni u;
    u.d = a.damping;
    if constexpr (kIsKry<MODE>) {
        // dangling mass of the input vector: the producer's per-block
        // records summed in a fixed order (identical in every block)
        __shared__ double s_dz;
        __shared__ int s_skip;
        double dz = 0.0, z1 = 0.0, z2 = 0.0;
        for (uint32_t i = threadIdx.x; i < a.kpart_n; i += NT) {
            const double4 q = a.kpart_in[i];
            dz += q.x;
            z1 += q.y;
            z2 += q.z;
        }
        block_sum3(dz, z1, z2, s_red);
        if (threadIdx.x == 0) {
            s_dz = dz;
            // the BiCGStab half step already met the target: every block sums
            // the same records in the same order, so all of them skip together
            s_skip = a.ktol != nullptr && !((a.knorm2 ? sqrt(z2) : z1) > *a.ktol);
        }
        __syncthreads();
        if (s_skip) {
            if (blockIdx.x == 0 && threadIdx.x == 0) a.kpart_out[0] = make_double4(0.0, 0.0, 0.0, 1.0);
            return;
        }
        u.dsum = s_dz;
        u.tele = 0.0;
        u.dshare = u.d * u.dsum;
    } else if constexpr (MODE == MODE_EIG64) {
        u.dsum = u.tele = u.dshare = 0.0;
    } else {
        u.dsum = *(volatile double *)&ctl->dsum[a.parity];
        const double nf = (double)a.n;
        u.tele = __ddiv_rn(1.0 - u.d, nf);
        u.dshare = __ddiv_rn(__dmul_rn(u.d, u.dsum), nf);
    }
    const uint64_t pol_s = 0, pol_g = 0;  // created next to each load (saves registers)
    A *buf = s_buf + warp * kWarpBuf;
    double pd = 0.0, pds = 0.0, ps = 0.0;

    const uint32_t stride = gridDim.x * kW;
    uint32_t rb = blockIdx.x * kW + warp;
    uint4 d = rb < a.nrb ? __ldg(&a.rb[rb]) : make_uint4(0, 0, 0, 0);
    while (rb < a.nrb) {
        const uint32_t nxt = rb + stride;
        const uint4 dn = nxt < a.nrb ? __ldg(&a.rb[nxt]) : make_uint4(0, 0, 0, 0);
        if (d.y & kChunkFlag) {
            // slice of a hub row
            const A s = warp_row_sum<MODE, W, HOT>(a, d.z, d.w, lane, pol_s, pol_g, s_hot, hot);
            if (lane == 0) {
                const uint32_t h = d.y & ~kChunkFlag;
                const Hub hb = a.hubs[h];
                a.chunk_part[rb] = (double)s;
                __threadfence();
                const uint32_t t = atomicAdd(&a.hub_ticket[h], 1u);
                if (t == hb.nchunks - 1) {
                    __threadfence();
                    double y = 0.0;
                    for (uint32_t j = 0; j < hb.nchunks; j++) y += __ldcg(&a.chunk_part[hb.first_rb + j]);
                    double hd = 0.0, hds = 0.0, hs = 0.0;
                    const Pre<MODE> pr = epi_load<MODE>(a, hb.row);
                    epilogue<MODE>(a, u, hb.row, (A)y, pr, hd, hds, hs);
                    a.hub_rec[h] = make_double4(hd, hds, hs, 0.0);
                    a.hub_ticket[h] = 0u;
                }
            }
        } else if (d.y - d.x == 1u) {
            // a single row: whole warp
            Pre<MODE> pr;
            if (lane == 0) pr = epi_load<MODE>(a, d.x);
            const A s = warp_row_sum<MODE, W, HOT>(a, d.z, d.w, lane, pol_s, pol_g, s_hot, hot);
            if (lane == 0) epilogue<MODE>(a, u, d.x, s, pr, pd, pds, ps);
        } else {
            // 2..32 rows with < kWarpBuf arcs in total: products are staged in
            // the warp's buffer, then each row is summed by a group of tpr
            // lanes (the largest power of two with tpr * rows <= 32)
            const uint32_t r0 = d.x, p0 = d.z, nrows = d.y - r0;
            uint32_t tpr = 32;
            while (tpr > 1 && tpr * nrows > 32) tpr >>= 1;
            const uint32_t grp = lane / tpr, gl = lane % tpr;
            const bool has_row = grp < nrows;
            const uint32_t v = r0 + grp;
            uint32_t rs = 0, re = 0;
            Pre<MODE> pr;
            if (has_row) {
                rs = __ldg(&a.row_ptr[v]) - p0;
                re = __ldg(&a.row_ptr[v + 1]) - p0;
                if (gl == 0) pr = epi_load<MODE>(a, v);
            }
            stage<MODE, W, HOT>(a, p0, d.w, buf, lane, pol_s, pol_g, s_hot, hot);
            __syncwarp();
            A acc0 = A(0), acc1 = A(0);
            if (has_row) {
                uint32_t j = rs + gl;
                for (; j + tpr < re; j += 2 * tpr) {
                    acc0 += buf[j];
                    acc1 += buf[j + tpr];
                }
                if (j < re) acc0 += buf[j];
            }
            A acc = acc0 + acc1;
            for (uint32_t o = tpr >> 1; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
            if (has_row && gl == 0) epilogue<MODE>(a, u, v, acc, pr, pd, pds, ps);
            __syncwarp();
        }
        rb = nxt;
        d = dn;
    }

    // ---- deterministic reduction of (diff, dangling, sum): block tree, then
    // the last block adds block and hub records in index order
    if constexpr (MODE == MODE_EIG64) {
        // (max |y|, x.y, x.x): a max tree for the first, sums for the others
        double mx = pd;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        double z = 0.0;
        block_sum3(z, pds, ps, s_red);
        __syncthreads();
        if (lane == 0) s_red[warp] = mx;
        __syncthreads();
        if (threadIdx.x == 0) {
            for (int w = 1; w < kW; w++) mx = fmax(mx, s_red[w]);
            a.kpart_out[blockIdx.x] = make_double4(mx, pds, ps, 0.0);
        }
        return;
    }
    block_sum3(pd, pds, ps, s_red);
    if constexpr (kIsKry<MODE>) {
        // the consumer adds block and hub records itself
        if (threadIdx.x == 0) a.kpart_out[blockIdx.x] = make_double4(pd, pds, ps, 0.0);
        return;
    }
    if (threadIdx.x == 0) {
        a.blk_part[blockIdx.x] = make_double4(pd, pds, ps, 0.0);
        __threadfence();
        const uint32_t t = atomicAdd(&ctl->groups_done, 1u);
        s_flag = (t == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_flag) return;
    __threadfence();
    double x = 0.0, y = 0.0, z = 0.0;
    for (uint32_t i = threadIdx.x; i < gridDim.x; i += blockDim.x) {
        const double4 q = ldcg4(&a.blk_part[i]);
        x += q.x;
        y += q.y;
        z += q.z;
    }
    block_sum3(x, y, z, s_red);
    double hx = 0.0, hy = 0.0, hz = 0.0;
    for (uint32_t i = threadIdx.x; i < a.nhub; i += blockDim.x) {
        const double4 q = ldcg4(&a.hub_rec[i]);
        hx += q.x;
        hy += q.y;
        hz += q.z;
    }
    block_sum3(hx, hy, hz, s_red);
    if (threadIdx.x == 0) {
        const double diff = x + hx, dsn = y + hy, sum = z + hz;
        ctl->groups_done = 0u;
        ctl->dsum[a.parity ^ 1] = dsn;
        if constexpr (MODE == MODE_RESID64 || MODE == MODE_KRES64) {
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

template <int MODE, bool W, bool HOT, int NT>
static void kernel_config(uint32_t hot_entries, uint32_t blocks_per_sm, uint32_t n, LaunchCfg &c) {
    using A = typename ModeT<MODE>::A;
    static int sms = 0, smem_optin = 0;
    if (sms == 0) {
        int dev = 0;
        PRG_CUDA(cudaGetDevice(&dev));
        PRG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        PRG_CUDA(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    }
    const size_t bufs = (size_t)(NT / 32) * kWarpBuf * sizeof(A);
    size_t hot = 0;
    if (HOT) {
        // leave room for the kernel's static shared memory (reduction scratch)
        const size_t avail = ((size_t)smem_optin - bufs - 2048) / sizeof(A);
        hot = std::min<size_t>(std::min<size_t>(hot_entries, avail), n) & ~(size_t)3;
    }
    c.smem = bufs + hot * sizeof(A);
    c.hot = (uint32_t)hot;
    c.threads = NT;
    PRG_CUDA(cudaFuncSetAttribute(iter_kernel<MODE, W, HOT, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)c.smem));
    int occ = 0;
    PRG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, iter_kernel<MODE, W, HOT, NT>, NT, c.smem));
    int per = occ > 0 ? occ : 1;
    if (blocks_per_sm > 0 && (int)blocks_per_sm < per) per = (int)blocks_per_sm;
    c.grid = (unsigned)(sms * per);
}

template <int MODE, bool W>
static void hot_config(uint32_t hot, uint32_t hot_threads, uint32_t bps, uint32_t n, LaunchCfg &c) {
    if (hot_threads == 1024) kernel_config<MODE, W, true, 1024>(hot, bps, n, c);
    else if (hot_threads == 512) kernel_config<MODE, W, true, 512>(hot, bps, n, c);
    else kernel_config<MODE, W, true, kThreads>(hot, bps, n, c);
}

template <int MODE>
static void mode_config(bool weighted, uint32_t hot, uint32_t hot_threads, uint32_t bps, uint32_t n, LaunchCfg &c) {
    if (hot) {
        if (weighted) hot_config<MODE, true>(hot, hot_threads, bps, n, c);
        else hot_config<MODE, false>(hot, hot_threads, bps, n, c);
    } else {
        if (weighted) kernel_config<MODE, true, false, kThreads>(0, bps, n, c);
        else kernel_config<MODE, false, false, kThreads>(0, bps, n, c);
    }
}

LaunchCfg iteration_config(int mode, bool weighted, uint32_t hot_entries, uint32_t blocks_per_sm, uint32_t n,
                           uint32_t hot_threads) {
    LaunchCfg c;
    const uint32_t ht = hot_threads;
    switch (mode) {
        case MODE_PLAIN64: mode_config<MODE_PLAIN64>(weighted, hot_entries, ht, blocks_per_sm, n, c); break;
        case MODE_PPR64: mode_config<MODE_PPR64>(weighted, hot_entries, ht, blocks_per_sm, n, c); break;
        case MODE_RESID64: mode_config<MODE_RESID64>(weighted, hot_entries, ht, blocks_per_sm, n, c); break;
        case MODE_CORR32: mode_config<MODE_CORR32>(weighted, hot_entries, ht, blocks_per_sm, n, c); break;
        case MODE_KRY32: mode_config<MODE_KRY32>(weighted, hot_entries, ht, blocks_per_sm, n, c); break;
        case MODE_KRY64: mode_config<MODE_KRY64>(weighted, hot_entries, ht, blocks_per_sm, n, c); break;
        case MODE_EIG64: mode_config<MODE_EIG64>(weighted, hot_entries, ht, blocks_per_sm, n, c); break;
        default: mode_config<MODE_KRES64>(weighted, hot_entries, ht, blocks_per_sm, n, c); break;
    }
    return c;
}

template <int MODE, bool W>
static void hot_launch(const IterArgs &a, const LaunchCfg &c, cudaStream_t s) {
    const dim3 grid(c.grid), block(c.threads);
    if (c.threads == 1024) iter_kernel<MODE, W, true, 1024><<<grid, block, c.smem, s>>>(a);
    else if (c.threads == 512) iter_kernel<MODE, W, true, 512><<<grid, block, c.smem, s>>>(a);
    else iter_kernel<MODE, W, true, kThreads><<<grid, block, c.smem, s>>>(a);
}

template <int MODE>
static void mode_launch(bool weighted, const IterArgs &a, const LaunchCfg &c, cudaStream_t s) {
    const dim3 grid(c.grid), block(c.threads);
    if (c.hot) {
        if (weighted) hot_launch<MODE, true>(a, c, s);
        else hot_launch<MODE, false>(a, c, s);
    } else {
        if (weighted) iter_kernel<MODE, true, false, kThreads><<<grid, block, c.smem, s>>>(a);
        else iter_kernel<MODE, false, false, kThreads><<<grid, block, c.smem, s>>>(a);
    }
}

void launch_iteration(int mode, bool weighted, const IterArgs &a_in, const LaunchCfg &c, cudaStream_t s) {
    IterArgs a = a_in;
    a.hot = c.hot;
    a.l1hot = c.l1hot;
    if (c.seg && (mode == MODE_KRY32 || mode == MODE_KRY64 || mode == MODE_KRES64 || mode == MODE_PLAIN64 ||
                  mode == MODE_PPR64 || mode == MODE_EIG64)) {
        launch_seg(mode, a, c, s);
        return;
    }
    switch (mode) {
        case MODE_PLAIN64: mode_launch<MODE_PLAIN64>(weighted, a, c, s); break;
        case MODE_PPR64: mode_launch<MODE_PPR64>(weighted, a, c, s); break;
        case MODE_RESID64: mode_launch<MODE_RESID64>(weighted, a, c, s); break;
        case MODE_CORR32: mode_launch<MODE_CORR32>(weighted, a, c, s); break;
        case MODE_KRY32: mode_launch<MODE_KRY32>(weighted, a, c, s); break;
        case MODE_KRY64: mode_launch<MODE_KRY64>(weighted, a, c, s); break;
        case MODE_KRES64: mode_launch<MODE_KRES64>(weighted, a, c, s); break;
        case MODE_EIG64: mode_launch<MODE_EIG64>(weighted, a, c, s); break;
        default: break;
    }
    PRG_CUDA(cudaGetLastError());
}

// ------------------------------------------------------------------ gather probe

// Diagnostic: the FP32 matvec's gathers and nothing else, in the fastest
// arrangement measured for this access pattern: one 1024-thread block per SM,
// each thread streaming two 16-byte quads of col per step (grid-stride, so
// neighbouring warps read neighbouring quads, evict-first) and gathering
// their sources, with the first `hot` entries of x (degree-sorted graphs) in
// shared memory and the other ids >= l1hot gathered without L1 allocation.
// The sums go to out so nothing is optimised away.  No row structure, scan,
// reduction or epilogue: the time is a floor for any pass that reads this
// index stream and gathers once per arc.
constexpr int kProbeNT = 1024;
constexpr uint32_t kProbeHot = 49152;

__global__ void __launch_bounds__(kProbeNT, 1) gather_probe_kernel(const uint32_t *col, uint64_t arcs, const float *x,
                                                                   uint32_t hot, uint32_t l1hot, float *out) {
    extern __shared__ __align__(16) float s_hot[];
    for (uint32_t i = threadIdx.x * 4; i < hot; i += kProbeNT * 4)
        *reinterpret_cast<uint4 *>(s_hot + i) = __ldcg(reinterpret_cast<const uint4 *>(x + i));
    __syncthreads();
    const uint64_t nq = (arcs + 3) >> 2;  // col carries kColPad slots past the last arc
    const uint64_t pol_g = policy_evict_last();
    const uint64_t stride = (uint64_t)gridDim.x * kProbeNT;
    float acc = 0.f;
    auto g = [&](uint32_t v, uint64_t p) -> float {
        if (p >= arcs) return 0.f;
        if (v < hot) return s_hot[v];
        return v < l1hot ? ld_gather(x + v, pol_g) : ld_gather_na(x + v, pol_g);
    };
    for (uint64_t q0 = (uint64_t)blockIdx.x * kProbeNT + threadIdx.x; q0 < nq; q0 += 2 * stride) {
        uint4 c[2];
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const uint64_t q = q0 + u * stride;
            c[u] = q < nq ? ld_stream_u4(reinterpret_cast<const uint4 *>(col) + q, policy_evict_first())
                          : make_uint4(0u, 0u, 0u, 0u);
        }
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const uint64_t q = q0 + u * stride;
            const uint64_t p = q < nq ? 4 * q : arcs;
            acc += (g(c[u].x, p) + g(c[u].y, p + 1)) + (g(c[u].z, p + 2) + g(c[u].w, p + 3));
        }
    }
    out[(uint64_t)blockIdx.x * kProbeNT + threadIdx.x] = acc;
}

float gather_probe(const DeviceGraph &g, int reps, cudaStream_t s) {
    int dev = 0, sms = 0;
    PRG_CUDA(cudaGetDevice(&dev));
    PRG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const unsigned grid = (unsigned)sms;
    float *x = nullptr, *out = nullptr;
    PRG_CUDA(cudaMallocAsync((void **)&x, std::max<uint64_t>(g.n, 4) * 4, s));
    PRG_CUDA(cudaMallocAsync((void **)&out, (uint64_t)grid * kProbeNT * 4, s));
    PRG_CUDA(cudaMemsetAsync(x, 0, std::max<uint64_t>(g.n, 4) * 4, s));
    const uint32_t l1hot = g.perm != nullptr && g.l1_hot32 ? g.l1_hot32 : 0xFFFFFFFFu;
    const uint32_t hot = g.perm != nullptr ? std::min<uint32_t>(kProbeHot, g.n) & ~3u : 0u;
    const size_t smem = (size_t)hot * 4;
    PRG_CUDA(cudaFuncSetAttribute(gather_probe_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    cudaEvent_t e0, e1;
    PRG_CUDA(cudaEventCreate(&e0));
    PRG_CUDA(cudaEventCreate(&e1));
    gather_probe_kernel<<<grid, kProbeNT, smem, s>>>(g.col, g.arcs, x, hot, l1hot, out);  // warm-up
    PRG_CUDA(cudaEventRecord(e0, s));
    for (int r = 0; r < reps; r++) gather_probe_kernel<<<grid, kProbeNT, smem, s>>>(g.col, g.arcs, x, hot, l1hot, out);
    PRG_CUDA(cudaEventRecord(e1, s));
    PRG_CUDA(cudaGetLastError());
    PRG_CUDA(cudaEventSynchronize(e1));
    float ms = 0.f;
    PRG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFreeAsync(x, s);
    cudaFreeAsync(out, s);
    PRG_CUDA(cudaStreamSynchronize(s));
    return ms / (float)std::max(reps, 1);
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

void preload_gather_f64();  // csr_build.cu

void preload_fp64_support() {
    cudaFuncAttributes fa;
    PRG_CUDA(cudaFuncGetAttributes(&fa, fill_start_kernel));
    PRG_CUDA(cudaFuncGetAttributes(&fa, prepare64_kernel));
    PRG_CUDA(cudaFuncGetAttributes(&fa, prepare64_final));
    preload_gather_f64();
}

}  // namespace prg
