// segspmv.cu — the FP32 Krylov matvec y = A p (MODE_KRY32) as a
// tile-segmented pass over the in-CSR, for unweighted graphs.
//
// The row-block kernel (spmv.cu) walks rows: each warp stages a row-block's
// products and sums them per row, so every step waits on an index load and
// then on its gathers, and row pointers, descriptors and partial quads add
// load requests.  Here the arcs are cut into tiles of kSegTile = 256 and the
// pass streams them like a gather-only loop: a warp takes tiles in a
// grid-stride order (neighbouring warps read neighbouring tiles), each lane
// loads two 16-byte index quads and gathers their eight sources, and the row
// sums come from a segmented scan in registers (FP64 partial sums, so a row
// sum is rounded to FP32 once), driven by a bit per arc that
// marks the last arc of a row (built once per graph):
//   * in each lane, a running sum over its 4 arcs that restarts after a row end;
//   * across the 32 lanes, an inclusive scan of the lanes' open tails (5
//     shuffles) whose segment breaks come from one ballot of "lane holds a
//     row end", with no flag shuffles;
//   * the k-th row end of tile t belongs to nz_row[tile_j0[t] + k] (the rows
//     that have arcs, in order); its sum goes to the warp's shared buffer at
//     rank k, and the epilogues then run with lane i on rank i, so the loads
//     of the rows' operands coalesce.
// A row that began in an earlier tile is finished by a second, small kernel:
// tile t leaves the sum before its first row end (head) and the open sum
// after its last (tail); the row's total is the tails of the tiles it spans
// plus the head, added in tile order in FP64.  The same kernel applies the
// epilogue to the rows without arcs.  With degree-sorted ids the first 48 K
// entries of the gathered vector (about 45 % of the arcs' sources on R-MAT)
// sit in shared memory of the one 1024-thread block per SM.
//
// The epilogue and the records are those of iter_kernel<MODE_KRY32>:
//   y = p - d sum - d (dangling mass of p) t,  records (rh.y, y.p, y.y),
// with the dangling mass summed from the producer's block records in a fixed
// order and the half-step skip (ktol) decided the same way in both kernels.
// The schedule is static and all reductions use fixed trees, so the result
// is bit-reproducible run to run.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "prims.cuh"
#include "spmv.cuh"

namespace prg {

constexpr int kSegNT = 1024;       // threads of the tile kernel (one block per SM)
constexpr int kSegFixNT = 256;     // threads of the finishing kernel
constexpr uint32_t kSegHotMax = 49152;    // FP32 hot-prefix entries (192 KB of shared memory)
constexpr uint32_t kSegHotMax64 = 20480;  // FP64 hot-prefix entries (160 KB, beside 64 KB of row sums)

// ------------------------------------------------------------------ index build

__global__ void seg_rowend_kernel(const uint32_t *rp, uint32_t n, uint32_t *mask, uint32_t *nonempty) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        const uint32_t a = rp[v], b = rp[v + 1];
        nonempty[v] = b > a ? 1u : 0u;
        if (b > a) atomicOr(&mask[(b - 1) >> 5], 1u << ((b - 1) & 31));
    }
}

__global__ void seg_tilecount_kernel(const uint32_t *mask, uint64_t ntiles, uint32_t *cnt) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < ntiles;
         t += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t c = 0;
#pragma unroll
        for (int w = 0; w < (int)(kSegTile / 32); w++) c += __popc(mask[t * (kSegTile / 32) + w]);
        cnt[t] = c;
    }
}

__global__ void seg_split_rows_kernel(const uint32_t *nonempty, const uint32_t *pos, uint32_t n, uint32_t *nz,
                                      uint32_t *empty) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        if (nonempty[v]) nz[pos[v]] = v;
        else empty[v - pos[v]] = v;
    }
}

// Tiles whose first row end closes a row begun in an earlier tile: kind 1
// (short span) or 2 (more than kSegLongSpan tiles), else 0.
__global__ void seg_span_kind_kernel(const uint32_t *rp, const uint32_t *tile_j0, const uint32_t *nz, uint64_t ntiles,
                                     uint32_t *is_short, uint32_t *is_long) {
    for (uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; b < ntiles;
         b += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t k = 0;
        const uint32_t j = tile_j0[b];
        if (tile_j0[b + 1] != j) {
            const uint64_t t0 = rp[nz[j]] / kSegTile;
            if (t0 < b) k = b - t0 > kSegLongSpan ? 2u : 1u;
        }
        is_short[b] = k == 1u;
        is_long[b] = k == 2u;
    }
}

__global__ void seg_span_fill_kernel(const uint32_t *rp, const uint32_t *tile_j0, const uint32_t *nz, uint64_t ntiles,
                                     const uint32_t *is_short, const uint32_t *pos_short, const uint32_t *is_long,
                                     const uint32_t *pos_long, uint4 *span, uint4 *span_long) {
    for (uint64_t b = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; b < ntiles;
         b += (uint64_t)gridDim.x * blockDim.x) {
        if (!is_short[b] && !is_long[b]) continue;
        const uint32_t row = nz[tile_j0[b]];
        const uint4 e = make_uint4(row, (uint32_t)(rp[row] / kSegTile), (uint32_t)b, 0u);
        if (is_short[b]) span[pos_short[b]] = e;
        else span_long[pos_long[b]] = e;
    }
}

// Per-tile record of the 8-arcs-per-lane kernel: {tile_j0, the running
// row-end counts before mask words 0-3 and 4-7 as bytes, row ends in the
// tile | 1 << 31 when its first row end closes a row begun in an earlier
// tile}.
__global__ void seg_meta_kernel(const uint32_t *mask, const uint32_t *tile_j0, const uint32_t *rp,
                                const uint32_t *nz, uint64_t ntiles, uint4 *meta) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < ntiles;
         t += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = 0, c = 0;
#pragma unroll
        for (int w = 0; w < (int)(kSegTile / 32); w++) {
            if (w < 4) lo |= c << (8 * w);
            else hi |= c << (8 * (w - 4));
            c += __popc(mask[t * (kSegTile / 32) + w]);
        }
        const uint32_t j = tile_j0[t];
        const uint32_t began = c != 0u && (uint64_t)rp[nz[j]] < t * kSegTile ? 1u : 0u;
        meta[t] = make_uint4(j, lo, hi, c | began << 31);
    }
}

template <class T>
static T *salloc(uint64_t count, cudaStream_t s) {
    T *p = nullptr;
    PRG_CUDA(cudaMallocAsync((void **)&p, std::max<uint64_t>(count, 1) * sizeof(T), s));
    return p;
}

void seg_free(SegIndex &x, cudaStream_t s) {
    for (void *p : {(void *)x.mask, (void *)x.tile_j0, (void *)x.meta, (void *)x.nz_row, (void *)x.empty_row, (void *)x.head,
                    (void *)x.tail, (void *)x.span, (void *)x.span_long})
        if (p) cudaFreeAsync(p, s);
    x = SegIndex{};
}

void seg_build(const DeviceGraph &g, SegIndex &x, cudaStream_t s) {
    seg_free(x, s);
    const uint32_t n = g.n;
    const uint64_t ntiles = (g.arcs + kSegTile - 1) / kSegTile;
    const uint64_t words = ntiles * (kSegTile / 32) + 8;
    x.ntiles = ntiles;
    x.mask = salloc<uint32_t>(words, s);
    x.tile_j0 = salloc<uint32_t>(ntiles + 1, s);
    PRG_CUDA(cudaMemsetAsync(x.mask, 0, words * 4, s));
    uint32_t *nonempty = salloc<uint32_t>(n, s);
    uint32_t *pos = salloc<uint32_t>((uint64_t)n + 1, s);
    uint32_t *cnt = salloc<uint32_t>(ntiles, s);
    const unsigned gb = 148u * 8u;
    seg_rowend_kernel<<<gb, 256, 0, s>>>(g.row_ptr, n, x.mask, nonempty);
    seg_tilecount_kernel<<<gb, 256, 0, s>>>(x.mask, ntiles, cnt);
    PRG_CUDA(cudaGetLastError());
    exclusive_scan_u32(cnt, x.tile_j0, ntiles, s);
    exclusive_scan_u32(nonempty, pos, n, s);
    uint32_t nnz = 0;
    PRG_CUDA(cudaMemcpyAsync(&nnz, pos + n, 4, cudaMemcpyDeviceToHost, s));
    PRG_CUDA(cudaStreamSynchronize(s));
    x.n_nz = nnz;
    x.n_empty = n - nnz;
    x.nz_row = salloc<uint32_t>(x.n_nz, s);
    x.empty_row = salloc<uint32_t>(x.n_empty, s);
    seg_split_rows_kernel<<<gb, 256, 0, s>>>(nonempty, pos, n, x.nz_row, x.empty_row);
    if (nnz) {
        // nz_row is increasing and distinct, so it is the identity iff its last entry is nnz - 1
        uint32_t last = 0;
        PRG_CUDA(cudaMemcpyAsync(&last, x.nz_row + nnz - 1, 4, cudaMemcpyDeviceToHost, s));
        PRG_CUDA(cudaStreamSynchronize(s));
        x.dense = last == nnz - 1 ? 1u : 0u;
    }
    x.meta = salloc<uint4>(ntiles, s);
    seg_meta_kernel<<<gb, 256, 0, s>>>(x.mask, x.tile_j0, g.row_ptr, x.nz_row, ntiles, x.meta);
    PRG_CUDA(cudaGetLastError());
    x.head = salloc<double>(ntiles, s);
    x.tail = salloc<double>(ntiles, s);
    // the rows that span tiles, as two compacted lists in tile order
    uint32_t *is_short = salloc<uint32_t>(ntiles, s), *is_long = salloc<uint32_t>(ntiles, s);
    uint32_t *pos_short = salloc<uint32_t>(ntiles + 1, s), *pos_long = salloc<uint32_t>(ntiles + 1, s);
    seg_span_kind_kernel<<<gb, 256, 0, s>>>(g.row_ptr, x.tile_j0, x.nz_row, ntiles, is_short, is_long);
    PRG_CUDA(cudaGetLastError());
    exclusive_scan_u32(is_short, pos_short, ntiles, s);
    exclusive_scan_u32(is_long, pos_long, ntiles, s);
    uint32_t ns = 0, nl = 0;
    PRG_CUDA(cudaMemcpyAsync(&ns, pos_short + ntiles, 4, cudaMemcpyDeviceToHost, s));
    PRG_CUDA(cudaMemcpyAsync(&nl, pos_long + ntiles, 4, cudaMemcpyDeviceToHost, s));
    PRG_CUDA(cudaStreamSynchronize(s));
    x.n_span = ns;
    x.n_long = nl;
    x.span = salloc<uint4>(ns, s);
    x.span_long = salloc<uint4>(nl, s);
    seg_span_fill_kernel<<<gb, 256, 0, s>>>(g.row_ptr, x.tile_j0, x.nz_row, ntiles, is_short, pos_short, is_long,
                                            pos_long, x.span, x.span_long);
    PRG_CUDA(cudaGetLastError());
    for (void *p : {(void *)nonempty, (void *)pos, (void *)cnt, (void *)is_short, (void *)is_long,
                    (void *)pos_short, (void *)pos_long})
        cudaFreeAsync(p, s);
}

// ------------------------------------------------------------------ kernels

__device__ __forceinline__ void seg_block_sum3(double &a, double &b, double &c, double *sh) {
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

// Dangling mass of the input (the producer's block records summed in a
// fixed layout by the first kSegSumWarps warps, then in warp order by one
// thread, so both kernels of a launch and all their blocks get the same
// bits) and the half-step skip.  Returns false when the launch has nothing
// to do.
constexpr int kSegSumWarps = 8;  // both kernels have at least this many warps
__device__ __forceinline__ bool seg_prologue(const IterArgs &a, double &dz) {
    __shared__ double s_z[3][kSegSumWarps];
    __shared__ double s_dz;
    __shared__ int s_skip;
    const uint32_t w = threadIdx.x >> 5;
    if (w < (uint32_t)kSegSumWarps) {
        double z0 = 0.0, z1 = 0.0, z2 = 0.0;
        for (uint32_t i = threadIdx.x; i < a.kpart_n; i += 32 * kSegSumWarps) {
            const double4 q = a.kpart_in[i];
            z0 += q.x;
            z1 += q.y;
            z2 += q.z;
        }
        z0 = warp_sum(z0);
        z1 = warp_sum(z1);
        z2 = warp_sum(z2);
        if ((threadIdx.x & 31) == 0) {
            s_z[0][w] = z0;
            s_z[1][w] = z1;
            s_z[2][w] = z2;
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double z0 = 0.0, z1 = 0.0, z2 = 0.0;
        for (int k = 0; k < kSegSumWarps; k++) {
            z0 += s_z[0][k];
            z1 += s_z[1][k];
            z2 += s_z[2][k];
        }
        s_dz = z0;
        s_skip = a.ktol != nullptr && !((a.knorm2 ? sqrt(z2) : z1) > *a.ktol);
    }
    __syncthreads();
    dz = s_dz;
    return !s_skip;
}

// Epilogue operands of one row, loaded apart from the epilogue so that their
// latency can overlap other work.
struct SegPre {
    float in, rh, t;
};

struct SegEpi {
    float d, dshare;
    double pd, pds, ps;
    __device__ __forceinline__ SegPre load(const IterArgs &a, uint32_t v) const {
        SegPre q;
        q.in = __ldcs(a.x32_in + v);
        q.rh = a.rh32 ? __ldcs(a.rh32 + v) : 0.0f;
        q.t = a.t32 ? a.t32[v] : (float)a.inv_n;
        return q;
    }
    // y = p - (d sum + d dsum t) and its records, as iter_kernel<MODE_KRY32>
    __device__ __forceinline__ void fin(const IterArgs &a, uint32_t v, const SegPre &q, float sum) {
        const float out = q.in - (d * sum + dshare * q.t);
        __stcs(a.x32_out + v, out);
        pd += (double)q.rh * (double)out;
        pds += (double)out * (double)q.in;
        ps += (double)out * (double)out;
    }
    __device__ __forceinline__ void row(const IterArgs &a, uint32_t v, float sum) { fin(a, v, load(a, v), sum); }
};

// Segmented sums of one 128-arc block (lane owns 4 consecutive arcs).  v: the
// lane's products; f: their row-end bits.  carry: the open sum entering the
// block, updated to the one leaving it.  emit(rank, sum, first) for every
// row end in arc order, rank counted within the block, `first` for the
// block's first row end.
template <class Emit>
__device__ __forceinline__ void seg_block(const float (&v)[4], uint32_t f, double &carry, uint32_t lane, Emit emit) {
    // FP64 partial sums: a row's FP32 products are added exactly enough that
    // the row sum is rounded to FP32 once, at its end
    const double s0 = v[0];
    const double s1 = (f & 1u) ? (double)v[1] : s0 + v[1];
    const double s2 = (f & 2u) ? (double)v[2] : s1 + v[2];
    const double s3 = (f & 4u) ? (double)v[3] : s2 + v[3];
    const double sk[4] = {s0, s1, s2, s3};
    double tv = (f & 8u) ? 0.0 : s3;  // the lane's open tail
    const uint32_t E = __ballot_sync(0xffffffffu, f != 0u);
    // inclusive scan of the open tails; lane L stops adding once a lane of
    // the range it already covers, (L - o, L], holds a row end
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double ov = __shfl_up_sync(0xffffffffu, tv, o);
        if (lane >= (uint32_t)o) {
            const uint32_t hi = lane == 31u ? 0xffffffffu : ((1u << (lane + 1)) - 1u);
            const uint32_t rng = hi & ~((1u << (lane - o + 1)) - 1u);
            if ((E & rng) == 0u) tv += ov;
        }
    }
    double cin = __shfl_up_sync(0xffffffffu, tv, 1);
    const uint32_t below = E & lanemask_lt();
    if (lane == 0) cin = 0.0;
    if (below == 0u) cin += carry;
    uint32_t rank = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) rank += __popc(__ballot_sync(0xffffffffu, (f >> k) & 1u) & lanemask_lt());
    bool first = true;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        if ((f >> k) & 1u) {
            emit(rank, sk[k] + (first ? cin : 0.0), first && below == 0u);
            first = false;
            rank++;
        }
    }
    const double last = __shfl_sync(0xffffffffu, tv, 31);
    carry = E ? last : carry + last;
}

// Dynamic shared memory: [32 warp buffers of kSegTile row sums][hot prefix].
template <bool HOT>
__global__ void __launch_bounds__(kSegNT, 1) kry32_seg_kernel(const IterArgs a) {
    extern __shared__ __align__(16) float s_dyn[];
    float *s_sums = s_dyn;                            // per warp: the tile's row sums by rank
    float *s_hot = s_dyn + (kSegNT / 32) * kSegTile;  // hot prefix
    __shared__ double s_red[96];
    if (*(volatile const int32_t *)a.kdone) return;
    const uint32_t H = HOT ? a.hot : 0u;
    if (HOT) {
        // hot prefix of the gathered vector (H is a multiple of 4; the
        // vector is 256-byte aligned)
        for (uint32_t i = threadIdx.x * 4; i < H; i += kSegNT * 4)
            *reinterpret_cast<uint4 *>(s_hot + i) = __ldcg(reinterpret_cast<const uint4 *>(a.xt32_in + i));
    }
    double dz = 0.0;
    if (!seg_prologue(a, dz)) {
        if (blockIdx.x == 0 && threadIdx.x == 0) a.kpart_out[0] = make_double4(0.0, 0.0, 0.0, 1.0);
        return;
    }
    SegEpi ep{(float)a.damping, (float)(a.damping * dz), 0.0, 0.0, 0.0};
    const uint32_t lane = threadIdx.x & 31;
    float *sums = s_sums + (threadIdx.x >> 5) * kSegTile;
    const uint64_t warp = (blockIdx.x * (uint64_t)kSegNT + threadIdx.x) >> 5;
    const uint64_t nwarps = (gridDim.x * (uint64_t)kSegNT) >> 5;
    const float *xt = a.xt32_in;
    for (uint64_t t = warp; t < a.seg_ntiles; t += nwarps) {
        const uint64_t P0 = t * kSegTile;
        uint4 c[2];
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const uint64_t pos = P0 + 4u * (lane + 32u * u);
            // a quad that starts before the last arc stays inside col's padding
            c[u] = pos < a.arcs ? ld_stream_u4(reinterpret_cast<const uint4 *>(a.col + pos), policy_evict_first())
                                : make_uint4(0u, 0u, 0u, 0u);
        }
        const uint32_t mw0 = __ldg(&a.seg_mask[t * (kSegTile / 32) + (lane >> 3)]);
        const uint32_t mw1 = __ldg(&a.seg_mask[t * (kSegTile / 32) + 4 + (lane >> 3)]);
        const uint32_t j0 = __ldg(&a.seg_tile_j0[t]);
        float v[2][4];
        const uint64_t pol_g = policy_evict_last();
#pragma unroll
        for (int u = 0; u < 2; u++) {
            const uint32_t cc[4] = {c[u].x, c[u].y, c[u].z, c[u].w};
#pragma unroll
            for (int k = 0; k < 4; k++) {
                const uint64_t p = P0 + 4u * (lane + 32u * u) + k;
                float g = 0.0f;
                if (p < a.arcs) {
                    if (HOT && cc[k] < H) g = s_hot[cc[k]];
                    else g = cc[k] < a.l1hot ? ld_gather(xt + cc[k], pol_g) : ld_gather_na(xt + cc[k], pol_g);
                }
                v[u][k] = g;
            }
        }
        const uint32_t sh = (4u * lane) & 31u;
        const uint32_t f0 = (mw0 >> sh) & 0xFu, f1 = (mw1 >> sh) & 0xFu;
        const uint32_t cnt0 = __reduce_add_sync(0xffffffffu, __popc(f0));
        const uint32_t cnt = cnt0 + __reduce_add_sync(0xffffffffu, __popc(f1));
        double carry = 0.0;
        // each row end leaves its sum at its rank; the tile's first one also
        // as the head (the finishing kernel uses it when that row began in
        // an earlier tile)
        seg_block(v[0], f0, carry, lane, [&](uint32_t r, double sum, bool first) {
            sums[r] = (float)sum;
            if (first) a.seg_head[t] = sum;
        });
        seg_block(v[1], f1, carry, lane, [&](uint32_t r, double sum, bool first) {
            sums[cnt0 + r] = (float)sum;
            if (first && cnt0 == 0u) a.seg_head[t] = sum;
        });
        if (lane == 0) a.seg_tail[t] = carry;
        __syncwarp();
        // epilogues of the tile's rows, lane i taking rank i: their rows are
        // consecutive in nz_row order, so the operand loads coalesce
        for (uint32_t i = lane; i < cnt; i += 32) {
            const uint32_t row = __ldg(&a.seg_nz[j0 + i]);
            if (i == 0 && __ldg(&a.row_ptr[row]) < P0) continue;  // begun earlier: finished later
            ep.row(a, row, sums[i]);
        }
        __syncwarp();
    }
    seg_block_sum3(ep.pd, ep.pds, ep.ps, s_red);
    if (threadIdx.x == 0) a.kpart_out[blockIdx.x] = make_double4(ep.pd, ep.pds, ep.ps, 0.0);
}

// One 32-byte index load (eight consecutive u32, 32-byte aligned address),
// evict-first in L2 and not allocated in L1.
__device__ __forceinline__ void ld_stream_u8(const uint32_t *p, uint64_t pol, uint32_t (&c)[8]) {
    asm("ld.global.nc.L1::no_allocate.L2::cache_hint.v8.u32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8], %9;"
        : "=r"(c[0]), "=r"(c[1]), "=r"(c[2]), "=r"(c[3]), "=r"(c[4]), "=r"(c[5]), "=r"(c[6]), "=r"(c[7])
        : "l"(p), "l"(pol));
}

// ------------------------------------------------------------------ pass kinds
// The 8-arcs-per-lane tile kernel and the finishing kernel are shared by two
// passes, which differ in value type, gathered vector, prologue, epilogue and
// records:
//   Kry32Pass — the FP32 Krylov matvec above (MODE_KRY32);
//   Res64Pass — the FP64 residual pass r = G(x) - x of the refined and
//               Krylov solves (MODE_KRES64), with iter_kernel<MODE_KRES64>'s
//               epilogue and its Ctl bookkeeping done by the last finishing
//               block.

struct Kry32Pass {
    using V = float;
    using Pre = SegPre;
    SegEpi ep;
    __device__ static bool stopped(const IterArgs &a) { return *(volatile const int32_t *)a.kdone != 0; }
    __device__ static const float *source(const IterArgs &a) { return a.xt32_in; }
    // false: the half-step skip holds (the tile kernel's block 0 marks it)
    __device__ bool begin(const IterArgs &a, bool mark) {
        double dz = 0.0;
        if (!seg_prologue(a, dz)) {
            if (mark && blockIdx.x == 0 && threadIdx.x == 0) a.kpart_out[0] = make_double4(0.0, 0.0, 0.0, 1.0);
            return false;
        }
        ep = SegEpi{(float)a.damping, (float)(a.damping * dz), 0.0, 0.0, 0.0};
        return true;
    }
    __device__ Pre load(const IterArgs &a, uint32_t v) const { return ep.load(a, v); }
    __device__ void fin(const IterArgs &a, uint32_t v, const Pre &q, float sum) { ep.fin(a, v, q, sum); }
    __device__ void end(const IterArgs &a, unsigned rec0, double *s_red, bool) {
        seg_block_sum3(ep.pd, ep.pds, ep.ps, s_red);
        if (threadIdx.x == 0) a.kpart_out[rec0 + blockIdx.x] = make_double4(ep.pd, ep.pds, ep.ps, 0.0);
    }
};

// FP64 Krylov matvec (MODE_KRY64): iter_kernel<MODE_KRY64>'s epilogue,
// y = p - (d sum + d dsum t) with records (rh.y, y.p, y.y).
struct Kry64Pre {
    double in, rh, t;
};

struct Kry64Pass {
    using V = double;
    using Pre = Kry64Pre;
    double d, dshare, pd, pds, ps;
    __device__ static bool stopped(const IterArgs &a) { return *(volatile const int32_t *)a.kdone != 0; }
    __device__ static const double *source(const IterArgs &a) { return a.xt64_in; }
    __device__ bool begin(const IterArgs &a, bool mark) {
        double dz = 0.0;
        if (!seg_prologue(a, dz)) {
            if (mark && blockIdx.x == 0 && threadIdx.x == 0) a.kpart_out[0] = make_double4(0.0, 0.0, 0.0, 1.0);
            return false;
        }
        d = a.damping;
        dshare = a.damping * dz;
        pd = pds = ps = 0.0;
        return true;
    }
    __device__ Pre load(const IterArgs &a, uint32_t v) const {
        Pre q;
        q.in = __ldcs(a.x64_in + v);
        q.rh = a.rh64 ? __ldcs(a.rh64 + v) : 0.0;
        q.t = a.t64 ? a.t64[v] : a.inv_n;
        return q;
    }
    __device__ void fin(const IterArgs &a, uint32_t v, const Pre &q, double y) {
        const double out = q.in - (d * y + dshare * q.t);
        __stcs(a.x64_out + v, out);
        pd += q.rh * out;
        pds += out * q.in;
        ps += out * out;
    }
    __device__ void end(const IterArgs &a, unsigned rec0, double *s_red, bool) {
        seg_block_sum3(pd, pds, ps, s_red);
        if (threadIdx.x == 0) a.kpart_out[rec0 + blockIdx.x] = make_double4(pd, pds, ps, 0.0);
    }
};

// The adjacency product of the eigenvector and HITS iterations (MODE_EIG64,
// unweighted): y = shift x + A x with records (max |y|, x.y, x.x), the first
// a max over the block.
struct Eig64Pre {
    double in;
};

struct Eig64Pass {
    using V = double;
    using Pre = Eig64Pre;
    double shift, mx, xy, xx;
    __device__ static bool stopped(const IterArgs &a) { return a.kdone && *(volatile const int32_t *)a.kdone != 0; }
    __device__ static const double *source(const IterArgs &a) { return a.xt64_in; }
    __device__ bool begin(const IterArgs &a, bool) {
        shift = a.shift;
        mx = xy = xx = 0.0;
        __syncthreads();  // the hot prefix is in place
        return true;
    }
    __device__ Pre load(const IterArgs &a, uint32_t v) const { return Pre{a.x64_in[v]}; }
    __device__ void fin(const IterArgs &a, uint32_t v, const Pre &q, double y) {
        const double out = shift * q.in + y;
        a.x64_out[v] = out;
        mx = fmax(mx, fabs(out));
        xy += q.in * out;
        xx += q.in * q.in;
    }
    __device__ void end(const IterArgs &a, unsigned rec0, double *s_red, bool) {
        double m = mx;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
        double z = 0.0;
        seg_block_sum3(z, xy, xx, s_red);
        __syncthreads();
        const uint32_t w = threadIdx.x >> 5;
        if ((threadIdx.x & 31) == 0) s_red[w] = m;
        __syncthreads();
        if (threadIdx.x == 0) {
            for (uint32_t k = 1; k < (blockDim.x >> 5); k++) m = fmax(m, s_red[k]);
            a.kpart_out[rec0 + blockIdx.x] = make_double4(m, xy, xx, 0.0);
        }
    }
};

struct Res64Pre {
    double old, t;
};

struct Res64Pass {
    using V = double;
    using Pre = Res64Pre;
    double d, dsum, tele, dshare, pd, ps;
    __device__ static bool stopped(const IterArgs &) { return false; }
    __device__ static const double *source(const IterArgs &a) { return a.xt64_in; }
    __device__ bool begin(const IterArgs &a, bool) {
        d = a.damping;
        dsum = *(volatile const double *)&a.ctl->dsum[a.parity];
        const double nf = (double)a.n;
        tele = __ddiv_rn(1.0 - d, nf);
        dshare = __ddiv_rn(__dmul_rn(d, dsum), nf);
        pd = ps = 0.0;
        __syncthreads();  // the hot prefix is in place
        return true;
    }
    __device__ Pre load(const IterArgs &a, uint32_t v) const {
        Pre q;
        q.old = __ldcs(a.x64_in + v);
        q.t = a.t64 ? a.t64[v] : 0.0;
        return q;
    }
    // iter_kernel<MODE_KRES64>'s epilogue: x' = G(x), r = x' - x
    __device__ void fin(const IterArgs &a, uint32_t v, const Pre &q, double y) {
        double out;
        if (a.t64) out = __dadd_rn(__dmul_rn(1.0 - d, q.t), __dmul_rn(d, __dadd_rn(y, __dmul_rn(dsum, q.t))));
        else out = __dadd_rn(__dadd_rn(tele, dshare), __dmul_rn(d, y));
        a.x64_out[v] = out;
        const double r = out - q.old;
        pd += fabs(r);
        ps += out;
        if (a.b64_out) __stcs(a.b64_out + v, r);
        else __stcs(a.b32_out + v, (float)r);
    }
    // block record (|r|, 0, x'); the last block of the last kernel adds all
    // records in index order and updates Ctl as iter_kernel<MODE_KRES64> does
    __device__ void end(const IterArgs &a, unsigned rec0, double *s_red, bool last_stage) {
        __shared__ int s_last;
        double z = 0.0;
        seg_block_sum3(pd, z, ps, s_red);
        if (threadIdx.x == 0) {
            a.blk_part[rec0 + blockIdx.x] = make_double4(pd, z, ps, 0.0);
            if (last_stage) {
                __threadfence();
                s_last = atomicAdd(&a.ctl->groups_done, 1u) == gridDim.x - 1;
            }
        }
        if (!last_stage) return;
        __syncthreads();
        if (!s_last) return;
        __threadfence();
        const uint32_t nrec = rec0 + gridDim.x;
        double x = 0.0, y = 0.0, w = 0.0;
        for (uint32_t i = threadIdx.x; i < nrec; i += blockDim.x) {
            const double2 q0 = __ldcg(reinterpret_cast<const double2 *>(&a.blk_part[i]));
            const double2 q1 = __ldcg(reinterpret_cast<const double2 *>(&a.blk_part[i]) + 1);
            x += q0.x;
            y += q0.y;
            w += q1.x;
        }
        seg_block_sum3(x, y, w, s_red);
        if (threadIdx.x == 0) {
            Ctl *ctl = a.ctl;
            ctl->groups_done = 0u;
            ctl->dsum[a.parity ^ 1] = y;
            ctl->rnorm = x;
            ctl->gsum = w;
            ctl->resid_passes += 1u;
            const double t = ctl->rho * x;
            ctl->thr = t > ctl->floor_abs ? t : ctl->floor_abs;
            ctl->iters = 0u;
            ctl->done = 0;
            ctl->parity_last = a.parity;
            __threadfence();
        }
    }
};

// Bulk prefetch of `bytes` (a multiple of 16, 16-byte aligned address) into L2.
__device__ __forceinline__ void prefetch_l2(const void *p, uint32_t bytes) {
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

struct Plain64Pre {
    double old, dv, t;
};

// The FP64 power step of the drop-ins and the certified FP64 loop
// (MODE_PLAIN64 / MODE_PPR64): iter_kernel's epilogue (the reference's update
// in its rounding order, the L1 change, the next dangling mass, the next
// scaled vector x'/outdeg) and its Ctl bookkeeping, done by the last
// finishing block; both kernels return at once after convergence.
struct Plain64Pass {
    using V = double;
    using Pre = Plain64Pre;
    double d, dsum, tele, dshare, pd, pds;
    __device__ static bool stopped(const IterArgs &a) { return *(volatile const int32_t *)&a.ctl->done != 0; }
    __device__ static const double *source(const IterArgs &a) { return a.xt64_in; }
    __device__ bool begin(const IterArgs &a, bool) {
        d = a.damping;
        dsum = *(volatile const double *)&a.ctl->dsum[a.parity];
        const double nf = (double)a.n;
        tele = __ddiv_rn(1.0 - d, nf);
        dshare = __ddiv_rn(__dmul_rn(d, dsum), nf);
        pd = pds = 0.0;
        __syncthreads();  // the hot prefix is in place
        return true;
    }
    __device__ Pre load(const IterArgs &a, uint32_t v) const {
        Pre q;
        q.old = a.x64_in[v];
        q.dv = a.dval[v];
        q.t = a.t64 ? a.t64[v] : 0.0;
        return q;
    }
    __device__ void fin(const IterArgs &a, uint32_t v, const Pre &q, double y) {
        double out;
        if (a.t64) {
            // personalized_pagerank.rs:169-170
            out = __dadd_rn(__dmul_rn(1.0 - d, q.t), __dmul_rn(d, __dadd_rn(y, __dmul_rn(dsum, q.t))));
        } else {
            // pagerank.rs:129: teleport + dangling_share + d * incoming
            out = __dadd_rn(__dadd_rn(tele, dshare), __dmul_rn(d, y));
        }
        a.x64_out[v] = out;
        pd += fabs(out - q.old);
        if (q.dv == 0.0) {
            pds += out;
            a.xt64_out[v] = 0.0;
        } else {
            a.xt64_out[v] = out / q.dv;  // the reference's pr[u] / out_deg(u)
        }
    }
    // block record (|x' - x|, dangling x', 0); the last block of the last
    // kernel adds all records in index order and updates Ctl as
    // iter_kernel<MODE_PLAIN64> does
    __device__ void end(const IterArgs &a, unsigned rec0, double *s_red, bool last_stage) {
        __shared__ int s_last;
        double z = 0.0;
        seg_block_sum3(pd, pds, z, s_red);
        if (threadIdx.x == 0) {
            a.blk_part[rec0 + blockIdx.x] = make_double4(pd, pds, z, 0.0);
            if (last_stage) {
                __threadfence();
                s_last = atomicAdd(&a.ctl->groups_done, 1u) == gridDim.x - 1;
            }
        }
        if (!last_stage) return;
        __syncthreads();
        if (!s_last) return;
        __threadfence();
        const uint32_t nrec = rec0 + gridDim.x;
        double x = 0.0, y = 0.0, w = 0.0;
        for (uint32_t i = threadIdx.x; i < nrec; i += blockDim.x) {
            const double2 q0 = __ldcg(reinterpret_cast<const double2 *>(&a.blk_part[i]));
            const double2 q1 = __ldcg(reinterpret_cast<const double2 *>(&a.blk_part[i]) + 1);
            x += q0.x;
            y += q0.y;
            w += q1.x;
        }
        seg_block_sum3(x, y, w, s_red);
        if (threadIdx.x == 0) {
            Ctl *ctl = a.ctl;
            ctl->groups_done = 0u;
            ctl->dsum[a.parity ^ 1] = y;
            ctl->diff = x;
            ctl->iters += 1u;
            ctl->total_iters += 1u;
            ctl->parity_last = a.parity;
            if (x < ctl->thr || ctl->iters >= ctl->max_iter) ctl->done = 1;
            __threadfence();
        }
    }
};

// The tile kernel with lane L owning the 8 consecutive arcs 8L..8L+7 of the
// tile (one 32-byte index load, one scan per tile):
//   * in the lane, a running FP64 sum over its arcs that restarts after each
//     row end; the rows that begin and end inside the lane go straight to
//     the warp's buffer, the part before the lane's first row end is kept;
//   * across lanes, one unsegmented inclusive scan S of the lanes' open
//     tails with exclusive form X; the row that closes first in lane L began
//     after the last row end in a lane jb < L (jb = 0 if none), so its sum is
//     the kept part + X[L] - X[jb];
//   * ranks come from the tile record (row ends before the lane's mask word)
//     and the population count of the word's lower bits.
// The operands of the tile's first 32 rows are loaded while the gathers are
// in flight.  With HOT, sources at or above the hot prefix are gathered
// without L1 allocation.  Dynamic shared memory: [NT/32 warp buffers of
// kSegTile row sums][hot prefix], both of the pass's value type.  NT threads
// in one block per SM; with PIPE each warp loads its next tile's indices,
// mask word and record while it works on the current one.
template <class P, bool HOT, int NT, bool PIPE>
__global__ void __launch_bounds__(NT, 1) seg8_kernel(const IterArgs a) {
    using V = typename P::V;
    extern __shared__ __align__(16) unsigned char s_raw[];
    V *s_sums = reinterpret_cast<V *>(s_raw);         // per warp: the tile's row sums by rank
    V *s_hot = s_sums + (NT / 32) * kSegTile;         // hot prefix
    __shared__ double s_red[96];
    if (P::stopped(a)) return;
    const uint32_t H = HOT ? a.hot : 0u;
    const V *xt = P::source(a);
    if (HOT) {
        // H is a multiple of 4; the vector is 256-byte aligned
        constexpr uint32_t kPer = 16 / sizeof(V);
        for (uint32_t i = threadIdx.x * kPer; i < H; i += NT * kPer)
            *reinterpret_cast<uint4 *>(s_hot + i) = __ldcg(reinterpret_cast<const uint4 *>(xt + i));
    }
    P pass;
    if (!pass.begin(a, true)) return;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t lt = lanemask_lt();
    const uint32_t fshift = (lane & 3u) * 8u;  // the lane's byte in its mask word
    const uint32_t lower = (1u << fshift) - 1u;
    const uint32_t wsel = lane >> 2;            // the lane's mask word in the tile
    V *sums = s_sums + (threadIdx.x >> 5) * kSegTile;
    const uint64_t warp = (blockIdx.x * (uint64_t)NT + threadIdx.x) >> 5;
    const uint64_t nwarps = (gridDim.x * (uint64_t)NT) >> 5;
    const uint32_t L1 = a.l1hot;
    // tile t's indices (a lane that starts before the last arc stays inside
    // col's padding), the lane's mask word and the tile record
    auto load_tile = [&](uint64_t t, uint32_t (&c)[8], uint32_t &w, uint4 &m) {
        const uint64_t q = t * kSegTile + 8u * lane;
        if (t < a.seg_ntiles && q < a.arcs) {
            ld_stream_u8(a.col + q, policy_evict_first(), c);
        } else {
#pragma unroll
            for (int k = 0; k < 8; k++) c[k] = 0u;
        }
        if (t < a.seg_ntiles) {
            w = __ldg(&a.seg_mask[t * (kSegTile / 32) + wsel]);
            m = __ldg(&a.seg_meta[t]);
        } else {
            w = 0u;
            m = make_uint4(0u, 0u, 0u, 0u);
        }
    };
    // the 8 gathered values of tile t (zero past the last arc)
    auto gather_tile = [&](uint64_t t, const uint32_t (&c)[8], V (&v)[8]) {
        const uint64_t q = t * kSegTile + 8u * lane;
        const bool full = (t + 1) * kSegTile <= a.arcs;
        const uint64_t pol_g = policy_evict_last();
#pragma unroll
        for (int k = 0; k < 8; k++) {
            if (HOT) v[k] = c[k] < H ? s_hot[c[k]] : ld_gather_na(xt + c[k], pol_g);
            else v[k] = c[k] < L1 ? ld_gather(xt + c[k], pol_g) : ld_gather_na(xt + c[k], pol_g);
        }
        if (!full) {  // the last tile (warp-uniform branch)
#pragma unroll
            for (int k = 0; k < 8; k++)
                if (q + k >= a.arcs) v[k] = V(0);
        }
    };
    // with PIPE the next tile's indices, mask word and record are loaded while
    // the warp works on the current tile (issuing its gathers early as well
    // measured slower: the pass is bound by L1TEX and MIO throughput, not by
    // the latency that more loads in flight would hide)
    // one tile: its indices, mask word and record are in (cc, mw, meta);
    // with PIPE the next tile's go to (ccn, mwn, metan)
    auto work = [&](uint64_t t, const uint32_t (&cc)[8], uint32_t mw, const uint4 &meta, uint32_t (&ccn)[8],
                    uint32_t &mwn, uint4 &metan) {
        const uint64_t P0 = t * kSegTile;
        // a later tile of the warp's indices into L2 (full tiles only, so the
        // range stays inside col): the first one not yet being loaded
        constexpr uint32_t ahead = PIPE ? 2u : 1u;
        if (a.seg_prefetch && lane == 0u && P0 + (ahead * nwarps + 1u) * kSegTile <= a.arcs)
            prefetch_l2(a.col + P0 + ahead * nwarps * kSegTile, kSegTile * 4u);
        if (PIPE) load_tile(t + nwarps, ccn, mwn, metan);
        V v[8];
        gather_tile(t, cc, v);
        const uint32_t j0 = meta.x, cnt = meta.w & 0x7FFFFFFFu;
        const bool began = (meta.w >> 31) != 0u;
        // rank i's row (i < 32), skipping the one begun in an earlier tile
        const bool mine = lane < cnt && !(lane == 0u && began);
        uint32_t row = 0;
        typename P::Pre pre{};
        if (mine) {
            row = a.seg_dense ? j0 + lane : __ldg(&a.seg_nz[j0 + lane]);
            pre = pass.load(a, row);
        }
        // in-lane segmented sums
        const uint32_t f = (mw >> fshift) & 0xFFu;
        const uint32_t wpre = ((wsel < 4u ? meta.y : meta.z) >> (8u * (wsel & 3u))) & 0xFFu;
        const uint32_t r0 = wpre + __popc(mw & lower);
        uint32_t r = r0;
        double acc = 0.0, h = 0.0;
#pragma unroll
        for (int k = 0; k < 8; k++) {
            acc += (double)v[k];
            if ((f >> k) & 1u) {
                if (r == r0) h = acc;
                else sums[r] = (V)acc;
                r++;
                acc = 0.0;
            }
        }
        // across lanes
        double S = acc;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const double ov = __shfl_up_sync(0xffffffffu, S, o);
            if (lane >= (uint32_t)o) S += ov;
        }
        double X = __shfl_up_sync(0xffffffffu, S, 1);
        if (lane == 0u) X = 0.0;
        const uint32_t E = __ballot_sync(0xffffffffu, f != 0u);
        const uint32_t below = E & lt;
        const int jb = below ? 31 - __clz(below) : 0;
        const int jl = E ? 31 - __clz(E) : 0;
        const double Xb = __shfl_sync(0xffffffffu, X, jb);
        const double Xl = __shfl_sync(0xffffffffu, X, jl);
        if (f) {
            const double first = h + (X - Xb);
            sums[r0] = (V)first;
            if (r0 == 0u && began) a.seg_head[t] = first;  // closes a spanning row
        }
        if (lane == 31u) a.seg_tail[t] = S - Xl;
        __syncwarp();
        if (mine) pass.fin(a, row, pre, sums[lane]);
        for (uint32_t i = lane + 32u; i < cnt; i += 32u) {
            const uint32_t rw = a.seg_dense ? j0 + i : __ldg(&a.seg_nz[j0 + i]);
            pass.fin(a, rw, pass.load(a, rw), sums[i]);
        }
        __syncwarp();
    };
    if (PIPE) {
        // two tiles per trip with the buffers' roles swapped, so nothing is
        // copied between them
        uint32_t ca[8], cb[8], ma = 0u, mb = 0u;
        uint4 ea, eb;
        load_tile(warp, ca, ma, ea);
        for (uint64_t t = warp; t < a.seg_ntiles; t += 2 * nwarps) {
            work(t, ca, ma, ea, cb, mb, eb);
            if (t + nwarps >= a.seg_ntiles) break;
            work(t + nwarps, cb, mb, eb, ca, ma, ea);
        }
    } else {
        uint32_t cc[8], mw = 0u, cn[8], mn = 0u;
        uint4 meta, en;
        for (uint64_t t = warp; t < a.seg_ntiles; t += nwarps) {
            load_tile(t, cc, mw, meta);
            work(t, cc, mw, meta, cn, mn, en);
        }
    }
    pass.end(a, 0u, s_red, false);
}

// Rows that span tiles and rows without arcs; records after the tile
// kernel's.  A spanning row's total is the open tails of the tiles from its
// first to the one before its closing tile, plus that tile's head, in tile
// order in FP64: one thread per row for spans of up to kSegLongSpan tiles,
// one warp (lanes strided over the tiles, then a fixed tree) for longer ones.
template <class P>
__global__ void __launch_bounds__(kSegFixNT) seg_finish(const IterArgs a, unsigned rec0) {
    using V = typename P::V;
    __shared__ double s_red[96];
    if (P::stopped(a)) return;
    P pass;
    if (!pass.begin(a, false)) return;
    const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = tid; i < a.seg_nspan; i += nth) {
        const uint4 e = a.seg_span[i];
        double sum = 0.0;
#pragma unroll 4
        for (uint32_t t = e.y; t < e.z; t++) sum += __ldcg(&a.seg_tail[t]);
        sum += __ldcg(&a.seg_head[e.z]);
        pass.fin(a, e.x, pass.load(a, e.x), (V)sum);
    }
    const uint32_t lane = threadIdx.x & 31;
    for (uint64_t i = tid >> 5; i < a.seg_nlong; i += nth >> 5) {
        const uint4 e = a.seg_span_long[i];
        double sum = 0.0;
        for (uint32_t t = e.y + lane; t < e.z; t += 32) sum += __ldcg(&a.seg_tail[t]);
        sum = warp_sum(sum);
        if (lane == 0) pass.fin(a, e.x, pass.load(a, e.x), (V)(sum + __ldcg(&a.seg_head[e.z])));
    }
    // rows without arcs, four per thread and step (the list is 256-byte
    // aligned), their operand loads issued together; with dense ids they are
    // the range n - nempty .. n-1
    if (a.seg_dense) {
        // four rows per thread and step, nth apart, so that every load and
        // store of a warp covers consecutive rows
        const uint64_t e0 = a.n - a.seg_nempty;
        for (uint64_t i = tid; i < a.seg_nempty; i += 4 * nth) {
            typename P::Pre q[4];
#pragma unroll
            for (int k = 0; k < 4; k++)
                if (i + k * nth < a.seg_nempty) q[k] = pass.load(a, (uint32_t)(e0 + i + k * nth));
#pragma unroll
            for (int k = 0; k < 4; k++)
                if (i + k * nth < a.seg_nempty) pass.fin(a, (uint32_t)(e0 + i + k * nth), q[k], V(0));
        }
        pass.end(a, rec0, s_red, true);
        return;
    }
    const uint64_t ne4 = a.seg_nempty >> 2;
    const uint4 *e4 = reinterpret_cast<const uint4 *>(a.seg_empty);
    for (uint64_t i = tid; i < ne4; i += nth) {
        const uint4 q = __ldg(e4 + i);
        const typename P::Pre p0 = pass.load(a, q.x), p1 = pass.load(a, q.y), p2 = pass.load(a, q.z),
                              p3 = pass.load(a, q.w);
        pass.fin(a, q.x, p0, V(0));
        pass.fin(a, q.y, p1, V(0));
        pass.fin(a, q.z, p2, V(0));
        pass.fin(a, q.w, p3, V(0));
    }
    for (uint64_t i = (ne4 << 2) + tid; i < a.seg_nempty; i += nth) {
        const uint32_t v = a.seg_empty[i];
        pass.fin(a, v, pass.load(a, v), V(0));
    }
    pass.end(a, rec0, s_red, true);
}

// The tile kernel of pass P for a launch shape: hot prefix or not, threads
// per block (1024, 768 or 512), pipelined tile loads or not.
template <class P, bool HOT, int NT, bool PIPE>
static void seg8_go(const IterArgs &a, const LaunchCfg &c, cudaStream_t s) {
    seg8_kernel<P, HOT, NT, PIPE><<<c.seg_g1, NT, c.smem, s>>>(a);
}
using Seg8Go = void (*)(const IterArgs &, const LaunchCfg &, cudaStream_t);
template <class P>
static Seg8Go seg8_pick(bool hot, int nt, bool pipe, const void **entry) {
#define PRG_SEG8_PICK(H, N, Q)                                          \
    if (hot == H && nt == N && pipe == Q) {                             \
        if (entry) *entry = (const void *)seg8_kernel<P, H, N, Q>;      \
        return seg8_go<P, H, N, Q>;                                     \
    }
    PRG_SEG8_PICK(true, 1024, false)
    PRG_SEG8_PICK(true, 1024, true)
    PRG_SEG8_PICK(true, 768, false)
    PRG_SEG8_PICK(true, 768, true)
    PRG_SEG8_PICK(true, 512, false)
    PRG_SEG8_PICK(true, 512, true)
    PRG_SEG8_PICK(false, 1024, false)
    PRG_SEG8_PICK(false, 1024, true)
    PRG_SEG8_PICK(false, 768, false)
    PRG_SEG8_PICK(false, 768, true)
    PRG_SEG8_PICK(false, 512, false)
    PRG_SEG8_PICK(false, 512, true)
#undef PRG_SEG8_PICK
    throw CudaError(cudaErrorInvalidValue, "segmented pass: unsupported launch shape");
}

LaunchCfg seg_config(const DeviceGraph &g, uint32_t hot_entries, int variant, int mode) {
    int dev = 0, sms = 0;
    PRG_CUDA(cudaGetDevice(&dev));
    PRG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    const bool res = mode != MODE_KRY32;  // FP64 passes
    const size_t vb = res ? sizeof(double) : sizeof(float);
    LaunchCfg c;
    c.seg = res || variant == 2 ? 2 : 1;
    c.threads = c.seg == 2 ? (int)g.seg_threads : kSegNT;
    // pipelined loads pay in the FP32 matvec; the FP64 passes spill with them
    // and run about 2 % slower (R-MAT scale 24)
    c.seg_pipe = c.seg == 2 && !res && g.seg_pipe != 0;
    c.hot = std::min<uint32_t>(std::min<uint32_t>(hot_entries, res ? kSegHotMax64 : kSegHotMax), g.n) & ~3u;
    c.smem = ((size_t)(c.threads / 32) * kSegTile + c.hot) * vb;
    const void *k = nullptr;
    if (mode == MODE_KRES64) seg8_pick<Res64Pass>(c.hot != 0, c.threads, c.seg_pipe, &k);
    else if (mode == MODE_KRY64) seg8_pick<Kry64Pass>(c.hot != 0, c.threads, c.seg_pipe, &k);
    else if (mode == MODE_EIG64) seg8_pick<Eig64Pass>(c.hot != 0, c.threads, c.seg_pipe, &k);
    else if (res) seg8_pick<Plain64Pass>(c.hot != 0, c.threads, c.seg_pipe, &k);
    else if (c.seg == 2) seg8_pick<Kry32Pass>(c.hot != 0, c.threads, c.seg_pipe, &k);
    else k = c.hot ? (const void *)kry32_seg_kernel<true> : (const void *)kry32_seg_kernel<false>;
    PRG_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)c.smem));
    c.seg_g1 = (unsigned)sms;
    c.seg_g2 = (unsigned)sms * 4u;
    c.grid = c.seg_g1 + c.seg_g2;  // block records the consumers add
    c.hub_recs = 0;
    return c;
}

void launch_seg(int mode, const IterArgs &a, const LaunchCfg &c, cudaStream_t s) {
    if (mode == MODE_KRES64) {
        seg8_pick<Res64Pass>(c.hot != 0, c.threads, c.seg_pipe, nullptr)(a, c, s);
        seg_finish<Res64Pass><<<c.seg_g2, kSegFixNT, 0, s>>>(a, c.seg_g1);
    } else if (mode == MODE_EIG64) {
        seg8_pick<Eig64Pass>(c.hot != 0, c.threads, c.seg_pipe, nullptr)(a, c, s);
        seg_finish<Eig64Pass><<<c.seg_g2, kSegFixNT, 0, s>>>(a, c.seg_g1);
    } else if (mode == MODE_KRY64) {
        seg8_pick<Kry64Pass>(c.hot != 0, c.threads, c.seg_pipe, nullptr)(a, c, s);
        seg_finish<Kry64Pass><<<c.seg_g2, kSegFixNT, 0, s>>>(a, c.seg_g1);
    } else if (mode == MODE_PLAIN64 || mode == MODE_PPR64) {
        seg8_pick<Plain64Pass>(c.hot != 0, c.threads, c.seg_pipe, nullptr)(a, c, s);
        seg_finish<Plain64Pass><<<c.seg_g2, kSegFixNT, 0, s>>>(a, c.seg_g1);
    } else {
        if (c.seg == 2) seg8_pick<Kry32Pass>(c.hot != 0, c.threads, c.seg_pipe, nullptr)(a, c, s);
        else if (c.hot) kry32_seg_kernel<true><<<c.seg_g1, kSegNT, c.smem, s>>>(a);
        else kry32_seg_kernel<false><<<c.seg_g1, kSegNT, c.smem, s>>>(a);
        seg_finish<Kry32Pass><<<c.seg_g2, kSegFixNT, 0, s>>>(a, c.seg_g1);
    }
    PRG_CUDA(cudaGetLastError());
}

}  // namespace prg
