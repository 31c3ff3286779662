// csr_build.cu — device construction of the in-arc CSR (the transpose the
// power iteration pulls over), out-degree / out-strength and the row-block
// work list of the SpMV.
//
// Semantics follow rust-igraph exactly:
//   * arcs: directed edge u->v gives in_adj[v] += u; an undirected edge
//     {u,v} gives in_adj[u] += v then in_adj[v] += u, a self-loop gives
//     in_adj[v] += v twice (pagerank.rs:76-101, pagerank_weighted.rs:103-124,
//     personalized_pagerank.rs:125-143);
//   * rows keep edge-id order: the arcs are produced in edge order and
//     sorted by destination with a STABLE radix sort, so row v lists its
//     in-neighbours in the same order as the reference's Vec<Vec<u32>>;
//   * out-degree = neighbors_iter(v).len(): out-edges for directed graphs,
//     all incident edge ends (self-loop twice) for undirected ones
//     (graph.rs:877-900, pagerank.rs:69-72);
//   * out-strength accumulates w per arc end (self-loop adds 2w,
//     pagerank_weighted.rs:81-101); a vertex is dangling iff its divisor is 0.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "graph.cuh"
#include "prims.cuh"

namespace prg {

static inline unsigned grid_for(uint64_t n, unsigned per_block, unsigned cap = 148u * 64u) {
    uint64_t g = (n + per_block - 1) / per_block;
    if (g < 1) g = 1;
    if (g > cap) g = cap;
    return (unsigned)g;
}

template <class T>
static T *dalloc(uint64_t count, cudaStream_t s) {
    void *p = nullptr;
    PRG_CUDA(cudaMallocAsync(&p, std::max<uint64_t>(count, 1) * sizeof(T), s));
    return (T *)p;
}
template <class T>
static void dfree(T *&p, cudaStream_t s) {
    if (p) cudaFreeAsync(p, s);
    p = nullptr;
}

// ------------------------------------------------------------------ scan

constexpr int kScanItems = 16;
constexpr int kScanTile = kThreads * kScanItems;

__global__ void __launch_bounds__(kThreads) scan_tile_sums(const uint32_t *in, uint64_t n, uint32_t *bsum) {
    __shared__ uint32_t sh[32];
    uint64_t base = (uint64_t)blockIdx.x * kScanTile;
    uint32_t acc = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        uint64_t idx = base + (uint64_t)i * kThreads + threadIdx.x;
        if (idx < n) acc += in[idx];
    }
    uint32_t t = block_sum<uint32_t>(acc, sh);
    if (threadIdx.x == 0) bsum[blockIdx.x] = t;
}

// Single-block exclusive scan of a (moderate) array in place; writes total.
__global__ void __launch_bounds__(1024) scan_single_block(uint32_t *a, uint64_t n, uint32_t *total) {
    __shared__ uint32_t sh[33];
    uint64_t per = (n + blockDim.x - 1) / blockDim.x;
    uint64_t lo = per * threadIdx.x, hi = lo + per < n ? lo + per : n;
    uint32_t s = 0;
    for (uint64_t i = lo; i < hi; i++) s += a[i];
    uint32_t tot;
    uint32_t pre = block_excl_scan(s, sh, &tot);
    for (uint64_t i = lo; i < hi; i++) {
        uint32_t v = a[i];
        a[i] = pre;
        pre += v;
    }
    if (threadIdx.x == 0 && total) *total = tot;
}

__global__ void __launch_bounds__(kThreads) scan_tiles_apply(const uint32_t *in, uint32_t *out, uint64_t n,
                                                             const uint32_t *boff) {
    __shared__ uint32_t sh[33];
    __shared__ uint32_t tile[kScanTile];
    uint64_t base = (uint64_t)blockIdx.x * kScanTile;
    // coalesced load into shared, then each thread scans a contiguous run
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        uint64_t idx = base + (uint64_t)i * kThreads + threadIdx.x;
        tile[i * kThreads + threadIdx.x] = idx < n ? in[idx] : 0u;
    }
    __syncthreads();
    uint32_t run[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        run[i] = tile[threadIdx.x * kScanItems + i];
        s += run[i];
    }
    uint32_t tot;
    uint32_t pre = block_excl_scan(s, sh, &tot) + boff[blockIdx.x];
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        tile[threadIdx.x * kScanItems + i] = pre;
        pre += run[i];
    }
    __syncthreads();
#pragma unroll
    for (int i = 0; i < kScanItems; i++) {
        uint64_t idx = base + (uint64_t)i * kThreads + threadIdx.x;
        if (idx < n) out[idx] = tile[i * kThreads + threadIdx.x];
    }
}

void exclusive_scan_u32(const uint32_t *in, uint32_t *out, uint64_t n, cudaStream_t s) {
    uint64_t nb = (n + kScanTile - 1) / kScanTile;
    if (nb == 0) nb = 1;
    uint32_t *bsum = dalloc<uint32_t>(nb + 1, s);
    scan_tile_sums<<<(unsigned)nb, kThreads, 0, s>>>(in, n, bsum);
    scan_single_block<<<1, 1024, 0, s>>>(bsum, nb, out + n);
    scan_tiles_apply<<<(unsigned)nb, kThreads, 0, s>>>(in, out, n, bsum);
    PRG_CUDA(cudaGetLastError());
    dfree(bsum, s);
}

// ------------------------------------------------------------------ radix sort

constexpr int kRsItems = 8;
constexpr int kRsTile = kThreads * kRsItems;  // 2048 keys
constexpr int kRsWarps = kThreads / 32;

__global__ void __launch_bounds__(kThreads) rs_upsweep(const uint32_t *keys, uint64_t N, uint64_t chunk, int shift,
                                                       uint32_t *counts, uint32_t G) {
    __shared__ uint32_t h[kRsWarps][256];
    for (int i = threadIdx.x; i < kRsWarps * 256; i += kThreads) (&h[0][0])[i] = 0;
    __syncthreads();
    uint64_t begin = (uint64_t)blockIdx.x * chunk;
    uint64_t end = begin + chunk < N ? begin + chunk : N;
    int w = threadIdx.x >> 5;
    for (uint64_t i = begin + threadIdx.x; i < end; i += kThreads) {
        uint32_t d = (keys[i] >> shift) & 255u;
        atomicAdd(&h[w][d], 1u);
    }
    __syncthreads();
    uint32_t t = threadIdx.x;
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kRsWarps; k++) s += h[k][t];
    counts[(uint64_t)t * G + blockIdx.x] = s;
}

// Stable scatter: each chunk is processed tile by tile; within a tile keys
// are ranked per warp with __match_any_sync in position order, then ordered
// by digit in shared memory and written out in digit runs (coalesced).
__global__ void __launch_bounds__(kThreads) rs_downsweep(const uint32_t *kin, const uint32_t *vin, uint32_t *kout,
                                                         uint32_t *vout, uint64_t N, uint64_t chunk, int shift,
                                                         const uint32_t *offsets, uint32_t G) {
    __shared__ uint32_t s_wh[kRsWarps][256];
    __shared__ uint32_t s_keys[kRsTile];
    __shared__ uint32_t s_vals[kRsTile];
    __shared__ uint32_t s_cnt[256];
    __shared__ uint32_t s_dstart[256];
    __shared__ uint32_t s_off[256];
    __shared__ uint32_t s_scan[33];

    const int tid = threadIdx.x, w = tid >> 5, lane = tid & 31;
    uint64_t begin = (uint64_t)blockIdx.x * chunk;
    uint64_t end = begin + chunk < N ? begin + chunk : N;
    s_off[tid] = offsets[(uint64_t)tid * G + blockIdx.x];
    const uint32_t ltmask = lanemask_lt();

    for (uint64_t tb = begin; tb < end; tb += kRsTile) {
        for (int i = tid; i < kRsWarps * 256; i += kThreads) (&s_wh[0][0])[i] = 0;
        __syncthreads();
        uint32_t key[kRsItems], val[kRsItems], dig[kRsItems], rank[kRsItems];
#pragma unroll
        for (int i = 0; i < kRsItems; i++) {
            uint64_t pos = tb + (uint64_t)w * (32 * kRsItems) + (uint64_t)i * 32 + lane;
            bool valid = pos < end;
            key[i] = valid ? kin[pos] : 0u;
            val[i] = valid ? vin[pos] : 0u;
            dig[i] = valid ? ((key[i] >> shift) & 255u) : 256u;
        }
#pragma unroll
        for (int i = 0; i < kRsItems; i++) {
            uint32_t d = dig[i];
            uint32_t peers = __match_any_sync(0xffffffffu, d);
            uint32_t before = d < 256u ? s_wh[w][d] : 0u;
            __syncwarp();
            if (d < 256u && (peers & ltmask) == 0u) s_wh[w][d] = before + __popc(peers);
            __syncwarp();
            rank[i] = before + __popc(peers & ltmask);
        }
        __syncthreads();
        {  // per digit: exclusive prefix across warps, tile count
            uint32_t run = 0;
#pragma unroll
            for (int k = 0; k < kRsWarps; k++) {
                uint32_t c = s_wh[k][tid];
                s_wh[k][tid] = run;
                run += c;
            }
            s_cnt[tid] = run;
        }
        __syncthreads();
        uint32_t tot;
        uint32_t ds = block_excl_scan(s_cnt[tid], s_scan, &tot);
        s_dstart[tid] = ds;
        __syncthreads();
#pragma unroll
        for (int i = 0; i < kRsItems; i++) {
            uint32_t d = dig[i];
            if (d < 256u) {
                uint32_t lp = s_dstart[d] + s_wh[w][d] + rank[i];
                s_keys[lp] = key[i];
                s_vals[lp] = val[i];
            }
        }
        __syncthreads();
        uint32_t nvalid = tot;
        for (uint32_t j = tid; j < nvalid; j += kThreads) {
            uint32_t k = s_keys[j];
            uint32_t d = (k >> shift) & 255u;
            uint64_t gpos = (uint64_t)s_off[d] + (j - s_dstart[d]);
            kout[gpos] = k;
            vout[gpos] = s_vals[j];
        }
        __syncthreads();
        s_off[tid] += s_cnt[tid];
        __syncthreads();
    }
}

// Stable passes over the 8-bit digits at shifts first_shift, +8, ... below
// key_bits; the result ends in *keys / *vals.
static void radix_passes(uint32_t **keys, uint32_t **vals, uint32_t **keys_alt, uint32_t **vals_alt, uint64_t N,
                         int first_shift, int key_bits, cudaStream_t s) {
    if (N <= 1 || key_bits <= first_shift) return;
    uint64_t tiles = (N + kRsTile - 1) / kRsTile;
    uint64_t G = std::min<uint64_t>(tiles, 148u * 8u);
    uint64_t chunk_tiles = (tiles + G - 1) / G;
    uint64_t chunk = chunk_tiles * kRsTile;
    G = (N + chunk - 1) / chunk;
    uint32_t *counts = dalloc<uint32_t>(256 * G + 1, s);  // + the scan's total
    for (int shift = first_shift; shift < key_bits; shift += 8) {
        rs_upsweep<<<(unsigned)G, kThreads, 0, s>>>(*keys, N, chunk, shift, counts, (uint32_t)G);
        exclusive_scan_u32(counts, counts, 256 * G, s);  // in place: each tile is loaded before it is written
        rs_downsweep<<<(unsigned)G, kThreads, 0, s>>>(*keys, *vals, *keys_alt, *vals_alt, N, chunk, shift, counts,
                                                     (uint32_t)G);
        PRG_CUDA(cudaGetLastError());
        std::swap(*keys, *keys_alt);
        std::swap(*vals, *vals_alt);
    }
    dfree(counts, s);
}

void radix_sort_pairs(uint32_t **keys, uint32_t **vals, uint32_t **keys_alt, uint32_t **vals_alt, uint64_t N,
                      int key_bits, cudaStream_t s) {
    radix_passes(keys, vals, keys_alt, vals_alt, N, 0, key_bits, s);
}

// One stable pass on the 8-bit digit at `shift`: (keys, vals) -> (keys_out,
// vals_out).
static void radix_pass_pairs(uint32_t *keys, uint32_t *vals, uint32_t *keys_out, uint32_t *vals_out, uint64_t N,
                             int shift, cudaStream_t s) {
    if (N <= 1) {
        if (N == 1) {
            PRG_CUDA(cudaMemcpyAsync(keys_out, keys, 4, cudaMemcpyDeviceToDevice, s));
            PRG_CUDA(cudaMemcpyAsync(vals_out, vals, 4, cudaMemcpyDeviceToDevice, s));
        }
        return;
    }
    radix_passes(&keys, &vals, &keys_out, &vals_out, N, shift, shift + 8, s);
}

// ------------------------------------------------------------------ CSR

Tuning &tuning() {
    static Tuning t;
    return t;
}

__global__ void gather_f64_kernel(double *dst, const double *src, const uint32_t *idx, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = src[idx[i]];
}

void gather_f64(double *dst, const double *src, const uint32_t *idx, uint32_t n, cudaStream_t s) {
    gather_f64_kernel<<<grid_for(n, kThreads), kThreads, 0, s>>>(dst, src, idx, n);
    PRG_CUDA(cudaGetLastError());
}

void preload_gather_f64() {
    cudaFuncAttributes fa;
    PRG_CUDA(cudaFuncGetAttributes(&fa, gather_f64_kernel));
}

// ---- degree-sorted relabelling.  On skewed (power-law) graphs the vertices
// that are gathered most often are those with the largest out-degree; giving
// them the smallest internal ids packs the hot part of the rank vector into a
// few cache lines (L1/L2 hits instead of one sector per arc).  The order is
// out-degree descending, then caller id (stable sort); on directed graphs the
// vertices without in-arcs come after all others.  That puts the rows with
// arcs at ids 0 .. k-1, so a pass that walks arcs finds the row of its i-th
// row end at id i without an index, and a pass over the rows without arcs
// reads one contiguous range.  On power-law graphs it costs the hot prefix
// nothing: a vertex without in-arcs rarely has a large out-degree (none with
// out-degree >= 16 among the 2.2 M of R-MAT scale 22).

__global__ void max_u32_kernel(const uint32_t *a, uint32_t n, uint32_t *out) {
    uint32_t mx = 0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) mx = max(mx, a[v]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, mx);
}

// noin: 1 for a vertex without in-arcs (null: out-degree alone); it is the
// key's most significant bit
__global__ void relabel_keys(const uint32_t *deg, const uint8_t *noin, uint32_t n, uint32_t maxdeg, int bits,
                             uint32_t *key, uint32_t *val) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        key[v] = noin ? (uint32_t)noin[v] << bits | (maxdeg - deg[v]) : maxdeg - deg[v];
        val[v] = v;
    }
}

// noin[v] = 0 for every arc head v (noin starts as all ones).  Flags only
// fall from 1 to 0, so a read that still sees 1 just leads to a repeated
// store; reading first keeps the stores to one per vertex instead of one per
// arc (the hot heads of a skewed graph are read from cache).
__global__ void mark_heads(const uint32_t *to, uint64_t m, uint32_t n, uint8_t *noin) {
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v = to[e];
        if (v < n && noin[v]) noin[v] = 0;
    }
}

__global__ void mark_empty_rows(const uint32_t *cnt, uint32_t n, uint8_t *noin) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        noin[v] = cnt[v] == 0u ? 1 : 0;
}

__global__ void relabel_finish(const uint32_t *perm, const uint32_t *deg_old, uint32_t n, uint32_t *iperm,
                               uint32_t *deg_new) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t o = perm[i];
        iperm[o] = i;
        deg_new[i] = deg_old[o];
    }
}

__global__ void relabel_edges(const uint32_t *from, const uint32_t *to, uint64_t m, const uint32_t *iperm,
                              uint32_t *rf, uint32_t *rt) {
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (uint64_t)gridDim.x * blockDim.x) {
        rf[e] = iperm[from[e]];
        rt[e] = iperm[to[e]];
    }
}

// Arc a of the in-CSR before sorting: key = destination row, value = source
// (unweighted) or arc id (weighted, to fetch the edge weight after the sort).
__global__ void make_arcs(const uint32_t *from, const uint32_t *to, uint64_t m, bool directed, bool carry_id,
                          uint32_t *key, uint32_t *val) {
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t u = from[e], v = to[e];
        if (directed) {
            key[e] = v;
            val[e] = carry_id ? (uint32_t)e : u;
        } else {
            // arc 2e: in_adj[u] += v ; arc 2e+1: in_adj[v] += u (self-loop: both v)
            key[2 * e] = u;
            val[2 * e] = carry_id ? (uint32_t)(2 * e) : v;
            key[2 * e + 1] = v;
            val[2 * e + 1] = carry_id ? (uint32_t)(2 * e + 1) : u;
        }
    }
}

// Out-degree by atomics.  Degree-heavy vertices usually have small ids (the
// generators, and any degree-sorted numbering, put them there); their counts
// are first gathered in a per-block shared-memory histogram so thousands of
// updates to one hub do not serialise on a single L2 address.
constexpr uint32_t kDegBins = 12288;
constexpr int kDegThreads = 1024;

__global__ void __launch_bounds__(kDegThreads) out_degree_kernel(const uint32_t *from, const uint32_t *to, uint64_t m,
                                                                 bool directed, uint32_t n, uint32_t *deg) {
    __shared__ uint32_t bins[kDegBins];
    for (uint32_t i = threadIdx.x; i < kDegBins; i += kDegThreads) bins[i] = 0u;
    __syncthreads();
    auto add = [&](uint32_t v) {
        if (v >= n) return;  // out-of-range ids are reported by the caller's range check
        if (v < kDegBins) atomicAdd_block(&bins[v], 1u);
        else atomicAdd(&deg[v], 1u);
    };
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (uint64_t)gridDim.x * blockDim.x) {
        add(from[e]);
        if (!directed) add(to[e]);
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < kDegBins && i < n; i += kDegThreads)
        if (bins[i]) atomicAdd(&deg[i], bins[i]);
}

// row_ptr of a CSR from its sorted row keys, through the rows' arc counts:
// the first arc i of a row leaves i, the row's last arc turns it into
// last + 1 - i, and rows without arcs keep 0; an exclusive scan of the counts
// gives row_ptr[0..n].  Work is one thread per arc however long the runs of
// rows without arcs are.
__global__ void row_first_arc(const uint32_t *key, uint64_t N, uint32_t *cnt) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (uint64_t)gridDim.x * blockDim.x)
        if (i == 0 || key[i - 1] != key[i]) cnt[key[i]] = (uint32_t)i;
}
__global__ void row_last_arc(const uint32_t *key, uint64_t N, uint32_t *cnt) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (uint64_t)gridDim.x * blockDim.x)
        if (i + 1 == N || key[i + 1] != key[i]) cnt[key[i]] = (uint32_t)(i + 1) - cnt[key[i]];
}
static void row_ptr_from_sorted(const uint32_t *key, uint64_t N, uint32_t n, uint32_t *row_ptr, cudaStream_t s) {
    PRG_CUDA(cudaMemsetAsync(row_ptr, 0, ((uint64_t)n + 1) * 4, s));
    if (N) {
        row_first_arc<<<grid_for(N, kThreads), kThreads, 0, s>>>(key, N, row_ptr);
        row_last_arc<<<grid_for(N, kThreads), kThreads, 0, s>>>(key, N, row_ptr);
    }
    exclusive_scan_u32(row_ptr, row_ptr, n, s);  // in place; writes row_ptr[n] = N
}

// After sorting arc ids: fetch source and weight of every arc.
__global__ void gather_arcs(const uint32_t *ids, const uint32_t *from, const uint32_t *to, const double *w,
                            uint64_t arcs, bool directed, uint32_t *col, double *w64, float *w32) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < arcs;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t a = ids[i];
        uint64_t e = directed ? a : (a >> 1);
        uint32_t src = directed ? from[e] : ((a & 1u) ? from[e] : to[e]);
        col[i] = src;
        double we = w[e];
        w64[i] = we;
        w32[i] = (float)we;
    }
}

// Segmented row sums of per-arc weights (one warp per row, fixed tree).
__global__ void row_weight_sums(const uint32_t *ptr, const double *wv, const uint32_t *perm, uint32_t nrows,
                                double *outsum) {
    uint32_t warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    uint32_t lane = threadIdx.x & 31;
    uint32_t nw = (gridDim.x * blockDim.x) >> 5;
    for (uint32_t r = warp; r < nrows; r += nw) {
        double acc = 0.0;
        for (uint32_t p = ptr[r] + lane; p < ptr[r + 1]; p += 32) acc += perm ? wv[perm[p]] : wv[p];
        acc = warp_sum(acc);
        if (lane == 0) outsum[r] = acc;
    }
}

__global__ void finish_degrees(uint32_t n, const uint32_t *deg, double *strength_io, bool weighted, double *dval,
                               float *inv32, uint32_t *n_dangling) {
    uint32_t cnt = 0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) {
        double d = weighted ? strength_io[v] : (double)deg[v];
        dval[v] = d;
        inv32[v] = d > 0.0 ? (float)(1.0 / d) : 0.0f;
        cnt += d == 0.0 ? 1u : 0u;
    }
    cnt = warp_sum(cnt);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(n_dangling, cnt);
}

__global__ void max_degree_kernel(const uint32_t *row_ptr, uint32_t n, uint32_t *out) {
    uint32_t mx = 0;
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x)
        mx = max(mx, row_ptr[v + 1] - row_ptr[v]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, mx);
}

// ------------------------------------------------------------------ row-blocks
//
// Row-blocks are the work units of one warp of the iteration kernel.  A row
// is "short" (deg <= shortmax), "long" (shortmax < deg <= split: one warp
// streams it) or a hub (deg > split: ceil(deg/split) chunk row-blocks whose
// partial sums are combined by the last chunk to finish).  A run of short
// rows forms a stream row-block; a new one starts at row r when r is a
// multiple of 32, when the previous row was not short, or when row r's first
// arc crosses a multiple of capw.  A stream block therefore holds <= 32 rows
// (32-row aligned, so its epilogue stores are coalesced) and
// < capw + shortmax <= kWarpBuf arcs; the kernel sums each of its rows with a
// power-of-two group of lanes sized to the row count.

__global__ void rb_count(const uint32_t *rp, uint32_t n, uint32_t capw, uint32_t shortmax, uint32_t split,
                         uint32_t *cnt, uint32_t *hubflag) {
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const uint32_t deg = rp[r + 1] - rp[r];
        uint32_t c, h = 0;
        if (deg > split) {
            c = (deg + split - 1) / split;
            h = 1;
        } else if (deg > shortmax) {
            c = 1;
        } else {
            bool start = (r % kRowCap == 0);
            if (!start) {
                const uint32_t pdeg = rp[r] - rp[r - 1];
                start = (pdeg > shortmax) || (rp[r] / capw != rp[r - 1] / capw);
            }
            c = start ? 1u : 0u;
        }
        cnt[r] = c;
        hubflag[r] = h;
    }
}

__global__ void rb_fill(const uint32_t *rp, uint32_t n, uint32_t shortmax, uint32_t split, const uint32_t *off,
                        const uint32_t *hoff, uint4 *rb, Hub *hubs) {
    for (uint32_t r = blockIdx.x * blockDim.x + threadIdx.x; r < n; r += gridDim.x * blockDim.x) {
        const uint32_t k = off[r], c = off[r + 1] - k;
        if (c == 0) continue;
        const uint32_t p0 = rp[r], p1 = rp[r + 1], deg = p1 - p0;
        if (deg > split) {
            const uint32_t h = hoff[r];
            hubs[h] = Hub{r, c, k, 0};
            for (uint32_t j = 0; j < c; j++) {
                const uint32_t lo = p0 + j * split, hi = min(p1, lo + split);
                rb[k + j] = make_uint4(r, kChunkFlag | h, lo, hi);
            }
        } else if (deg > shortmax) {
            rb[k] = make_uint4(r, r + 1, p0, p1);
        } else {
            rb[k] = make_uint4(r, 0, p0, 0);  // end filled by rb_fix
        }
    }
}

__global__ void rb_fix(const uint32_t *rp, uint4 *rb, uint32_t nrb, uint32_t n) {
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < nrb; k += gridDim.x * blockDim.x) {
        uint4 d = rb[k];
        if (d.y == 0u) {  // stream row-block: runs to the next row-block's first row
            d.y = (k + 1 < nrb) ? rb[k + 1].x : n;
            d.w = rp[d.y];
            rb[k] = d;
        }
    }
}

void build_row_blocks(DeviceGraph &g, uint32_t capw, uint32_t shortmax, uint32_t split, cudaStream_t s) {
    // a stream row-block holds < capw + shortmax arcs, which must fit the warp buffer
    shortmax = std::max<uint32_t>(1u, std::min<uint32_t>(shortmax, kWarpBuf / 2));
    capw = std::max<uint32_t>(32u, std::min<uint32_t>(capw, kWarpBuf - shortmax));
    split = std::max<uint32_t>(split, std::max<uint32_t>(shortmax, 256u));
    const uint32_t n = g.n;
    if (g.rb) cudaFreeAsync(g.rb, s);
    if (g.hubs) cudaFreeAsync(g.hubs, s);
    g.rb = nullptr;
    g.hubs = nullptr;
    uint32_t *cnt = dalloc<uint32_t>(n + 1, s), *off = dalloc<uint32_t>(n + 1, s);
    uint32_t *hf = dalloc<uint32_t>(n + 1, s), *hoff = dalloc<uint32_t>(n + 1, s);
    const unsigned gb = grid_for(n, kThreads);
    rb_count<<<gb, kThreads, 0, s>>>(g.row_ptr, n, capw, shortmax, split, cnt, hf);
    exclusive_scan_u32(cnt, off, n, s);
    exclusive_scan_u32(hf, hoff, n, s);
    uint32_t hv[2];
    PRG_CUDA(cudaMemcpyAsync(&hv[0], off + n, 4, cudaMemcpyDeviceToHost, s));
    PRG_CUDA(cudaMemcpyAsync(&hv[1], hoff + n, 4, cudaMemcpyDeviceToHost, s));
    PRG_CUDA(cudaStreamSynchronize(s));
    g.nrb = hv[0];
    g.nhub = hv[1];
    g.rb = dalloc<uint4>(g.nrb, s);
    g.hubs = dalloc<Hub>(g.nhub, s);
    rb_fill<<<gb, kThreads, 0, s>>>(g.row_ptr, n, shortmax, split, off, hoff, g.rb, g.hubs);
    rb_fix<<<grid_for(g.nrb, kThreads), kThreads, 0, s>>>(g.row_ptr, g.rb, g.nrb, n);
    PRG_CUDA(cudaGetLastError());
    dfree(cnt, s);
    dfree(off, s);
    dfree(hf, s);
    dfree(hoff, s);
    g.capw = capw;
    g.shortmax = shortmax;
    g.split = split;
}

static int bits_for(uint32_t maxkey) {
    int b = 0;
    while (b < 32 && (maxkey >> b) != 0) b++;
    return b;
}

// Divisors, dangling count, maximum in-degree and row-blocks of a graph whose
// row_ptr / col (/ weights) and deg are built; strength (weighted graphs, n
// entries, freed here) holds the out-strengths.
static void finish_graph(DeviceGraph &g, double *&strength, cudaStream_t s) {
    const uint32_t n = g.n;
    const unsigned gn = grid_for(n, kThreads);
    PRG_CUDA(cudaMallocAsync((void **)&g.dval, std::max<uint64_t>(n, 1) * 8, s));
    PRG_CUDA(cudaMallocAsync((void **)&g.inv32, std::max<uint64_t>(n, 1) * 4, s));
    uint32_t *d_nd = dalloc<uint32_t>(2, s);
    PRG_CUDA(cudaMemsetAsync(d_nd, 0, 8, s));
    finish_degrees<<<gn, kThreads, 0, s>>>(n, g.deg, strength, g.weighted, g.dval, g.inv32, d_nd);
    max_degree_kernel<<<gn, kThreads, 0, s>>>(g.row_ptr, n, d_nd + 1);
    PRG_CUDA(cudaGetLastError());
    uint32_t hnd[2];
    PRG_CUDA(cudaMemcpyAsync(hnd, d_nd, 8, cudaMemcpyDeviceToHost, s));
    dfree(strength, s);
    dfree(d_nd, s);
    PRG_CUDA(cudaStreamSynchronize(s));
    g.n_dangling = hnd[0];
    g.max_in_degree = hnd[1];
    build_row_blocks(g, g.capw, g.shortmax, g.split, s);
}

// Degree-sorted relabelling of the vertices when g.relabel asks for it (1) or
// the degree distribution is skewed (2: max degree >= 32 x mean, n >= 4096):
// g.perm (new -> old), g.iperm (old -> new) and g.deg in new ids.  Needs
// g.deg (out-degree) and g.arcs; on directed graphs either the arc heads
// (to, m) or the in-degrees in caller ids (in_cnt).  Returns whether it
// relabelled.
static bool relabel_vertices(DeviceGraph &g, cudaStream_t s, const uint32_t *to, uint64_t m,
                             const uint32_t *in_cnt = nullptr) {
    const uint32_t n = g.n;
    if (n < 2 || g.relabel == 0) return false;
    const unsigned gn = grid_for(n, kThreads);
    uint32_t *d_mx = dalloc<uint32_t>(1, s), maxdeg = 0;
    PRG_CUDA(cudaMemsetAsync(d_mx, 0, 4, s));
    max_u32_kernel<<<gn, kThreads, 0, s>>>(g.deg, n, d_mx);
    PRG_CUDA(cudaMemcpyAsync(&maxdeg, d_mx, 4, cudaMemcpyDeviceToHost, s));
    PRG_CUDA(cudaStreamSynchronize(s));
    dfree(d_mx, s);
    const double mean = (double)g.arcs / (double)n;
    const bool skewed = n >= 4096 && (double)maxdeg >= 32.0 * (mean > 1.0 ? mean : 1.0);
    if (g.relabel != 1 && !skewed) return false;
    uint32_t *pk = dalloc<uint32_t>(n, s), *pv = dalloc<uint32_t>(n, s);
    uint32_t *pk1 = dalloc<uint32_t>(n, s), *pv1 = dalloc<uint32_t>(n, s);
    // the no-in-arc bit: directed graphs whose key still fits 32 bits with it
    uint8_t *noin = nullptr;
    if (g.directed && bits_for(maxdeg) < 32 && (in_cnt || to)) {
        noin = dalloc<uint8_t>(n, s);
        if (in_cnt) {
            mark_empty_rows<<<gn, kThreads, 0, s>>>(in_cnt, n, noin);
        } else {
            PRG_CUDA(cudaMemsetAsync(noin, 1, n, s));
            if (m) mark_heads<<<grid_for(m, kThreads), kThreads, 0, s>>>(to, m, n, noin);
        }
    }
    relabel_keys<<<gn, kThreads, 0, s>>>(g.deg, noin, n, maxdeg, bits_for(maxdeg), pk, pv);
    radix_sort_pairs(&pk, &pv, &pk1, &pv1, n, bits_for(maxdeg) + (noin ? 1 : 0), s);
    dfree(noin, s);
    PRG_CUDA(cudaMallocAsync((void **)&g.perm, (uint64_t)n * 4, s));
    PRG_CUDA(cudaMallocAsync((void **)&g.iperm, (uint64_t)n * 4, s));
    PRG_CUDA(cudaMemcpyAsync(g.perm, pv, (uint64_t)n * 4, cudaMemcpyDeviceToDevice, s));
    uint32_t *deg_new = dalloc<uint32_t>(n, s);
    relabel_finish<<<gn, kThreads, 0, s>>>(g.perm, g.deg, n, g.iperm, deg_new);
    cudaFreeAsync(g.deg, s);
    g.deg = deg_new;
    dfree(pk, s);
    dfree(pv, s);
    dfree(pk1, s);
    dfree(pv1, s);
    return true;
}

void build_graph(DeviceGraph &g, const uint32_t *d_from, const uint32_t *d_to, const double *d_w, cudaStream_t s) {
    cudaEvent_t e0, e1;
    PRG_CUDA(cudaEventCreate(&e0));
    PRG_CUDA(cudaEventCreate(&e1));
    PRG_CUDA(cudaEventRecord(e0, s));
    const uint32_t n = g.n;
    const uint64_t m = g.m;
    const bool directed = g.directed, weighted = d_w != nullptr;
    g.weighted = weighted;
    const uint64_t arcs = directed ? m : 2 * m;
    g.arcs = arcs;
    unsigned ge = grid_for(m, kThreads), ga = grid_for(arcs, kThreads), gn = grid_for(n, kThreads);

    // out-degree (unweighted divisor; also kept for weighted graphs)
    PRG_CUDA(cudaMallocAsync((void **)&g.deg, std::max<uint64_t>(n, 1) * 4, s));
    PRG_CUDA(cudaMemsetAsync(g.deg, 0, std::max<uint64_t>(n, 1) * 4, s));
    if (m) out_degree_kernel<<<148 * 2, kDegThreads, 0, s>>>(d_from, d_to, m, directed, n, g.deg);

    // optional degree-sorted relabelling (internal ids); the edge list the CSR
    // is built from becomes (ef, et)
    const uint32_t *ef = d_from, *et = d_to;
    uint32_t *rf = nullptr, *rt = nullptr;
    if (relabel_vertices(g, s, d_to, m)) {
        rf = dalloc<uint32_t>(m, s);
        rt = dalloc<uint32_t>(m, s);
        if (m) relabel_edges<<<ge, kThreads, 0, s>>>(d_from, d_to, m, g.iperm, rf, rt);
        ef = rf;
        et = rt;
    }

    // arcs in edge order, then stable sort by destination
    uint32_t *k0 = dalloc<uint32_t>(arcs, s), *v0 = dalloc<uint32_t>(arcs, s);
    uint32_t *k1 = dalloc<uint32_t>(arcs, s), *v1 = dalloc<uint32_t>(arcs, s);
    if (m) make_arcs<<<ge, kThreads, 0, s>>>(ef, et, m, directed, weighted, k0, v0);

    radix_sort_pairs(&k0, &v0, &k1, &v1, arcs, bits_for(n ? n - 1 : 0), s);

    // row_ptr from the boundaries of the sorted destinations
    PRG_CUDA(cudaMallocAsync((void **)&g.row_ptr, (uint64_t)(n + 1) * 4, s));
    row_ptr_from_sorted(k0, arcs, n, g.row_ptr, s);
    PRG_CUDA(cudaGetLastError());

    const uint64_t padded = arcs + kColPad;
    PRG_CUDA(cudaMallocAsync((void **)&g.col, padded * 4, s));
    PRG_CUDA(cudaMemsetAsync(g.col, 0, padded * 4, s));
    double *strength = nullptr;
    if (!weighted) {
        if (arcs) PRG_CUDA(cudaMemcpyAsync(g.col, v0, arcs * 4, cudaMemcpyDeviceToDevice, s));
    } else {
        PRG_CUDA(cudaMallocAsync((void **)&g.w64, padded * 8, s));
        PRG_CUDA(cudaMallocAsync((void **)&g.w32, padded * 4, s));
        PRG_CUDA(cudaMemsetAsync(g.w64, 0, padded * 8, s));
        PRG_CUDA(cudaMemsetAsync(g.w32, 0, padded * 4, s));
        if (arcs) gather_arcs<<<ga, kThreads, 0, s>>>(v0, ef, et, d_w, arcs, directed, g.col, g.w64, g.w32);
        strength = dalloc<double>(n, s);
        if (!directed) {
            // undirected: arcs out of u are exactly the arcs into u (same weights)
            row_weight_sums<<<grid_for((uint64_t)n * 32, kThreads), kThreads, 0, s>>>(g.row_ptr, g.w64, nullptr, n,
                                                                                   strength);
        } else {
            // directed: group edge ids by source with a second stable sort
            uint32_t *sk = dalloc<uint32_t>(m, s), *sv = dalloc<uint32_t>(m, s);
            uint32_t *sk1 = dalloc<uint32_t>(m, s), *sv1 = dalloc<uint32_t>(m, s);
            uint32_t *optr = dalloc<uint32_t>(n + 1, s);
            if (m) {
                PRG_CUDA(cudaMemcpyAsync(sk, ef, m * 4, cudaMemcpyDeviceToDevice, s));
                make_arcs<<<ge, kThreads, 0, s>>>(ef, et, m, true, true, sk1, sv);  // sv = edge ids
            }
            radix_sort_pairs(&sk, &sv, &sk1, &sv1, m, bits_for(n ? n - 1 : 0), s);
            row_ptr_from_sorted(sk, m, n, optr, s);
            row_weight_sums<<<grid_for((uint64_t)n * 32, kThreads), kThreads, 0, s>>>(optr, d_w, sv, n, strength);
            dfree(sk, s);
            dfree(sv, s);
            dfree(sk1, s);
            dfree(sv1, s);
            dfree(optr, s);
        }
    }
    dfree(k0, s);
    dfree(v0, s);
    dfree(k1, s);
    dfree(v1, s);
    dfree(rf, s);
    dfree(rt, s);

    finish_graph(g, strength, s);
    PRG_CUDA(cudaEventRecord(e1, s));
    PRG_CUDA(cudaEventSynchronize(e1));
    PRG_CUDA(cudaEventElapsedTime(&g.build_ms, e0, e1));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
}

// ------------------------------------------------------------------ streamed build from host edges
//
// The edge list arrives in chunks (host -> device copies on a side stream);
// each chunk is processed while the next one is in flight.  An arc's final
// CSR position is
//     row_ptr[dst] + (arcs into dst in earlier chunks) + (rank among the
//                                                          chunk's arcs into dst)
// and only row_ptr needs the whole list.  So every chunk is stably sorted by
// destination on arrival, its ranks are added to the running per-destination
// counts (off[arc], cnt[dst]), and after the last chunk one scan of the
// counts and one scatter place every arc.  Within a row the arcs keep their
// arc order, exactly as the sort of the whole list in build_graph leaves
// them, so both builds produce the same CSR.

// Start of each destination's run in the sorted chunk: base = cnt - i.
__global__ void chunk_ranks_begin(const uint32_t *keys, uint64_t N, uint32_t n, const uint32_t *cnt, uint32_t *base) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t k = keys[i];
        if (k < n && (i == 0 || keys[i - 1] != k)) base[k] = cnt[k] - (uint32_t)i;
    }
}

// off[arc] = arcs into its destination before it; the run's last arc
// advances cnt.  (u32 arithmetic: base + i is the true count.)
__global__ void chunk_ranks_end(const uint32_t *keys, const uint32_t *vals, uint64_t N, uint32_t n,
                                const uint32_t *base, uint32_t *cnt, uint32_t *off) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t k = keys[i];
        if (k >= n) continue;
        const uint32_t b = base[k];
        off[vals[i]] = b + (uint32_t)i;
        if (i + 1 == N || keys[i + 1] != k) cnt[k] = b + (uint32_t)i + 1u;
    }
}

__global__ void gather_u32_kernel(uint32_t *dst, const uint32_t *src, const uint32_t *idx, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) dst[i] = src[idx[i]];
}

// The arcs' final positions, row_ptr[dst] + off[arc], are a permutation of
// [0, arcs).  Writing each arc straight to its position would be one random
// 4-byte HBM write per arc.  Instead: (1) arc_positions writes (position,
// value) pairs in arc order; (2) one stable radix pass on the position's top
// 8 bits groups them into 256 windows of consecutive positions; (3)
// place_arcs writes each window while its slice of col sits in L2.
// value = the relabelled source (unweighted) or the arc id (weighted: the
// source and the edge weight are fetched when placing).
__global__ void arc_positions(const uint32_t *from, const uint32_t *to, uint64_t arcs, bool directed, bool weighted,
                              const uint32_t *iperm, const uint32_t *row_ptr, const uint32_t *off, uint32_t *pos,
                              uint32_t *val) {
    for (uint64_t a = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; a < arcs;
         a += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t e = directed ? a : (a >> 1);
        uint32_t dst = to[e], src = from[e];
        if (!directed && (a & 1u) == 0u) {
            dst = from[e];
            src = to[e];
        }
        if (iperm) {
            dst = iperm[dst];
            src = iperm[src];
        }
        pos[a] = row_ptr[dst] + off[a];
        val[a] = weighted ? (uint32_t)a : src;
    }
}

__global__ void place_arcs(const uint32_t *pos, const uint32_t *val, uint64_t arcs, bool directed,
                           const uint32_t *from, const uint32_t *to, const double *w, const uint32_t *iperm,
                           uint32_t *col, double *w64, float *w32) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < arcs; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t p = pos[i];
        if (p >= arcs) continue;  // never for a consistent build
        if (!w) {
            col[p] = val[i];
            continue;
        }
        const uint32_t a = val[i];
        const uint64_t e = directed ? a : (a >> 1);
        uint32_t src = (directed || (a & 1u)) ? from[e] : to[e];
        if (iperm) src = iperm[src];
        col[p] = src;
        const double we = w[e];
        w64[p] = we;
        w32[p] = (float)we;
    }
}

bool build_graph_host(DeviceGraph &g, const uint32_t *h_from, const uint32_t *h_to, const double *h_w, cudaStream_t s,
                      uint32_t *max_endpoint) {
    cudaEvent_t e0, e1;
    PRG_CUDA(cudaEventCreate(&e0));
    PRG_CUDA(cudaEventCreate(&e1));
    PRG_CUDA(cudaEventRecord(e0, s));
    const uint32_t n = g.n;
    const uint64_t m = g.m;
    const bool directed = g.directed, weighted = h_w != nullptr;
    g.weighted = weighted;
    const uint64_t arcs = directed ? m : 2 * m;
    g.arcs = arcs;
    const uint64_t chunk = std::max<uint64_t>(kStreamChunkMin, (m + kStreamChunks - 1) / kStreamChunks);
    const uint64_t nchunks = (m + chunk - 1) / chunk;
    const uint64_t chunk_arcs = directed ? chunk : 2 * chunk;
    const int key_bits = bits_for(n ? n - 1 : 0);

    uint32_t *d_from = dalloc<uint32_t>(m, s), *d_to = dalloc<uint32_t>(m, s);
    double *d_w = weighted ? dalloc<double>(m, s) : nullptr;
    PRG_CUDA(cudaMallocAsync((void **)&g.deg, std::max<uint64_t>(n, 1) * 4, s));
    PRG_CUDA(cudaMemsetAsync(g.deg, 0, std::max<uint64_t>(n, 1) * 4, s));
    uint32_t *cnt = dalloc<uint32_t>(n, s), *base = dalloc<uint32_t>(n, s), *off = dalloc<uint32_t>(arcs, s);
    PRG_CUDA(cudaMemsetAsync(cnt, 0, std::max<uint64_t>(n, 1) * 4, s));
    uint32_t *d_mx = dalloc<uint32_t>(1, s);
    PRG_CUDA(cudaMemsetAsync(d_mx, 0, 4, s));
    uint32_t *ka = dalloc<uint32_t>(chunk_arcs, s), *va = dalloc<uint32_t>(chunk_arcs, s);
    uint32_t *kb = dalloc<uint32_t>(chunk_arcs, s), *vb = dalloc<uint32_t>(chunk_arcs, s);

    cudaStream_t cs;
    PRG_CUDA(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    std::vector<cudaEvent_t> ev(nchunks + 1);
    for (cudaEvent_t &e : ev) PRG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    // the copy stream starts once the allocations above are usable
    PRG_CUDA(cudaEventRecord(ev[nchunks], s));
    PRG_CUDA(cudaStreamWaitEvent(cs, ev[nchunks], 0));
    for (uint64_t c = 0; c < nchunks; c++) {
        const uint64_t b = c * chunk, len = std::min(chunk, m - b);
        const uint64_t a0 = directed ? b : 2 * b, la = directed ? len : 2 * len;
        PRG_CUDA(cudaMemcpyAsync(d_from + b, h_from + b, len * 4, cudaMemcpyHostToDevice, cs));
        PRG_CUDA(cudaMemcpyAsync(d_to + b, h_to + b, len * 4, cudaMemcpyHostToDevice, cs));
        if (weighted) PRG_CUDA(cudaMemcpyAsync(d_w + b, h_w + b, len * 8, cudaMemcpyHostToDevice, cs));
        PRG_CUDA(cudaEventRecord(ev[c], cs));
        PRG_CUDA(cudaStreamWaitEvent(s, ev[c], 0));
        const unsigned gl = grid_for(len, kThreads), gla = grid_for(la, kThreads);
        max_u32_kernel<<<gl, kThreads, 0, s>>>(d_from + b, (uint32_t)len, d_mx);
        max_u32_kernel<<<gl, kThreads, 0, s>>>(d_to + b, (uint32_t)len, d_mx);
        out_degree_kernel<<<148 * 2, kDegThreads, 0, s>>>(d_from + b, d_to + b, len, directed, n, g.deg);
        make_arcs<<<gl, kThreads, 0, s>>>(d_from + b, d_to + b, len, directed, true, ka, va);
        uint32_t *k0 = ka, *v0 = va, *k1 = kb, *v1 = vb;
        radix_sort_pairs(&k0, &v0, &k1, &v1, la, key_bits, s);
        chunk_ranks_begin<<<gla, kThreads, 0, s>>>(k0, la, n, cnt, base);
        chunk_ranks_end<<<gla, kThreads, 0, s>>>(k0, v0, la, n, base, cnt, off + a0);
        PRG_CUDA(cudaGetLastError());
    }
    const bool trace = std::getenv("PRG_TRACE") != nullptr;
    cudaEvent_t t_copy = nullptr, t_loop = nullptr, t_tail[4] = {};
    if (trace) {
        PRG_CUDA(cudaEventCreate(&t_copy));
        PRG_CUDA(cudaEventCreate(&t_loop));
        for (cudaEvent_t &e : t_tail) PRG_CUDA(cudaEventCreate(&e));
        PRG_CUDA(cudaEventRecord(t_copy, cs));
        PRG_CUDA(cudaEventRecord(t_loop, s));
    }
    uint32_t mx = 0;
    PRG_CUDA(cudaMemcpyAsync(&mx, d_mx, 4, cudaMemcpyDeviceToHost, s));
    PRG_CUDA(cudaStreamSynchronize(s));
    PRG_CUDA(cudaStreamSynchronize(cs));
    for (cudaEvent_t &e : ev) cudaEventDestroy(e);
    cudaStreamDestroy(cs);
    dfree(ka, s);
    dfree(va, s);
    dfree(kb, s);
    dfree(vb, s);
    dfree(d_mx, s);
    *max_endpoint = mx;
    if (m > 0 && mx >= n) {
        dfree(d_from, s);
        dfree(d_to, s);
        dfree(d_w, s);
        dfree(cnt, s);
        dfree(base, s);
        dfree(off, s);
        if (trace) {
            cudaEventDestroy(t_copy);
            cudaEventDestroy(t_loop);
            for (cudaEvent_t &e : t_tail) cudaEventDestroy(e);
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        return false;
    }

    const unsigned gn = grid_for(n, kThreads), ga = grid_for(arcs, kThreads);
    const bool relabelled = relabel_vertices(g, s, nullptr, 0, cnt);
    if (trace) PRG_CUDA(cudaEventRecord(t_tail[0], s));
    uint32_t *rows = cnt;
    if (relabelled) {
        gather_u32_kernel<<<gn, kThreads, 0, s>>>(base, cnt, g.perm, n);  // base is free now
        rows = base;
    }
    PRG_CUDA(cudaMallocAsync((void **)&g.row_ptr, (uint64_t)(n + 1) * 4, s));
    exclusive_scan_u32(rows, g.row_ptr, n, s);
    const uint64_t padded = arcs + kColPad;
    PRG_CUDA(cudaMallocAsync((void **)&g.col, padded * 4, s));
    PRG_CUDA(cudaMemsetAsync(g.col, 0, padded * 4, s));
    if (weighted) {
        PRG_CUDA(cudaMallocAsync((void **)&g.w64, padded * 8, s));
        PRG_CUDA(cudaMallocAsync((void **)&g.w32, padded * 4, s));
        PRG_CUDA(cudaMemsetAsync(g.w64, 0, padded * 8, s));
        PRG_CUDA(cudaMemsetAsync(g.w32, 0, padded * 4, s));
    }
    if (trace) PRG_CUDA(cudaEventRecord(t_tail[1], s));
    if (arcs) {
        const uint32_t *ip = relabelled ? g.iperm : nullptr;
        uint32_t *pk = dalloc<uint32_t>(arcs, s), *pv = dalloc<uint32_t>(arcs, s);
        uint32_t *pk1 = dalloc<uint32_t>(arcs, s), *pv1 = dalloc<uint32_t>(arcs, s);
        arc_positions<<<ga, kThreads, 0, s>>>(d_from, d_to, arcs, directed, weighted, ip, g.row_ptr, off, pk, pv);
        const int pbits = bits_for((uint32_t)(arcs - 1));
        radix_pass_pairs(pk, pv, pk1, pv1, arcs, std::max(0, pbits - 8), s);
        place_arcs<<<ga, kThreads, 0, s>>>(pk1, pv1, arcs, directed, d_from, d_to, d_w, ip, g.col, g.w64, g.w32);
        dfree(pk, s);
        dfree(pv, s);
        dfree(pk1, s);
        dfree(pv1, s);
    }
    PRG_CUDA(cudaGetLastError());
    if (trace) PRG_CUDA(cudaEventRecord(t_tail[2], s));
    double *strength = nullptr;
    if (weighted) {
        // undirected only: arcs out of u are exactly the arcs into u (same weights)
        strength = dalloc<double>(n, s);
        row_weight_sums<<<grid_for((uint64_t)n * 32, kThreads), kThreads, 0, s>>>(g.row_ptr, g.w64, nullptr, n,
                                                                               strength);
    }
    dfree(d_from, s);
    dfree(d_to, s);
    dfree(d_w, s);
    dfree(cnt, s);
    dfree(base, s);
    dfree(off, s);
    finish_graph(g, strength, s);
    PRG_CUDA(cudaEventRecord(e1, s));
    PRG_CUDA(cudaEventSynchronize(e1));
    PRG_CUDA(cudaEventElapsedTime(&g.build_ms, e0, e1));
    if (trace) {
        float c = 0, l = 0, r = 0, sc = 0, sca = 0;
        cudaEventElapsedTime(&c, e0, t_copy);
        cudaEventElapsedTime(&l, e0, t_loop);
        cudaEventElapsedTime(&r, t_loop, t_tail[0]);
        cudaEventElapsedTime(&sc, t_tail[0], t_tail[1]);
        cudaEventElapsedTime(&sca, t_tail[1], t_tail[2]);
        std::fprintf(stderr,
                     "[prg] streamed build: %llu chunks, copies done %.2f ms, chunk work done %.2f ms, relabel %.2f, "
                     "scan+alloc %.2f, scatter %.2f, finish %.2f, total %.2f ms\n",
                     (unsigned long long)nchunks, c, l, r, sc, sca, g.build_ms - l - r - sc - sca, g.build_ms);
        cudaEventDestroy(t_copy);
        cudaEventDestroy(t_loop);
        for (cudaEvent_t &e : t_tail) cudaEventDestroy(e);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return true;
}

void free_graph(DeviceGraph &g) {
    cudaFree(g.row_ptr);
    cudaFree(g.col);
    cudaFree(g.w64);
    cudaFree(g.w32);
    cudaFree(g.deg);
    cudaFree(g.dval);
    cudaFree(g.inv32);
    cudaFree(g.rb);
    cudaFree(g.hubs);
    cudaFree(g.perm);
    cudaFree(g.iperm);
    g = DeviceGraph{};
}

// ------------------------------------------------------------------ R-MAT

// Counter-based R-MAT: edge e draws `scale` uniforms from its own SplitMix64
// stream seeded with seed ^ (e * 0xD1B54A32D192ED03).  Bit-identical to the
// CPU generator used by the tests (same integer mixing, same double compare).
__global__ void rmat_kernel(uint32_t scale, uint64_t m, double t1, double t2, double t3, uint64_t seed,
                            uint32_t *from, uint32_t *to) {
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t st = seed ^ (e * 0xD1B54A32D192ED03ULL);
        uint32_t u = 0, v = 0;
        for (uint32_t l = 0; l < scale; l++) {
            st += 0x9E3779B97F4A7C15ULL;
            uint64_t z = st;
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
            z ^= z >> 31;
            double x = (double)(z >> 11) * (1.0 / 9007199254740992.0);
            uint32_t rb, cb;
            if (x < t1) { rb = 0; cb = 0; }
            else if (x < t2) { rb = 0; cb = 1; }
            else if (x < t3) { rb = 1; cb = 0; }
            else { rb = 1; cb = 1; }
            u = (u << 1) | rb;
            v = (v << 1) | cb;
        }
        from[e] = u;
        to[e] = v;
    }
}

void rmat_generate(uint32_t scale, uint64_t m, double a, double b, double c, uint64_t seed, uint32_t *d_from,
                   uint32_t *d_to, cudaStream_t s) {
    double t1 = a, t2 = a + b, t3 = a + b + c;
    rmat_kernel<<<grid_for(m, kThreads, 148u * 32u), kThreads, 0, s>>>(scale, m, t1, t2, t3, seed, d_from, d_to);
    PRG_CUDA(cudaGetLastError());
}

}  // namespace prg

namespace prg {

// ---- further seeded generators (training graphs for the warm start) ------
// Counter-based like the R-MAT generator: edge e draws from its own
// SplitMix64 stream seeded with seed ^ (e * 0xD1B54A32D192ED03).

__device__ __forceinline__ double sm_unit(uint64_t &st) {
    st += 0x9E3779B97F4A7C15ULL;
    uint64_t z = st;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
}

// Chung-Lu power law: both endpoints drawn with probability proportional to
// (i + i0)^(-alpha) by inverting the continuous cumulative weight; alpha =
// 1/(gamma - 1) (gamma = 3 gives the degree law of preferential attachment).
__global__ void chung_lu_kernel(uint32_t n, uint64_t m, double alpha, double i0, uint64_t seed, uint32_t *from,
                                uint32_t *to) {
    const double b = 1.0 - alpha;
    const double lo = pow(i0, b), hi = pow((double)n + i0, b);
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t st = seed ^ (e * 0xD1B54A32D192ED03ULL);
        uint32_t ends[2];
        for (int k = 0; k < 2; k++) {
            const double u = sm_unit(st);
            double x = pow(lo + u * (hi - lo), 1.0 / b) - i0;
            uint32_t v = x < 0.0 ? 0u : (uint32_t)x;
            ends[k] = v >= n ? n - 1 : v;
        }
        from[e] = ends[0];
        to[e] = ends[1];
    }
}

// Block model with a fixed edge count: block of the edge uniform among
// `blocks` equal blocks; with probability p_in both ends in that block,
// otherwise the target in another uniformly chosen block.
__global__ void sbm_edges_kernel(uint32_t n, uint64_t m, uint32_t blocks, double p_in, uint64_t seed, uint32_t *from,
                                 uint32_t *to) {
    const uint32_t bs = n / blocks;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < m; e += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t st = seed ^ (e * 0xD1B54A32D192ED03ULL);
        const uint32_t b0 = min((uint32_t)(sm_unit(st) * blocks), blocks - 1);
        uint32_t b1 = b0;
        if (sm_unit(st) >= p_in && blocks > 1) {
            b1 = min((uint32_t)(sm_unit(st) * (blocks - 1)), blocks - 2);
            if (b1 >= b0) b1++;
        }
        const uint32_t u = b0 * bs + min((uint32_t)(sm_unit(st) * bs), bs - 1);
        const uint32_t v = b1 * bs + min((uint32_t)(sm_unit(st) * bs), bs - 1);
        from[e] = u;
        to[e] = v;
    }
}

void generate_device(int kind, uint32_t n, uint64_t m, double p0, double p1, double p2, uint64_t seed,
                     uint32_t *d_from, uint32_t *d_to, cudaStream_t s) {
    const unsigned grid = grid_for(m, kThreads, 148u * 32u);
    if (kind == 0) {
        uint32_t scale = 0;
        while ((1ull << scale) < n) scale++;
        rmat_generate(scale, m, p0, p1, p2, seed, d_from, d_to, s);
    } else if (kind == 1) {
        chung_lu_kernel<<<grid, kThreads, 0, s>>>(n, m, p0, p1 > 0 ? p1 : 1.0, seed, d_from, d_to);
    } else {
        sbm_edges_kernel<<<grid, kThreads, 0, s>>>(n, m, (uint32_t)p0, p1, seed, d_from, d_to);
    }
    PRG_CUDA(cudaGetLastError());
}

}  // namespace prg
