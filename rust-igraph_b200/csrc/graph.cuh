// graph.cuh — the device-resident graph behind a prg_graph handle and the
// build entry points (csr_build.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "prg_internal.cuh"

namespace prg {

struct DeviceGraph {
    uint32_t n = 0;
    uint64_t m = 0;      // edges as the caller passed them
    uint64_t arcs = 0;   // in-CSR entries (2m for undirected graphs)
    bool directed = true;
    bool weighted = false;
    int device = 0;

    uint32_t *row_ptr = nullptr;  // n+1
    uint32_t *col = nullptr;      // arcs + kColPad
    double *w64 = nullptr;        // arcs + kColPad (weighted)
    float *w32 = nullptr;         // arcs + kColPad (weighted)
    uint32_t *deg = nullptr;      // n
    double *dval = nullptr;       // n: out-degree / out-strength as double
    float *inv32 = nullptr;       // n: 1/dval in FP32, 0 when dangling

    uint32_t *perm = nullptr;     // internal id -> caller id (null when not relabelled)
    uint32_t *iperm = nullptr;    // caller id -> internal id
    uint4 *rb = nullptr;          // row-blocks {row_begin, row_end | kChunkFlag|hub, arc_begin, arc_end}
    uint32_t nrb = 0;
    Hub *hubs = nullptr;
    uint32_t nhub = 0;
    uint32_t n_dangling = 0;
    uint32_t max_in_degree = 0;

    // row-block tuning used to build `rb` (autotuned or defaults)
    uint32_t capw = kCapW;
    uint32_t shortmax = kShortMax;
    uint32_t split = kSplit;
    uint32_t blocks_per_sm = 0;  // persistent grid = SMs x this (0 = occupancy maximum)
    int relabel = 2;             // 0 keep caller ids, 1 degree-sorted ids, 2 decide from the degree skew
    // relabelled graphs: entries of the gathered vector's hot prefix each
    // block of an FP32 / FP64 pass keeps in shared memory (0 = off), and the
    // block size of those passes (256: several blocks per SM; 512 or 1024:
    // one block per SM with a larger prefix)
    uint32_t hot_cache = 0, hot_cache64 = 8192, hot_threads = 1024;
    // unweighted graphs: the FP32 Krylov matvec as the tile-segmented pass
    // (segspmv.cu), with a hot prefix of seg_hot entries on relabelled graphs
    uint32_t seg_kry32 = 2, seg_hot = 32768;
    // ... and the FP64 residual pass of the refined / Krylov solves, with a
    // hot prefix of seg_hot64 entries
    uint32_t seg_res64 = 1, seg_hot64 = 8192;
    // ... and the FP64 power step of the drop-ins and the certified loop, and
    // the FP64 Krylov matvec
    uint32_t seg_plain64 = 1;
    // ... and the adjacency product of the eigenvector and HITS iterations
    uint32_t seg_eig64 = 1;
    uint32_t seg_prefetch = 1;  // segmented passes: prefetch each warp's next index tile into L2
    // their tile kernel: threads of its one block per SM (1024, 768 or 512)
    // and, in the FP32 matvec, whether each warp loads its next tile while
    // working on the current one
    uint32_t seg_threads = 1024, seg_pipe = 1;
    // relabelled graphs: gathers of ids >= l1_hot32 (FP32 passes) / l1_hot64
    // (FP64 passes) bypass L1, keeping it for the hot prefix (0 = all allocate)
    uint32_t l1_hot32 = 16384, l1_hot64 = 2048;
    uint32_t batch_vec = 0;      // batched tile width / 32 chosen by the autotuner (0 = process default)

    float build_ms = 0.f;
};

// Builds the in-CSR, degrees and row-blocks from device edge arrays.
// d_w may be null (unweighted).  All work is on `s`; temporaries use the
// stream-ordered allocator.
void build_graph(DeviceGraph &g, const uint32_t *d_from, const uint32_t *d_to, const double *d_w,
                 cudaStream_t s);
// The same graph from HOST edge arrays, streamed: chunks of the edge list are
// copied on a side stream and sorted on arrival while the next chunk is in
// flight, then one scan and one scatter finish the CSR (identical to
// build_graph's).  Not for directed weighted graphs (their out-strengths
// need a second sort by source).  Returns false, with nothing built, when
// an endpoint is >= n (its maximum in *max_endpoint).
bool build_graph_host(DeviceGraph &g, const uint32_t *h_from, const uint32_t *h_to, const double *h_w, cudaStream_t s,
                      uint32_t *max_endpoint);
constexpr uint64_t kStreamChunks = 16;             // chunks of the streamed build
constexpr uint64_t kStreamChunkMin = 1ull << 22;   // smallest chunk (edges)
constexpr uint64_t kStreamMinEdges = 1ull << 23;   // smaller edge lists take the one-shot build

// Rebuilds only the row-blocks with new tuning (autotuner).
void build_row_blocks(DeviceGraph &g, uint32_t capw, uint32_t shortmax, uint32_t split, cudaStream_t s);
void free_graph(DeviceGraph &g);

// Process-wide defaults applied to graphs built afterwards (prg_set_tuning).
struct Tuning {
    uint32_t capw = kCapW, shortmax = kShortMax, split = kSplit, blocks_per_sm = 0;
    int relabel = 2;
    int unroll = 8;
    // FP64 passes on relabelled graphs: a 8 K-entry shared-memory hot prefix in
    // one 1024-thread block per SM (measured 7 % faster at R-MAT s24)
    uint32_t hot_cache = 0, hot_cache64 = 8192, hot_threads = 1024;
    uint32_t seg_kry32 = 2;      // unweighted graphs: tile-segmented FP32 Krylov matvec, 2 with 8 arcs per lane
                                 // (1 with 4-arc lane quads, 0 = row-block kernel)
    uint32_t seg_hot = 32768;    // its shared-memory hot prefix on relabelled graphs (entries)
    uint32_t seg_res64 = 1;      // unweighted graphs: tile-segmented FP64 residual pass (0 = row-block kernel)
    uint32_t seg_hot64 = 8192;   // its hot prefix (entries)
    uint32_t seg_plain64 = 1;    // unweighted graphs: tile-segmented FP64 power step and Krylov matvec
                                 // (0 = row-block kernels)
    uint32_t seg_eig64 = 1;      // unweighted graphs: tile-segmented eigenvector / HITS product
    uint32_t seg_prefetch = 1;   // segmented passes: L2 prefetch of each warp's next index tile
    uint32_t seg_threads = 1024;  // segmented passes: tile-kernel block size (1024, 768 or 512)
    uint32_t seg_pipe = 1;        // segmented FP32 matvec: load each warp's next tile ahead
    uint32_t l1_hot32 = 16384, l1_hot64 = 2048;
    double refine_switch = 5e-7;
    uint32_t batch_vec = 2;
    double krylov_rel = 1e-4;
    double krylov_floor = 0.7;         // refined / Krylov inner solves aim at this fraction of the final threshold
    uint32_t batch_barrier_extra = 0;  // test hook: batched grid barriers wait for arrivals that never come
    uint32_t batch_cheb = 0;           // batched solver on undirected graphs: 1 Chebyshev steps, 0 plain steps
};
Tuning &tuning();

// dst[i] = src[idx[i]] for i < n (FP64 vectors).
void gather_f64(double *dst, const double *src, const uint32_t *idx, uint32_t n, cudaStream_t s);

// Stable LSD radix sort of (key, value) u32 pairs on the low `key_bits` bits.
// On return *keys / *vals point at the sorted data (buffers may be swapped
// with *keys_alt / *vals_alt).
void radix_sort_pairs(uint32_t **keys, uint32_t **vals, uint32_t **keys_alt, uint32_t **vals_alt, uint64_t N,
                      int key_bits, cudaStream_t s);
// out[0..n] = exclusive prefix sums of in[0..n), out[n] = total (u32).
void exclusive_scan_u32(const uint32_t *in, uint32_t *out, uint64_t n, cudaStream_t s);

// Seeded device generators: kind 0 R-MAT (p0..p2 = a, b, c; n rounded up to
// a power of two), 1 Chung-Lu power law (p0 = alpha, p1 = offset), 2 block
// model (p0 = blocks, p1 = intra-block probability).
void generate_device(int kind, uint32_t n, uint64_t m, double p0, double p1, double p2, uint64_t seed,
                     uint32_t *d_from, uint32_t *d_to, cudaStream_t s);

// Device R-MAT generator (same stream layout as the oracle's or_rmat).
void rmat_generate(uint32_t scale, uint64_t m, double a, double b, double c, uint64_t seed, uint32_t *d_from,
                   uint32_t *d_to, cudaStream_t s);

}  // namespace prg
