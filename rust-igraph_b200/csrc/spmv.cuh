// spmv.cuh — launch interface of the fused PageRank iteration kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "graph.cuh"

namespace prg {

// Iteration flavours.  All share one kernel body (spmv.cu); they differ in
// the gather precision and the per-vertex epilogue.
enum IterMode : int {
    // FP64, uniform teleport, the reference's update
    //   x'[v] = (1-d)/n + d*dsum/n + d*sum_{u->v} w*x[u]/s[u]   (pagerank.rs:116-129)
    MODE_PLAIN64 = 0,
    // FP64, reset-vector teleport and dangling redistribution
    //   x'[v] = (1-d)*r[v] + d*(sum + dsum*r[v])               (personalized_pagerank.rs:169-170)
    MODE_PPR64 = 1,
    // FP64 residual pass of the refined solver: g = G(x), r = g - x (stored
    // FP32), and the FP32 correction iteration is seeded with e0 = r
    MODE_RESID64 = 2,
    // FP32 correction iteration  e' = d*P^T(e/s) + d*dsum_e*t + r
    MODE_CORR32 = 3,
    // Krylov matvec y = A p of the PageRank linear system
    //   A p = p - d*P^T(p/s) - d*dsum_p*t     (pagerank_linsys.rs:221-238)
    // with the dot products (rh.y, y.p, y.y) reduced per block
    MODE_KRY32 = 4,  // FP32 vectors and gathers
    MODE_KRY64 = 5,  // FP64 vectors and gathers
    // FP64 residual pass of the Krylov solvers: g = G(x) and r = g - x
    // (written FP32 to b32_out or FP64 to b64_out), ||r||_1 and sum(g)
    MODE_KRES64 = 6,
    // adjacency product for eigenvector centrality / HITS:
    //   y = shift * x + A x  (plain sums of gathered x, no degree scaling)
    // with per-block records (max |y|, x.y, x.x)
    MODE_EIG64 = 7,
};
constexpr int kModes = 8;

// Row-end index of the in-CSR for the tile-segmented matvec (segspmv.cu):
// the arcs are cut into tiles of kSegTile; bit p of `mask` is set when arc p
// is the last arc of its row; tile_j0[t] counts the row ends before tile t;
// nz_row lists the rows that have arcs and empty_row those that have none.
constexpr uint32_t kSegTile = 256;
constexpr uint32_t kSegLongSpan = 32;
struct SegIndex {
    uint64_t ntiles = 0;
    uint32_t *mask = nullptr;       // ntiles * 8 words (+ 8 pad)
    uint32_t *tile_j0 = nullptr;    // ntiles + 1
    // per tile: {tile_j0, running row-end counts before mask words 0-3 and
    // 4-7 (one byte each), row ends in the tile | 1 << 31 when its first
    // row end closes a row begun in an earlier tile}
    uint4 *meta = nullptr;
    uint32_t *nz_row = nullptr;     // n_nz
    uint32_t *empty_row = nullptr;  // n_empty
    uint32_t n_nz = 0, n_empty = 0;
    // the rows with arcs are ids 0 .. n_nz-1 (nz_row[i] = i; degree-sorted
    // ids of a directed graph put them first), the others n_nz .. n-1
    uint32_t dense = 0;
    // rows closed in a later tile than they begin: {row, first tile, closing
    // tile, 0}, in tile order; spans of more than kSegLongSpan tiles apart
    uint4 *span = nullptr, *span_long = nullptr;
    uint32_t n_span = 0, n_long = 0;
    double *head = nullptr;         // per tile: the sum up to its first row end
    double *tail = nullptr;         // per tile: the open sum after its last row end
};

struct IterArgs {
    // graph
    const uint32_t *row_ptr;
    const uint32_t *col;
    const double *w64;
    const float *w32;
    const double *dval;
    const float *inv32;
    const uint4 *rb;
    const Hub *hubs;
    uint32_t nrb, nhub, n;
    uint32_t hot;  // sources below this id are gathered from the shared-memory hot prefix (set at launch)
    uint32_t l1hot;  // sources at or above this id are gathered without L1 allocation (set at launch)
    // vectors (FP64 modes use the *64 pointers, CORR32 the *32 ones)
    const double *xt64_in;
    const double *x64_in;
    double *x64_out;
    double *xt64_out;
    const float *xt32_in;
    const float *x32_in;
    float *x32_out;
    float *xt32_out;
    const double *t64;  // teleport distribution (null = uniform 1/n)
    const float *t32;
    const float *b32;   // CORR32: additive residual r
    float *b32_out;     // RESID64: residual r written here
    double *b64_out;    // RESID64: residual r in FP64 (optional)
    // Krylov matvec (MODE_KRY*): the input vector p is x*_in, its scaled copy
    // p/s is xt*_in, y goes to x*_out; rh* (optional) is the shadow residual
    const float *rh32;
    const double *rh64;
    const double4 *kpart_in;  // producer's per-block records; .x summed = dangling mass of p
    uint32_t kpart_n;
    double4 *kpart_out;       // per-block (rh.y, y.p, y.y)
    const int32_t *kdone;     // nonzero: the Krylov solve has stopped, return at once (may be null for EIG64)
    const double *ktol;       // MODE_KRY*, optional: when the input's norm (kpart_in .y = L1 / .z = squares
                              // summed) is <= *ktol the launch does nothing but mark kpart_out[0].w = 1
    int32_t knorm2;           // with ktol: compare the 2-norm instead of the L1 norm
    double shift;             // MODE_EIG64: weight of the diagonal term
    // scalars
    double damping;
    double inv_n;
    // tile-segmented FP32 Krylov matvec (MODE_KRY32 with LaunchCfg::seg)
    uint64_t arcs;
    const uint32_t *seg_mask, *seg_tile_j0, *seg_nz, *seg_empty;
    const uint4 *seg_meta;
    double *seg_head, *seg_tail;
    const uint4 *seg_span, *seg_span_long;
    uint64_t seg_ntiles;
    uint32_t seg_nempty, seg_nspan, seg_nlong;
    uint32_t seg_dense;  // SegIndex::dense: row of rank j is j, rows without arcs are n - seg_nempty .. n-1
    uint32_t seg_prefetch;  // the tile kernel prefetches each warp's next index tile into L2
    // reduction scratch
    Ctl *ctl;
    double4 *blk_part;   // one record per block of the persistent grid
    double *chunk_part;  // one partial sum per chunk row-block
    double4 *hub_rec;    // (diff, dangling, sum) contribution of each hub row
    uint32_t *hub_ticket;
    int parity;
};

struct LaunchCfg {
    unsigned grid = 0;  // persistent grid; for the segmented matvec, the record count seg_g1 + seg_g2
    int threads = kThreads;
    size_t smem = 0;   // dynamic shared memory (warp buffers + hot prefix)
    uint32_t hot = 0;  // hot-prefix length (vertices)
    uint32_t l1hot = 0xFFFFFFFFu;  // gathers of ids >= l1hot bypass L1
    uint32_t hub_recs = 0;  // hub-row records a Krylov consumer adds after the block records
    int seg = 0;            // MODE_KRY32: tile-segmented kernel pair (segspmv.cu): 1 = 4-arc lane quads,
                            // 2 = 8 consecutive arcs per lane
    unsigned seg_g1 = 0, seg_g2 = 0;  // its main and finishing grids
    bool seg_pipe = false;            // its tile kernel loads each warp's next tile ahead
};

// Persistent launch shape of the iteration kernel on this device: 256-thread
// blocks, as many per SM as fit (or blocks_per_sm), each optionally holding
// the first hot_entries values of the gathered vector in shared memory.
// With a hot prefix, hot_threads = 512 or 1024 gives one block of that size
// per SM instead, whose hot prefix can take most of the SM's shared memory.
LaunchCfg iteration_config(int mode, bool weighted, uint32_t hot_entries, uint32_t blocks_per_sm, uint32_t n,
                           uint32_t hot_threads = kThreads);
void launch_iteration(int mode, bool weighted, const IterArgs &a, const LaunchCfg &c, cudaStream_t s);

// Tile-segmented FP32 Krylov matvec (segspmv.cu): builds the row-end index of
// g (unweighted graphs), frees it, gives its launch shape (hot prefix of up
// to hot_entries vertices in shared memory) and launches it (two kernels:
// the tiles, then the rows that span tiles and the rows without arcs).
void seg_build(const DeviceGraph &g, SegIndex &x, cudaStream_t s);
void seg_free(SegIndex &x, cudaStream_t s);
LaunchCfg seg_config(const DeviceGraph &g, uint32_t hot_entries, int variant, int mode = MODE_KRY32);
void launch_seg(int mode, const IterArgs &a, const LaunchCfg &c, cudaStream_t s);

// Average time (ms) of a pass that only streams g's column indices and gathers
// one FP32 value per arc with the FP32 matvec's load policies (reps timed
// launches after one warm-up): the gather floor of g's index stream.
float gather_probe(const DeviceGraph &g, int reps, cudaStream_t s);

// x <- x + e (e may be null), xt <- x / dval, dangling sum and total sum of
// x into ctl->dsum[parity] / ctl->gsum via a deterministic two-level tree.
void launch_prepare64(const DeviceGraph &g, double *x, const float *e, double *xt, Ctl *ctl, int parity,
                      double4 *part, cudaStream_t s);
// x <- x / sum (final FP64 normalisation of the refined result).
void launch_normalise(double *x, uint32_t n, const Ctl *ctl, cudaStream_t s);
// x <- t (FP64 copy) or uniform 1/n when t is null.
void launch_fill_start(double *x, const double *t, uint32_t n, cudaStream_t s);
// Loads the start, prepare and id-gather kernels now (CUDA loads kernels
// lazily, allocating device memory at that point).
void preload_fp64_support();

}  // namespace prg
