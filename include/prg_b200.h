/*
 * prg_b200.h — C ABI of the B200 PageRank library (libprg_b200.so).
 *
 * This is the drop-in boundary for rust-igraph's PageRank hot path.  A Rust
 * wrapper crate (build.rs compiles the CUDA sources with nvcc for sm_100a and
 * links this library) binds these symbols behind the crate's own signatures:
 *
 *   pagerank(&Graph) -> IgraphResult<Vec<f64>>
 *       src/algorithms/properties/pagerank.rs:52          -> prg_pagerank
 *   pagerank_weighted(&Graph, &[f64]) -> IgraphResult<Vec<f64>>
 *       src/algorithms/properties/pagerank_weighted.rs:52 -> prg_pagerank_weighted
 *   personalized_pagerank(&Graph, &[f64], f64) -> IgraphResult<Vec<f64>>
 *       src/algorithms/properties/personalized_pagerank.rs:65  -> prg_personalized_pagerank
 *   personalized_pagerank_default(&Graph, &[f64])
 *       src/algorithms/properties/personalized_pagerank.rs:206 -> prg_personalized_pagerank (d = 0.85)
 *   personalized_pagerank_vs(&Graph, &[u32], f64)
 *       src/algorithms/properties/personalized_pagerank.rs:241 -> prg_personalized_pagerank_vs
 *
 * The graph crosses the boundary as rust-igraph stores it: n, the edge list
 * (from[e], to[e]) in edge-id order (src/core/graph.rs:126-152, Graph::edge
 * at :1152) and the directedness flag (:582).  Outputs are caller-allocated
 * double[n] host arrays.  Every entry point is synchronous; calls on
 * different graph handles may run from different threads (each handle owns
 * a CUDA stream); one handle must not be used by two threads at once (the
 * reference Graph is !Sync, src/core/cache.rs:88-91).
 *
 * Status codes map one-to-one onto rust-igraph's IgraphError variants
 * (src/core/error.rs:14-66); prg_last_error() returns the message text
 * (the reference's own wording for validation errors).
 */
#ifndef PRG_B200_H
#define PRG_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct prg_graph prg_graph;

enum prg_status {
    PRG_OK = 0,
    PRG_ERR_INVALID_ARGUMENT = 1,     /* IgraphError::InvalidArgument(String) */
    PRG_ERR_VERTEX_OUT_OF_RANGE = 2,  /* IgraphError::VertexOutOfRange */
    PRG_ERR_INTERNAL = 3,             /* IgraphError::Internal(&'static str) */
    PRG_ERR_CUDA = 4,                 /* IgraphError::Internal("cuda: ...") */
    PRG_ERR_OUT_OF_MEMORY = 5,        /* IgraphError::Internal("cuda: out of memory") */
    PRG_ERR_DID_NOT_CONVERGE = 6,     /* IgraphError::DidNotConverge (never raised by the drop-ins) */
    PRG_ERR_TIMEOUT = 7,              /* a bounded device wait expired (batched solver) */
    PRG_ERR_PARSE = 8,                /* IgraphError::Parse { line, message } */
    PRG_ERR_IO = 9,                   /* IgraphError::Io (the text is not valid UTF-8) */
    PRG_ERR_UNSUPPORTED = 10          /* IgraphError::Unsupported(&'static str) */
};

enum prg_precision {
    PRG_PRECISION_FP64 = 0,           /* FP64 power iteration (the drop-in path) */
    PRG_PRECISION_FP32_REFINED = 1,   /* FP32 SpMV inner solves, FP64 residual refinement, certified stop */
    PRG_PRECISION_FP64_KRYLOV = 2,    /* FP64 BiCGStab on the linear system, certified stop */
    PRG_PRECISION_LINSYS = 3          /* pagerank_linsys() rule: ||b - Ax||_2 < 1e-13 ||b||_2, returns x */
};

enum prg_inner {
    PRG_INNER_KRYLOV = 0,             /* refined: BiCGStab on A e = r in FP32 (default) */
    PRG_INNER_RICHARDSON = 1          /* refined: power-style correction e <- d M e + r in FP32 */
};

enum prg_stop {
    PRG_STOP_SUCCESSIVE = 0,          /* reference rule: stop when successive L1 change < eps */
    PRG_STOP_ERROR_BOUND = 1          /* stop when the certified L1 error vs the fixed point <= eps */
};

typedef struct prg_options {
    double damping;        /* default 0.85 (pagerank.rs:23) */
    double eps;            /* default 1e-10 (pagerank.rs:24) */
    uint32_t max_iter;     /* default 1000 (pagerank.rs:25); refined: cap on all SpMV passes */
    int32_t precision;     /* enum prg_precision */
    int32_t stop;          /* enum prg_stop (refined precision always uses ERROR_BOUND) */
    int32_t normalise;     /* refined: divide the result by its FP64 sum (default 1) */
    const double *start;   /* optional start vector (warm start), length n, host memory; NULL = reference start */
    int32_t inner;         /* enum prg_inner (refined precision only) */
} prg_options;

typedef struct prg_stats {
    uint32_t iterations;       /* SpMV passes of any precision */
    uint32_t fp64_passes;
    uint32_t fp32_passes;
    uint32_t residual_passes;  /* FP64 residual passes of the refined solver */
    double last_diff;          /* last successive L1 change (FP64 path) */
    double residual_l1;        /* ||G(x) - x||_1 of the returned vector's predecessor */
    double error_bound;        /* certified bound on ||x - x*||_1 */
    double solve_ms;           /* device time of the solve (CUDA events) */
    double build_ms;           /* device time of the graph build */
    uint64_t arcs;
    uint32_t n_dangling;
    uint32_t kernel_launches;  /* CUDA kernels this solve launched (graph nodes included) */
    double fp32_ms;            /* device time of the FP32 iteration graphs (CUDA events) */
    double fp64_ms;            /* device time of the FP64 iteration graphs / residual passes */
    double spmv_ms;            /* device time of the SpMV launches that did work: the power iteration's
                                  graphs, or the Krylov inner solve's matvec kernels (CUDA events) */
    uint32_t spmv_launches;    /* the SpMV launches spmv_ms covers */
} prg_stats;

/* Fills the reference defaults: d = 0.85, eps = 1e-10, max_iter = 1000,
 * FP64, successive-change stop, normalise = 1, no start vector. */
void prg_default_options(prg_options *opt);

/* ---- drop-ins: one call = upload, build, iterate, download ------------ */

/* rust-igraph pagerank() (pagerank.rs:52-143). */
int32_t prg_pagerank(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to, int32_t directed,
                     double *out);

/* rust-igraph pagerank_linsys() (pagerank_linsys.rs:99-160): the same fixed
 * point as a linear system (I - 0.85 M^T) x = 0.15/n * 1, solved to
 * ||b - A x||_2 < 1e-13 ||b||_2 from the uniform start; unweighted. */
int32_t prg_pagerank_linsys(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to, int32_t directed,
                            double *out);

/* rust-igraph eigenvector_centrality() (src/algorithms/properties/eigenvector.rs:118-125,
 * 286-372): undirected, unweighted; the max-normalised shifted power
 * iteration x' = (A + I) x to an L1 change < 1e-14 (at most 5000
 * iterations), negatives clamped.  *eigenvalue (optional) receives the
 * Rayleigh quotient x.Ax / x.x.  A directed graph gives PRG_ERR_UNSUPPORTED
 * like the reference. */
int32_t prg_eigenvector_centrality(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to, int32_t directed,
                                   double *out, double *eigenvalue);

/* rust-igraph hub_and_authority_scores() (src/algorithms/properties/hits.rs:122-230),
 * unweighted: hub[n], authority[n] (max element 1) and the dominant
 * eigenvalue of A A^T.  Undirected graphs: both vectors are the eigenvector
 * centrality and the eigenvalue its squared Rayleigh quotient. */
int32_t prg_hub_and_authority_scores(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to,
                                     int32_t directed, double *hub, double *authority, double *eigenvalue);

/* rust-igraph eigenvector_centrality_weighted() (eigenvector.rs:157-168, 375-538):
 * undirected, weights[e] per edge (weights_len must equal m); shifted power
 * iteration x' = (W + I) x from the vertex strengths, L1 stop 1e-12.
 * With a negative weight the iteration follows the reference's signed rules:
 * each iterate is divided by its component of greatest magnitude with its
 * sign (the lowest vertex id on ties), a zero strength on a vertex with
 * edges seeds 1, and nothing is clamped. */
int32_t prg_eigenvector_centrality_weighted(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to,
                                            int32_t directed, const double *weights, uint64_t weights_len,
                                            double *out, double *eigenvalue);

/* EigenvectorMode (eigenvector.rs:63-76). */
enum prg_eig_mode { PRG_EIG_OUT = 0, PRG_EIG_IN = 1, PRG_EIG_ALL = 2 };

/* rust-igraph eigenvector_centrality_full() (eigenvector.rs:238-285), with
 * eigenvector_centrality_directed / _directed_weighted as its cases;
 * weights may be NULL (unweighted), else weights_len must equal m; with a
 * negative weight the reference's signed rules apply as in
 * prg_eigenvector_centrality_weighted, and there is no DAG or zero-eigenvalue
 * shortcut.  Undirected graphs take the
 * symmetric path whatever the mode.  On directed graphs, Out / In walk the
 * in- / out-edges of each vertex (directed_path, eigenvector.rs:539-720):
 * a DAG gives 1 on vertices with zero out- / in-strength and eigenvalue 0;
 * otherwise a power iteration shifted by the largest row sum + 1 from the
 * in- / out-strengths, L1 stop 1e-12, and an eigenvalue <= 1e-12 gives the
 * zero vector.  All on a directed graph iterates over the out-edges, as the
 * reference's symmetric routines see a directed graph there. */
int32_t prg_eigenvector_centrality_full(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to,
                                        int32_t directed, int32_t mode, const double *weights, uint64_t weights_len,
                                        double *out, double *eigenvalue);

/* rust-igraph hub_and_authority_scores_weighted() (hits.rs:245-585): W W^T
 * power iteration from the out-strengths (directed) or the weighted shifted
 * iteration from the signed strengths with the squared Rayleigh quotient
 * (undirected).  With a negative weight each iterate is divided by its
 * signed component of greatest magnitude, which is then the eigenvalue
 * estimate, and nothing is clamped. */
int32_t prg_hub_and_authority_scores_weighted(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to,
                                              int32_t directed, const double *weights, uint64_t weights_len,
                                              double *hub, double *authority, double *eigenvalue);

/* Node flows of rust-igraph's Infomap flow model (community/infomap.rs:
 * 233-355, the private power_iteration_pagerank): tau = 0.15 teleportation
 * to vertex_weights / sum (uniform 1/n when NULL), arc weights edge_weights
 * (unit when NULL) normalised by the out-strength, the dangling mass sent
 * back through the teleport weights undamped, each iterate renormalised to
 * sum 1; stops at an L1 change < 1e-10 or after 1000 iterations.  Checks
 * the weights as infomap_with_options does (infomap.rs:175-218), in its
 * order and with its messages.  node_flow[n]; iterations (optional). */
int32_t prg_infomap_flow(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to, int32_t directed,
                         const double *edge_weights, uint64_t edge_weights_len, const double *vertex_weights,
                         uint64_t vertex_weights_len, double *node_flow, uint32_t *iterations);

/* rust-igraph pagerank_weighted() (pagerank_weighted.rs:52-161).
 * weights_len is the caller's slice length (checked against m like :62-68). */
int32_t prg_pagerank_weighted(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to,
                              int32_t directed, const double *weights, uint64_t weights_len, double *out);

/* rust-igraph personalized_pagerank() (personalized_pagerank.rs:65-182). */
int32_t prg_personalized_pagerank(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to,
                                  int32_t directed, const double *reset, uint64_t reset_len, double damping,
                                  double *out);

/* rust-igraph personalized_pagerank_vs() (personalized_pagerank.rs:241-268). */
int32_t prg_personalized_pagerank_vs(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to,
                                     int32_t directed, const uint32_t *reset_vids, uint64_t nvids,
                                     double damping, double *out);

/* ---- resident graphs: build once in HBM, solve many times ------------- */

/* Builds the device CSR from host arrays (weights may be NULL). */
int32_t prg_graph_create(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to,
                         const double *weights, int32_t directed, prg_graph **out);
/* Same from device arrays (already in this GPU's memory). */
int32_t prg_graph_create_device(uint32_t n, uint64_t m, const uint32_t *d_from, const uint32_t *d_to,
                                const double *d_weights, int32_t directed, prg_graph **out);
void prg_graph_destroy(prg_graph *g);
/* n, in-CSR arc count, dangling vertices, row-blocks, hub rows, build time (ms). */
int32_t prg_graph_info(const prg_graph *g, uint32_t *n, uint64_t *arcs, uint32_t *n_dangling, uint32_t *n_rowblocks,
                       uint32_t *n_hubs, double *build_ms);
/* The CUDA stream (cudaStream_t) every call on this handle runs on. */
void *prg_graph_stream(prg_graph *g);

/* Solve on a resident graph.  reset: host teleport vector (length n, raw,
 * normalised inside like personalized_pagerank.rs:110-111) or NULL for the
 * uniform teleport of pagerank().  out: host double[n]. */
int32_t prg_solve(prg_graph *g, const prg_options *opt, const double *reset, double *out, prg_stats *stats);
/* Same with device pointers: d_reset (already normalised, or NULL) and d_out. */
int32_t prg_solve_device(prg_graph *g, const prg_options *opt, const double *d_reset, double *d_out,
                         prg_stats *stats);

/* 1 if the graph uses degree-sorted internal vertex ids (results are always
 * returned in the caller's ids), else 0. */
int32_t prg_graph_relabelled(const prg_graph *g);

/* Read-only views of the device CSR in internal ids (row_ptr[n+1], col[arcs],
 * perm = internal -> caller id or NULL, inv32 = 1/out-degree in FP32), for
 * callers that run their own kernels over the resident graph. */
int32_t prg_graph_device_csr(const prg_graph *g, const uint32_t **row_ptr, const uint32_t **col,
                             const uint32_t **perm, const float **inv32);

/* Diagnostic with no counterpart in the reference: the average time (ms) of
 * a pass that only streams the graph's column indices and gathers one FP32
 * value per arc, with the FP32 matvec's load policies (reps timed passes after
 * one warm-up).  It bounds from below any pass over this graph that gathers
 * once per arc; bench.py reports the matvec against it. */
int32_t prg_graph_gather_probe(prg_graph *g, int32_t reps, double *ms_per_pass);

/* Diagnostic with no counterpart in the reference: one FP32 Krylov matvec
 * y = p - d (A pt + dz / n), the operator the refined and FP32 Krylov solves
 * apply, on the graph's INTERNAL ids (prg_graph_device_csr gives the CSR
 * and numbering).  A sums pt over each row's in-arcs; pt is p scaled by
 * 1/out-degree (inv32) and dz the dangling mass of p, both the caller's.
 * kernel: 0 the row-block pass, 1 the tile-segmented pass with 4-arc lane
 * quads, 2 the tile-segmented pass with 8 consecutive arcs per lane (1 and 2
 * need an unweighted graph).  dots (3 doubles, optional) = (p.y, y.p, y.y)
 * as the kernel's block records sum them; ms (optional) = its device time.
 * Device pointers, n entries each.  Tests compare the three kernels with an
 * FP64 restatement through it. */
int32_t prg_graph_matvec32(prg_graph *g, int32_t kernel, const float *d_p, const float *d_pt, double dz,
                           double damping, float *d_y, double *dots, double *ms);

/* ---- learned warm start --------------------------------------------------- */
/* A two-layer message-passing network (hidden 32, 8-channel messages scaled
 * by 1/out-degree, BF16 weights, FP32 accumulation on the tensor cores) that
 * predicts the PageRank vector from degree features.  Its normalised output
 * is only a start vector for prg_solve / prg_solve_device (prg_options.start):
 * the fixed point, stop rule and checks are those of the plain method.  No
 * counterpart in the reference (an addition of this library). */
typedef struct prg_gnn prg_gnn;

uint32_t prg_gnn_param_count(void);
/* New network with seeded random weights. */
int32_t prg_gnn_create(uint64_t seed, prg_gnn **out);
void prg_gnn_destroy(prg_gnn *net);
/* FP32 master parameters to / from host float[prg_gnn_param_count()]. */
int32_t prg_gnn_get_params(const prg_gnn *net, float *host);
int32_t prg_gnn_set_params(prg_gnn *net, const float *host);
/* Predicted start vector (caller ids, sums to 1) into device double[n];
 * *ms = device time of the inference. */
int32_t prg_gnn_predict(prg_gnn *net, prg_graph *g, double *d_start, double *ms);
/* Loss sum_v w_v (y_v - log(n x*_v))^2 / n (w_v = n x*_v) against a target
 * PageRank vector (device, caller ids) and its gradient (host float[count],
 * optional), without updating the weights. */
int32_t prg_gnn_loss_grad(prg_gnn *net, prg_graph *g, const double *d_target, double *loss, float *host_grad);
/* One Adam step (lr) on that loss. */
int32_t prg_gnn_train_step(prg_gnn *net, prg_graph *g, const double *d_target, float lr, double *loss);

/* ---- autotuner --------------------------------------------------------- */

typedef struct prg_tune_result {
    uint32_t capw, shortmax, split;  /* row-block shape chosen */
    uint32_t blocks_per_sm;          /* persistent grid (0 = occupancy maximum) */
    uint32_t batch_tile_width;       /* batched solver columns per tile */
    uint32_t candidates;             /* configurations timed */
    int32_t from_cache;              /* 1 if read from cache_path instead of timed */
    uint32_t pad;
    double default_ms, best_ms;      /* FP64 + FP32 iteration time before / after */
    /* unweighted graphs (0 otherwise): the shared-memory hot prefixes chosen
     * for the tile-segmented FP32 matvec and FP64 passes, and the FP32
     * matvec's time with the default and the chosen prefix */
    uint32_t seg_hot, seg_hot64;
    double seg_default_ms, seg_best_ms;
} prg_tune_result;

/* Times candidate row-block shapes (stream window, short-row limit, hub
 * split), persistent-grid occupancies, on unweighted graphs the hot-prefix
 * lengths of the tile-segmented passes, and (tune_batch != 0) batched tile
 * widths on this graph with CUDA events and keeps the fastest.  cache_path
 * (optional): a text file of earlier results keyed by (n, arcs, directed,
 * weighted); a hit is applied without timing, a new result is appended. */
int32_t prg_autotune(prg_graph *g, int32_t tune_batch, const char *cache_path, prg_tune_result *out);

/* Process-wide tuning applied to graphs created afterwards (the autotuner's
 * knobs): "capw", "shortmax", "split" (row-block shape), "blocks_per_sm"
 * (persistent grid, 0 = occupancy maximum), "relabel" (0 off, 1 on, 2 auto on
 * skewed degree distributions), "refine_switch_e12" (refined precision: FP64
 * power steps until the successive change is below value * 1e-12, then FP32
 * corrections; default 500000), "batch_vec" (batched columns per lane: 1, 2
 * or 4), "hot_cache" (relabelled graphs: each block of the iteration kernel
 * keeps the first `value` entries of the gathered vector in shared memory,
 * 0 = off, at most 65536), "unroll" (iteration pairs per CUDA
 * graph), "krylov_rel_e12" (refined precision with the Krylov inner solver:
 * each FP32 inner solve reduces the residual by value * 1e-12; default 1e8,
 * i.e. 1e-4), "l1_hot32" / "l1_hot64" (relabelled graphs: FP32 / FP64
 * passes gather sources with ids >= value without allocating in L1, so L1
 * keeps the most-gathered prefix; defaults 16384 / 2048, 0 = all allocate),
 * "defaults" (any value: every key back to its default),
 * "krylov_floor_pct" (Krylov inner solves aim at this percentage of the
 * certified final threshold, 1-90; default 70), "seg_kry32" (unweighted
 * graphs: the tile-segmented FP32 Krylov matvec, 1 with 4-arc lane quads, 2
 * with 8 consecutive arcs per lane; 0 the row-block kernel),
 * "seg_hot" (its shared-memory hot prefix on relabelled graphs, entries),
 * "seg_res64" (unweighted graphs: 1 the tile-segmented FP64 residual pass
 * of the refined and Krylov solves, 0 the row-block kernel), "seg_hot64"
 * (its hot prefix, at most 20480 entries; the FP64 power step shares it),
 * "seg_eig64" (unweighted graphs: 1 the tile-segmented adjacency product of
 * the eigenvector and HITS iterations, the default; 0 the row-block kernel),
 * "seg_plain64" (unweighted graphs: 1 the tile-segmented FP64 power step of
 * the drop-ins and the certified FP64 loop, and the FP64 Krylov matvec of
 * the FP64 Krylov and pagerank_linsys solves; 0 the row-block kernel),
 * "seg_prefetch" (segmented passes:
 * 1 each warp prefetches its next tile of column indices into L2, 0 off),
 * "seg_threads" (their tile kernel's block size, one block per SM: 1024, 768
 * or 512), "seg_pipe" (1: each warp of the FP32 tile kernel loads its next
 * tile while it works on the current one),
 * "hot_cache32" / "hot_cache64" (hot prefix of the row-block kernel's FP32 /
 * FP64 passes), "hot_threads" (256, 512 or 1024: the row-block kernel's block
 * size when it keeps a hot prefix),
 * "batch_cheb" (batched solver on undirected graphs: 1 Chebyshev steps, 0
 * plain power steps, the default),
 * "batch_barrier_extra" (failure-detection test hook, 0 or 1: with 1 every
 * grid barrier of the batched solver waits for an arrival that never comes,
 * so its bounded wait (about 1.5 s) expires and the call returns
 * PRG_ERR_TIMEOUT with the context still usable; leave it 0). */
int32_t prg_set_tuning(const char *key, int64_t value);

/* ---- batched personalized PageRank ---------------------------------- */

typedef struct prg_batch_stats {
    uint64_t column_iterations; /* sum over columns of the iterations each ran */
    uint32_t max_iters;         /* iterations of the slowest column */
    uint32_t tiles;             /* column tiles (one persistent launch each) */
    uint32_t tile_width;        /* columns per tile (32 * vec) */
    uint32_t kernel_launches;
    double ms;                  /* device time (CUDA events) */
    uint32_t chebyshev;         /* 1: Chebyshev steps (undirected graph), 0: plain power steps */
    uint32_t pad;
} prg_batch_stats;

/* K personalized PageRank vectors at once (FP32 SpMM with FP32 accumulation).
 * Column k is rust-igraph personalized_pagerank_vs(graph, seeds_k, damping)
 * (personalized_pagerank.rs:241-268 building the reset, :65-182 iterating)
 * with seeds_k = seeds[seed_offsets[k] .. seed_offsets[k+1]) in caller ids,
 * stopped per column when its successive L1 change is < tol (the column then
 * freezes while the others continue) or after max_iter iterations.  On an
 * undirected graph (real spectrum) and with tuning key "batch_cheb" = 1, the
 * iterates between those tests are Chebyshev steps over an interval each
 * column estimates from the settled contraction ratio of its first power
 * steps (default 0: plain steps throughout): the test is still the change
 * one power step makes,
 * ||G(x) - x||_1 < tol, and the column returns that step, G(x), as the
 * reference does; only the sequence of iterates before it is shorter.  FP32
 * rounding puts a floor of about n ulp under that change, so a Chebyshev
 * column finishes with plain steps once its change is below 100 x tol; if
 * those stop falling within 10 x tol (a rounding cycle at the floor) it
 * freezes there, its answer within d/(1-d) of that change of the fixed
 * point.
 * tile_vec: columns per tile = 32 * tile_vec (1, 2 or 4; 0 = autotuned or 2).
 * out: host float[n * K], out[v * K + k].  column_iters: optional host
 * uint32[K].  Validation follows _vs: empty seed list or vertex >= n ->
 * PRG_ERR_INVALID_ARGUMENT; a device barrier that times out -> PRG_ERR_TIMEOUT. */
int32_t prg_ppr_batch(prg_graph *g, uint32_t K, const uint64_t *seed_offsets, const uint32_t *seeds, double damping,
                      double tol, uint32_t max_iter, uint32_t tile_vec, float *out, uint32_t *column_iters,
                      prg_batch_stats *stats);
/* Same with a device output buffer d_out (float[n * K]). */
int32_t prg_ppr_batch_device(prg_graph *g, uint32_t K, const uint64_t *seed_offsets, const uint32_t *seeds,
                             double damping, double tol, uint32_t max_iter, uint32_t tile_vec, float *d_out,
                             uint32_t *column_iters, prg_batch_stats *stats);

/* Allocation-free FP64 solve (no counterpart in the reference; an addition
 * for callers that must not allocate device memory at solve time, such as a
 * real-time loop that reserves memory up front or code running under another
 * framework's memory budget).  Same iteration and stop rule as prg_solve at
 * PRG_PRECISION_FP64 on a graph created earlier, with the same option checks;
 * opt->start, when set, is a device start vector in caller ids.  d_reset:
 * optional normalised teleport vector, d_out: double[n], both device memory
 * in caller ids.  All solve scratch lives in one static device array (about
 * 26.6 MiB per GPU, held until exit); limits: n <= 524,288, <= 262,144
 * row-blocks, <= 8,192 hub rows, FP64 only (else PRG_ERR_INVALID_ARGUMENT).
 * CUDA allocates that array (and loads the kernels) on first use, so
 * creating a graph handle within those limits (prg_graph_create*,
 * prg_read_edgelist) does it then; the solve itself, its first call
 * included, allocates nothing.  Calls share the array, so calls that
 * overlap on the GPU race; run them one at a time. */
int32_t prg_solve_noalloc(prg_graph *g, const prg_options *opt, const double *d_reset, double *d_out,
                          prg_stats *stats);

/* ---- edge-list reader ---------------------------------------------------- */

/* rust-igraph read_edgelist() (src/algorithms/io/edgelist.rs:25-72) with the
 * parsing on the GPU.  text: the file's bytes (len of them, host memory).
 * One edge "u v" per line (u32 ids, whitespace-separated); after trimming,
 * blank lines and lines starting with '#' are skipped; the graph is
 * undirected with n = max id + 1.  On success from/to (capacity entries,
 * host) receive the m edges in file order.  Errors, for the first failing
 * line in file order: PRG_ERR_PARSE with *err_line (1-based) and the
 * reference's message ("missing vertex id", "invalid vertex id `t`: ...",
 * "expected exactly two vertex ids"); PRG_ERR_IO when a line is not valid
 * UTF-8; PRG_ERR_INVALID_ARGUMENT when m exceeds capacity (*m is set). */
int32_t prg_parse_edgelist(const char *text, uint64_t len, uint32_t *from, uint32_t *to, uint64_t capacity,
                           uint64_t *m, uint32_t *n, uint64_t *err_line);
/* Same, building the resident graph straight from the parsed edges (they
 * never leave the GPU).  A text without edges gives *out = NULL, n = m = 0. */
int32_t prg_read_edgelist(const char *text, uint64_t len, prg_graph **out, uint32_t *n, uint64_t *m,
                          uint64_t *err_line);

/* Message of the last error on this thread ("" if none). */
const char *prg_last_error(void);
/* Its length in bytes: a message that quotes input text (an edge-list token)
 * may contain NUL bytes, so read prg_last_error_len() bytes, not up to NUL. */
uint64_t prg_last_error_len(void);

/* ---- device R-MAT generator (benchmark inputs) ------------------------ */
/* Counter-based R-MAT (same edge stream as the CPU generator in the tests):
 * writes m edges into device arrays d_from/d_to. */
int32_t prg_rmat_device(uint32_t scale, uint64_t m, double a, double b, double c, uint64_t seed,
                        uint32_t *d_from, uint32_t *d_to, void *stream);

/* Seeded device generators for warm-start training graphs: kind 0 R-MAT
 * (p0, p1, p2 = a, b, c; vertex ids < next power of two >= n), 1 Chung-Lu
 * power law (p0 = exponent alpha of the weight (i + p1)^-alpha), 2 block
 * model with a fixed edge count (p0 = number of equal blocks, p1 = probability
 * that an edge stays inside its block).  Writes m edges. */
int32_t prg_generate_device(int32_t kind, uint32_t n, uint64_t m, double p0, double p1, double p2, uint64_t seed,
                            uint32_t *d_from, uint32_t *d_to, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* PRG_B200_H */
