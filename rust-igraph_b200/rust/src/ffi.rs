//! Raw declarations of the C ABI in include/prg_b200.h (libprg_b200.so).
//! Every function is unsafe to call: pointers must be valid for the lengths
//! the header states, and device pointers must be memory of the graph's GPU.
#![allow(non_camel_case_types, dead_code)]

use std::os::raw::{c_char, c_void};

/// Opaque resident graph (device CSR, workspace and CUDA stream).
#[repr(C)]
pub struct prg_graph {
    _opaque: [u8; 0],
}

/// Opaque warm-start network.
#[repr(C)]
pub struct prg_gnn {
    _opaque: [u8; 0],
}

pub const PRG_OK: i32 = 0;
pub const PRG_ERR_INVALID_ARGUMENT: i32 = 1;
pub const PRG_ERR_VERTEX_OUT_OF_RANGE: i32 = 2;
pub const PRG_ERR_INTERNAL: i32 = 3;
pub const PRG_ERR_CUDA: i32 = 4;
pub const PRG_ERR_OUT_OF_MEMORY: i32 = 5;
pub const PRG_ERR_DID_NOT_CONVERGE: i32 = 6;
pub const PRG_ERR_TIMEOUT: i32 = 7;
pub const PRG_ERR_PARSE: i32 = 8;
pub const PRG_ERR_IO: i32 = 9;
pub const PRG_ERR_UNSUPPORTED: i32 = 10;

pub const PRG_PRECISION_FP64: i32 = 0;
pub const PRG_PRECISION_FP32_REFINED: i32 = 1;
pub const PRG_PRECISION_FP64_KRYLOV: i32 = 2;
pub const PRG_PRECISION_LINSYS: i32 = 3;
pub const PRG_INNER_KRYLOV: i32 = 0;
pub const PRG_INNER_RICHARDSON: i32 = 1;
pub const PRG_STOP_SUCCESSIVE: i32 = 0;
pub const PRG_STOP_ERROR_BOUND: i32 = 1;
pub const PRG_EIG_OUT: i32 = 0;
pub const PRG_EIG_IN: i32 = 1;
pub const PRG_EIG_ALL: i32 = 2;

#[repr(C)]
#[derive(Clone, Copy, Debug)]
pub struct prg_options {
    pub damping: f64,
    pub eps: f64,
    pub max_iter: u32,
    pub precision: i32,
    pub stop: i32,
    pub normalise: i32,
    pub start: *const f64,
    pub inner: i32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct prg_stats {
    pub iterations: u32,
    pub fp64_passes: u32,
    pub fp32_passes: u32,
    pub residual_passes: u32,
    pub last_diff: f64,
    pub residual_l1: f64,
    pub error_bound: f64,
    pub solve_ms: f64,
    pub build_ms: f64,
    pub arcs: u64,
    pub n_dangling: u32,
    pub kernel_launches: u32,
    pub fp32_ms: f64,
    pub fp64_ms: f64,
    pub spmv_ms: f64,
    pub spmv_launches: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct prg_tune_result {
    pub capw: u32,
    pub shortmax: u32,
    pub split: u32,
    pub blocks_per_sm: u32,
    pub batch_tile_width: u32,
    pub candidates: u32,
    pub from_cache: i32,
    pub pad: u32,
    pub default_ms: f64,
    pub best_ms: f64,
    pub seg_hot: u32,
    pub seg_hot64: u32,
    pub seg_default_ms: f64,
    pub seg_best_ms: f64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default)]
pub struct prg_batch_stats {
    pub column_iterations: u64,
    pub max_iters: u32,
    pub tiles: u32,
    pub tile_width: u32,
    pub kernel_launches: u32,
    pub ms: f64,
    pub chebyshev: u32,
    pub pad: u32,
}

unsafe extern "C" {
    pub fn prg_default_options(opt: *mut prg_options);

    // drop-ins: upload, build, iterate, download in one call
    pub fn prg_pagerank(n: u32, m: u64, from: *const u32, to: *const u32, directed: i32, out: *mut f64) -> i32;
    pub fn prg_pagerank_linsys(n: u32, m: u64, from: *const u32, to: *const u32, directed: i32, out: *mut f64)
    -> i32;
    pub fn prg_pagerank_weighted(
        n: u32, m: u64, from: *const u32, to: *const u32, directed: i32, weights: *const f64, weights_len: u64,
        out: *mut f64,
    ) -> i32;
    pub fn prg_personalized_pagerank(
        n: u32, m: u64, from: *const u32, to: *const u32, directed: i32, reset: *const f64, reset_len: u64,
        damping: f64, out: *mut f64,
    ) -> i32;
    pub fn prg_personalized_pagerank_vs(
        n: u32, m: u64, from: *const u32, to: *const u32, directed: i32, reset_vids: *const u32, nvids: u64,
        damping: f64, out: *mut f64,
    ) -> i32;
    pub fn prg_eigenvector_centrality(
        n: u32, m: u64, from: *const u32, to: *const u32, directed: i32, out: *mut f64, eigenvalue: *mut f64,
    ) -> i32;
    pub fn prg_eigenvector_centrality_weighted(
        n: u32, m: u64, from: *const u32, to: *const u32, directed: i32, weights: *const f64, weights_len: u64,
        out: *mut f64, eigenvalue: *mut f64,
    ) -> i32;
    pub fn prg_eigenvector_centrality_full(
        n: u32, m: u64, from: *const u32, to: *const u32, directed: i32, mode: i32, weights: *const f64,
        weights_len: u64, out: *mut f64, eigenvalue: *mut f64,
    ) -> i32;
    pub fn prg_hub_and_authority_scores(
        n: u32, m: u64, from: *const u32, to: *const u32, directed: i32, hub: *mut f64, authority: *mut f64,
        eigenvalue: *mut f64,
    ) -> i32;
    pub fn prg_hub_and_authority_scores_weighted(
        n: u32, m: u64, from: *const u32, to: *const u32, directed: i32, weights: *const f64, weights_len: u64,
        hub: *mut f64, authority: *mut f64, eigenvalue: *mut f64,
    ) -> i32;
    pub fn prg_infomap_flow(
        n: u32, m: u64, from: *const u32, to: *const u32, directed: i32, edge_weights: *const f64,
        edge_weights_len: u64, vertex_weights: *const f64, vertex_weights_len: u64, node_flow: *mut f64,
        iterations: *mut u32,
    ) -> i32;

    // resident graphs
    pub fn prg_graph_create(
        n: u32, m: u64, from: *const u32, to: *const u32, weights: *const f64, directed: i32,
        out: *mut *mut prg_graph,
    ) -> i32;
    pub fn prg_graph_create_device(
        n: u32, m: u64, d_from: *const u32, d_to: *const u32, d_weights: *const f64, directed: i32,
        out: *mut *mut prg_graph,
    ) -> i32;
    pub fn prg_graph_destroy(g: *mut prg_graph);
    pub fn prg_graph_info(
        g: *const prg_graph, n: *mut u32, arcs: *mut u64, n_dangling: *mut u32, n_rowblocks: *mut u32,
        n_hubs: *mut u32, build_ms: *mut f64,
    ) -> i32;
    pub fn prg_graph_stream(g: *mut prg_graph) -> *mut c_void;
    pub fn prg_solve(
        g: *mut prg_graph, opt: *const prg_options, reset: *const f64, out: *mut f64, stats: *mut prg_stats,
    ) -> i32;
    pub fn prg_solve_device(
        g: *mut prg_graph, opt: *const prg_options, d_reset: *const f64, d_out: *mut f64, stats: *mut prg_stats,
    ) -> i32;
    pub fn prg_solve_noalloc(
        g: *mut prg_graph, opt: *const prg_options, d_reset: *const f64, d_out: *mut f64, stats: *mut prg_stats,
    ) -> i32;
    pub fn prg_graph_relabelled(g: *const prg_graph) -> i32;
    pub fn prg_graph_device_csr(
        g: *const prg_graph, row_ptr: *mut *const u32, col: *mut *const u32, perm: *mut *const u32,
        inv32: *mut *const f32,
    ) -> i32;
    pub fn prg_graph_gather_probe(g: *mut prg_graph, reps: i32, ms_per_pass: *mut f64) -> i32;
    pub fn prg_graph_matvec32(
        g: *mut prg_graph,
        kernel: i32,
        d_p: *const f32,
        d_pt: *const f32,
        dz: f64,
        damping: f64,
        d_y: *mut f32,
        dots: *mut f64,
        ms: *mut f64,
    ) -> i32;

    // batched personalized PageRank
    pub fn prg_ppr_batch(
        g: *mut prg_graph, k: u32, seed_offsets: *const u64, seeds: *const u32, damping: f64, tol: f64,
        max_iter: u32, tile_vec: u32, out: *mut f32, column_iters: *mut u32, stats: *mut prg_batch_stats,
    ) -> i32;
    pub fn prg_ppr_batch_device(
        g: *mut prg_graph, k: u32, seed_offsets: *const u64, seeds: *const u32, damping: f64, tol: f64,
        max_iter: u32, tile_vec: u32, d_out: *mut f32, column_iters: *mut u32, stats: *mut prg_batch_stats,
    ) -> i32;

    // tuning and the warm-start network
    pub fn prg_autotune(g: *mut prg_graph, tune_batch: i32, cache_path: *const c_char, out: *mut prg_tune_result)
    -> i32;
    pub fn prg_set_tuning(key: *const c_char, value: i64) -> i32;
    pub fn prg_gnn_param_count() -> u32;
    pub fn prg_gnn_create(seed: u64, out: *mut *mut prg_gnn) -> i32;
    pub fn prg_gnn_destroy(net: *mut prg_gnn);
    pub fn prg_gnn_get_params(net: *const prg_gnn, host: *mut f32) -> i32;
    pub fn prg_gnn_set_params(net: *mut prg_gnn, host: *const f32) -> i32;
    pub fn prg_gnn_predict(net: *mut prg_gnn, g: *mut prg_graph, d_start: *mut f64, ms: *mut f64) -> i32;
    pub fn prg_gnn_loss_grad(
        net: *mut prg_gnn, g: *mut prg_graph, d_target: *const f64, loss: *mut f64, host_grad: *mut f32,
    ) -> i32;
    pub fn prg_gnn_train_step(net: *mut prg_gnn, g: *mut prg_graph, d_target: *const f64, lr: f32, loss: *mut f64)
    -> i32;

    // seeded device generators (benchmark and training inputs)
    pub fn prg_rmat_device(
        scale: u32, m: u64, a: f64, b: f64, c: f64, seed: u64, d_from: *mut u32, d_to: *mut u32,
        stream: *mut c_void,
    ) -> i32;
    pub fn prg_generate_device(
        kind: i32, n: u32, m: u64, p0: f64, p1: f64, p2: f64, seed: u64, d_from: *mut u32, d_to: *mut u32,
        stream: *mut c_void,
    ) -> i32;

    // edge-list reader
    pub fn prg_parse_edgelist(
        text: *const c_char, len: u64, from: *mut u32, to: *mut u32, capacity: u64, m: *mut u64, n: *mut u32,
        err_line: *mut u64,
    ) -> i32;
    pub fn prg_read_edgelist(
        text: *const c_char, len: u64, out: *mut *mut prg_graph, n: *mut u32, m: *mut u64, err_line: *mut u64,
    ) -> i32;

    pub fn prg_last_error() -> *const c_char;
    pub fn prg_last_error_len() -> u64;
}
