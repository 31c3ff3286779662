//! rust-igraph's PageRank hot path on an NVIDIA B200, through libprg_b200.
//!
//! The free functions keep rust-igraph's signatures, argument meaning and
//! errors, so a caller switches by changing the `use` path:
//!
//! | rust-igraph | here |
//! |---|---|
//! | `pagerank` (src/algorithms/properties/pagerank.rs:52) | [`pagerank`] -> `prg_pagerank` |
//! | `pagerank_weighted` (pagerank_weighted.rs:52) | [`pagerank_weighted`] -> `prg_pagerank_weighted` |
//! | `personalized_pagerank` (personalized_pagerank.rs:65) | [`personalized_pagerank`] |
//! | `personalized_pagerank_default` (:206) | [`personalized_pagerank_default`] (damping 0.85) |
//! | `personalized_pagerank_vs` (:241) | [`personalized_pagerank_vs`] |
//! | `pagerank_linsys` (pagerank_linsys.rs:99) | [`pagerank_linsys`] |
//! | `Graph::pagerank` etc. (src/core/graph.rs:1857, 5454, 6285, 7002) | [`PageRankExt`] |
//! | `eigenvector_centrality*`, `hub_and_authority_scores*`, `read_edgelist` | same names |
//!
//! The graph crosses the boundary as rust-igraph stores it: `vcount()`, the
//! edge list in edge-id order from `Graph::edge` (src/core/graph.rs:1152) and
//! `is_directed()`.  The library validates in the reference's order with its
//! message text; [`check`] maps its status codes onto `IgraphError`
//! (src/core/error.rs:14-69).  Every call is synchronous and runs on the GPU:
//! there is no CPU fallback, and a missing GPU is `IgraphError::Internal`.
//!
//! rust-igraph's own `Graph` methods cannot call this crate (it depends on
//! rust-igraph, and rust-igraph denies unsafe code), so the method forms
//! come as the extension trait [`PageRankExt`], implemented for `Graph`.

mod ffi;

pub use ffi::{PRG_PRECISION_FP32_REFINED, PRG_PRECISION_FP64, PRG_PRECISION_FP64_KRYLOV, PRG_PRECISION_LINSYS};
pub use ffi::{PRG_STOP_ERROR_BOUND, PRG_STOP_SUCCESSIVE};

use rust_igraph::{EigenvectorMode, EigenvectorScores, Graph, HitsScores, IgraphError, IgraphResult};

/// The edge list in edge-id order, as two id arrays.
fn edges(g: &Graph) -> IgraphResult<(Vec<u32>, Vec<u32>)> {
    let m = u32::try_from(g.ecount()).map_err(|_| IgraphError::Internal("ecount overflows u32"))?;
    let mut f = Vec::with_capacity(m as usize);
    let mut t = Vec::with_capacity(m as usize);
    for e in 0..m {
        let (a, b) = g.edge(e)?;
        f.push(a);
        t.push(b);
    }
    Ok((f, t))
}

/// The library's last message on this thread.  It may quote input bytes,
/// NUL included, so its full length is read.
fn last_message() -> String {
    // SAFETY: the library returns a buffer of prg_last_error_len() bytes that
    // stays valid until the next call on this thread.
    let bytes = unsafe {
        let p = ffi::prg_last_error() as *const u8;
        let len = ffi::prg_last_error_len() as usize;
        if p.is_null() || len == 0 { &[][..] } else { std::slice::from_raw_parts(p, len) }
    };
    String::from_utf8_lossy(bytes).into_owned()
}

/// "vertex id {id} out of range (vcount = {n})" -> (id, n).
fn vertex_range(msg: &str) -> (u32, u32) {
    let nums: Vec<u32> = msg
        .split(|c: char| !c.is_ascii_digit())
        .filter(|s| !s.is_empty())
        .filter_map(|s| s.parse().ok())
        .collect();
    match nums.as_slice() {
        [id, n, ..] => (*id, *n),
        _ => (u32::MAX, 0),
    }
}

/// `IgraphError::Internal` and `Unsupported` carry `&'static str`: the
/// library's messages for them are a fixed set, mapped here to the
/// reference's own strings where the reference raises the same error.
fn internal_static(msg: &str) -> &'static str {
    match msg {
        "ecount overflows u32" => "ecount overflows u32",
        "arc count exceeds the u32 CSR index range" => "arc count exceeds the u32 CSR index range",
        "vertex count exceeds 2^31 - 1" => "vertex count exceeds 2^31 - 1",
        "vertex id u32::MAX cannot be sized into n" => "vertex id u32::MAX cannot be sized into n",
        _ => "internal error in the GPU library (see prg_last_error)",
    }
}

fn unsupported_static(msg: &str) -> &'static str {
    if msg.contains("eigenvector_centrality_weighted") {
        "directed eigenvector_centrality_weighted — use eigenvector_centrality_directed_weighted"
    } else if msg.contains("eigenvector_centrality") {
        "directed eigenvector_centrality — use eigenvector_centrality_directed or _full"
    } else {
        "unsupported by the GPU library"
    }
}

/// Status code of libprg_b200 -> `IgraphResult`.
pub fn check(rc: i32) -> IgraphResult<()> {
    match rc {
        ffi::PRG_OK => Ok(()),
        ffi::PRG_ERR_INVALID_ARGUMENT => Err(IgraphError::InvalidArgument(last_message())),
        ffi::PRG_ERR_VERTEX_OUT_OF_RANGE => {
            let (id, n) = vertex_range(&last_message());
            Err(IgraphError::VertexOutOfRange { id, n })
        }
        ffi::PRG_ERR_INTERNAL => Err(IgraphError::Internal(internal_static(&last_message()))),
        ffi::PRG_ERR_CUDA => Err(IgraphError::Internal("cuda error (see prg_last_error)")),
        ffi::PRG_ERR_OUT_OF_MEMORY => Err(IgraphError::Internal("cuda: out of memory")),
        // never raised by the drop-ins, which return the last iterate as the
        // reference does
        ffi::PRG_ERR_DID_NOT_CONVERGE => Err(IgraphError::DidNotConverge { iters: 0, residual: f64::NAN }),
        ffi::PRG_ERR_TIMEOUT => Err(IgraphError::Internal("a bounded device wait timed out")),
        ffi::PRG_ERR_PARSE => Err(IgraphError::Parse { line: 0, message: last_message() }),
        ffi::PRG_ERR_IO => Err(IgraphError::Io(std::io::Error::new(std::io::ErrorKind::InvalidData, last_message()))),
        ffi::PRG_ERR_UNSUPPORTED => Err(IgraphError::Unsupported(unsupported_static(&last_message()))),
        _ => Err(IgraphError::Internal("unknown status from the GPU library")),
    }
}

fn directed(g: &Graph) -> i32 {
    i32::from(g.is_directed())
}

/// `pagerank()`: damping 0.85, successive L1 change < 1e-10, at most 1000
/// iterations, in FP64 on the GPU.
pub fn pagerank(graph: &Graph) -> IgraphResult<Vec<f64>> {
    let n = graph.vcount();
    let (f, t) = edges(graph)?;
    let mut out = vec![0.0; n as usize];
    // SAFETY: f and t hold m ids each and out holds n doubles.
    check(unsafe { ffi::prg_pagerank(n, f.len() as u64, f.as_ptr(), t.as_ptr(), directed(graph), out.as_mut_ptr()) })?;
    Ok(out)
}

/// `pagerank_weighted()`: weights in edge-id order, validated by the library
/// with the reference's messages (length, NaN, negative, infinite).
pub fn pagerank_weighted(graph: &Graph, weights: &[f64]) -> IgraphResult<Vec<f64>> {
    let n = graph.vcount();
    let (f, t) = edges(graph)?;
    let mut out = vec![0.0; n as usize];
    // SAFETY: weights holds weights.len() doubles, as passed.
    check(unsafe {
        ffi::prg_pagerank_weighted(
            n, f.len() as u64, f.as_ptr(), t.as_ptr(), directed(graph), weights.as_ptr(), weights.len() as u64,
            out.as_mut_ptr(),
        )
    })?;
    Ok(out)
}

/// `personalized_pagerank()`: reset of length vcount (normalised inside),
/// damping in (0, 1).
pub fn personalized_pagerank(graph: &Graph, reset: &[f64], damping: f64) -> IgraphResult<Vec<f64>> {
    let n = graph.vcount();
    let (f, t) = edges(graph)?;
    let mut out = vec![0.0; n as usize];
    // SAFETY: reset holds reset.len() doubles, as passed.
    check(unsafe {
        ffi::prg_personalized_pagerank(
            n, f.len() as u64, f.as_ptr(), t.as_ptr(), directed(graph), reset.as_ptr(), reset.len() as u64,
            damping, out.as_mut_ptr(),
        )
    })?;
    Ok(out)
}

/// `personalized_pagerank_default()`: damping 0.85.
pub fn personalized_pagerank_default(graph: &Graph, reset: &[f64]) -> IgraphResult<Vec<f64>> {
    personalized_pagerank(graph, reset, 0.85)
}

/// `personalized_pagerank_vs()`: uniform reset over the ids (duplicates add
/// weight).
pub fn personalized_pagerank_vs(graph: &Graph, reset_vids: &[u32], damping: f64) -> IgraphResult<Vec<f64>> {
    let n = graph.vcount();
    let (f, t) = edges(graph)?;
    let mut out = vec![0.0; n as usize];
    // SAFETY: reset_vids holds reset_vids.len() ids, as passed.
    check(unsafe {
        ffi::prg_personalized_pagerank_vs(
            n, f.len() as u64, f.as_ptr(), t.as_ptr(), directed(graph), reset_vids.as_ptr(),
            reset_vids.len() as u64, damping, out.as_mut_ptr(),
        )
    })?;
    Ok(out)
}

/// `pagerank_linsys()`: the same fixed point as a linear system, solved to
/// ||b - Ax||_2 < 1e-13 ||b||_2 from the uniform start.
pub fn pagerank_linsys(graph: &Graph) -> IgraphResult<Vec<f64>> {
    let n = graph.vcount();
    let (f, t) = edges(graph)?;
    let mut out = vec![0.0; n as usize];
    // SAFETY: as for pagerank.
    check(unsafe {
        ffi::prg_pagerank_linsys(n, f.len() as u64, f.as_ptr(), t.as_ptr(), directed(graph), out.as_mut_ptr())
    })?;
    Ok(out)
}

/// `eigenvector_centrality()` (undirected, unweighted).
pub fn eigenvector_centrality(graph: &Graph) -> IgraphResult<Vec<f64>> {
    let n = graph.vcount();
    let (f, t) = edges(graph)?;
    let mut out = vec![0.0; n as usize];
    // SAFETY: out holds n doubles; the eigenvalue is optional.
    check(unsafe {
        ffi::prg_eigenvector_centrality(
            n, f.len() as u64, f.as_ptr(), t.as_ptr(), directed(graph), out.as_mut_ptr(), std::ptr::null_mut(),
        )
    })?;
    Ok(out)
}

/// `eigenvector_centrality_weighted()` (undirected; signed rules for
/// negative weights).
pub fn eigenvector_centrality_weighted(graph: &Graph, weights: &[f64]) -> IgraphResult<EigenvectorScores> {
    let n = graph.vcount();
    let (f, t) = edges(graph)?;
    let mut vector = vec![0.0; n as usize];
    let mut eigenvalue = 0.0;
    // SAFETY: weights holds weights.len() doubles; vector holds n.
    check(unsafe {
        ffi::prg_eigenvector_centrality_weighted(
            n, f.len() as u64, f.as_ptr(), t.as_ptr(), directed(graph), weights.as_ptr(), weights.len() as u64,
            vector.as_mut_ptr(), &mut eigenvalue,
        )
    })?;
    Ok(EigenvectorScores { vector, eigenvalue })
}

/// `eigenvector_centrality_full()`; `_directed` and `_directed_weighted`
/// are its cases.
pub fn eigenvector_centrality_full(
    graph: &Graph,
    mode: EigenvectorMode,
    weights: Option<&[f64]>,
) -> IgraphResult<EigenvectorScores> {
    let n = graph.vcount();
    let (f, t) = edges(graph)?;
    let mut vector = vec![0.0; n as usize];
    let mut eigenvalue = 0.0;
    let m = match mode {
        EigenvectorMode::Out => ffi::PRG_EIG_OUT,
        EigenvectorMode::In => ffi::PRG_EIG_IN,
        EigenvectorMode::All => ffi::PRG_EIG_ALL,
    };
    let (wp, wl) = weights.map_or((std::ptr::null(), 0), |w| (w.as_ptr(), w.len() as u64));
    // SAFETY: wp is null or holds wl doubles; vector holds n.
    check(unsafe {
        ffi::prg_eigenvector_centrality_full(
            n, f.len() as u64, f.as_ptr(), t.as_ptr(), directed(graph), m, wp, wl, vector.as_mut_ptr(),
            &mut eigenvalue,
        )
    })?;
    Ok(EigenvectorScores { vector, eigenvalue })
}

pub fn eigenvector_centrality_directed(graph: &Graph, mode: EigenvectorMode) -> IgraphResult<EigenvectorScores> {
    eigenvector_centrality_full(graph, mode, None)
}

pub fn eigenvector_centrality_directed_weighted(
    graph: &Graph,
    mode: EigenvectorMode,
    weights: &[f64],
) -> IgraphResult<EigenvectorScores> {
    eigenvector_centrality_full(graph, mode, Some(weights))
}

/// `hub_and_authority_scores()`.
pub fn hub_and_authority_scores(graph: &Graph) -> IgraphResult<HitsScores> {
    let n = graph.vcount();
    let (f, t) = edges(graph)?;
    let mut hub = vec![0.0; n as usize];
    let mut authority = vec![0.0; n as usize];
    let mut eigenvalue = 0.0;
    // SAFETY: hub and authority hold n doubles each.
    check(unsafe {
        ffi::prg_hub_and_authority_scores(
            n, f.len() as u64, f.as_ptr(), t.as_ptr(), directed(graph), hub.as_mut_ptr(), authority.as_mut_ptr(),
            &mut eigenvalue,
        )
    })?;
    Ok(HitsScores { hub, authority, eigenvalue })
}

/// `hub_and_authority_scores_weighted()`.
pub fn hub_and_authority_scores_weighted(graph: &Graph, weights: &[f64]) -> IgraphResult<HitsScores> {
    let n = graph.vcount();
    let (f, t) = edges(graph)?;
    let mut hub = vec![0.0; n as usize];
    let mut authority = vec![0.0; n as usize];
    let mut eigenvalue = 0.0;
    // SAFETY: weights holds weights.len() doubles; hub and authority hold n.
    check(unsafe {
        ffi::prg_hub_and_authority_scores_weighted(
            n, f.len() as u64, f.as_ptr(), t.as_ptr(), directed(graph), weights.as_ptr(), weights.len() as u64,
            hub.as_mut_ptr(), authority.as_mut_ptr(), &mut eigenvalue,
        )
    })?;
    Ok(HitsScores { hub, authority, eigenvalue })
}

/// Node flows of Infomap's flow model (community/infomap.rs:233-355, the
/// private `power_iteration_pagerank`): `build_flow_state` would call this in
/// place of its own loop.
pub fn infomap_node_flow(graph: &Graph, edge_weights: Option<&[f64]>, vertex_weights: Option<&[f64]>)
-> IgraphResult<Vec<f64>> {
    let n = graph.vcount();
    let (f, t) = edges(graph)?;
    let mut flow = vec![0.0; n as usize];
    let (ep, el) = edge_weights.map_or((std::ptr::null(), 0), |w| (w.as_ptr(), w.len() as u64));
    let (vp, vl) = vertex_weights.map_or((std::ptr::null(), 0), |w| (w.as_ptr(), w.len() as u64));
    // SAFETY: ep / vp are null or hold el / vl doubles; flow holds n.
    check(unsafe {
        ffi::prg_infomap_flow(
            n, f.len() as u64, f.as_ptr(), t.as_ptr(), directed(graph), ep, el, vp, vl, flow.as_mut_ptr(),
            std::ptr::null_mut(),
        )
    })?;
    Ok(flow)
}

/// `read_edgelist()` with the parsing on the GPU: the same accepted texts,
/// the same first failing line and message.
pub fn read_edgelist<R: std::io::Read>(mut input: R) -> IgraphResult<Graph> {
    let mut text = Vec::new();
    input.read_to_end(&mut text)?;
    let cap = text.iter().filter(|&&b| b == b'\n').count() + 1;
    let mut f = vec![0u32; cap];
    let mut t = vec![0u32; cap];
    let (mut m, mut n, mut line) = (0u64, 0u32, 0u64);
    // SAFETY: f and t hold cap ids each, as passed.
    let rc = unsafe {
        ffi::prg_parse_edgelist(
            text.as_ptr() as *const _, text.len() as u64, f.as_mut_ptr(), t.as_mut_ptr(), cap as u64, &mut m,
            &mut n, &mut line,
        )
    };
    if rc == ffi::PRG_ERR_PARSE {
        return Err(IgraphError::Parse { line: line as usize, message: last_message() });
    }
    check(rc)?;
    let m = m as usize;
    let mut g = Graph::with_vertices(n);
    g.add_edges(f[..m].iter().copied().zip(t[..m].iter().copied()))?;
    Ok(g)
}

/// The method forms of rust-igraph's `Graph` (src/core/graph.rs:1857-1859,
/// 5454-5456, 6285-6289, 7002-7004), delegating to the free functions.
pub trait PageRankExt {
    fn pagerank(&self) -> IgraphResult<Vec<f64>>;
    fn pagerank_weighted(&self, weights: &[f64]) -> IgraphResult<Vec<f64>>;
    /// `personalized_pagerank_default`: damping 0.85.
    fn personalized_pagerank(&self, reset: &[f64]) -> IgraphResult<Vec<f64>>;
    fn pagerank_linsys(&self) -> IgraphResult<Vec<f64>>;
}

impl PageRankExt for Graph {
    fn pagerank(&self) -> IgraphResult<Vec<f64>> {
        pagerank(self)
    }
    fn pagerank_weighted(&self, weights: &[f64]) -> IgraphResult<Vec<f64>> {
        pagerank_weighted(self, weights)
    }
    fn personalized_pagerank(&self, reset: &[f64]) -> IgraphResult<Vec<f64>> {
        personalized_pagerank_default(self, reset)
    }
    fn pagerank_linsys(&self) -> IgraphResult<Vec<f64>> {
        pagerank_linsys(self)
    }
}

/// Solver options of a resident graph (`prg_options`).
#[derive(Clone, Copy, Debug)]
pub struct Options {
    pub damping: f64,
    pub eps: f64,
    pub max_iter: u32,
    /// `PRG_PRECISION_*`
    pub precision: i32,
    /// `PRG_STOP_*`
    pub stop: i32,
    pub normalise: bool,
}

impl Default for Options {
    /// The reference's constants: d = 0.85, eps = 1e-10, 1000 iterations,
    /// FP64, successive-change stop.
    fn default() -> Self {
        Options {
            damping: 0.85,
            eps: 1e-10,
            max_iter: 1000,
            precision: ffi::PRG_PRECISION_FP64,
            stop: ffi::PRG_STOP_SUCCESSIVE,
            normalise: true,
        }
    }
}

impl Options {
    fn to_c(self, start: *const f64) -> ffi::prg_options {
        ffi::prg_options {
            damping: self.damping,
            eps: self.eps,
            max_iter: self.max_iter,
            precision: self.precision,
            stop: self.stop,
            normalise: i32::from(self.normalise),
            start,
            inner: ffi::PRG_INNER_KRYLOV,
        }
    }
}

/// What one solve did (`prg_stats`).
pub type SolveStats = ffi::prg_stats;

/// A graph built once in GPU memory and solved many times.  One handle owns
/// one CUDA stream; it is `Send` but not `Sync`, like rust-igraph's `Graph`.
pub struct DeviceGraph {
    h: *mut ffi::prg_graph,
    n: u32,
}

// SAFETY: a handle may move between threads; the library serialises work on
// the handle's own stream.  It is not Sync: one thread at a time.
unsafe impl Send for DeviceGraph {}

impl DeviceGraph {
    /// Builds the device CSR from a rust-igraph graph (and optional weights
    /// in edge-id order).
    pub fn new(graph: &Graph, weights: Option<&[f64]>) -> IgraphResult<Self> {
        let n = graph.vcount();
        let (f, t) = edges(graph)?;
        if let Some(w) = weights {
            if w.len() != f.len() {
                return Err(IgraphError::InvalidArgument(format!(
                    "weights length {} must equal ecount {}",
                    w.len(),
                    f.len()
                )));
            }
        }
        let wp = weights.map_or(std::ptr::null(), |w| w.as_ptr());
        let mut h = std::ptr::null_mut();
        // SAFETY: f, t (and weights) hold m entries; h receives the handle.
        check(unsafe { ffi::prg_graph_create(n, f.len() as u64, f.as_ptr(), t.as_ptr(), wp, directed(graph), &mut h) })?;
        Ok(DeviceGraph { h, n })
    }

    /// Solves with `opts`; `reset` is a raw teleport vector (normalised
    /// inside) or None for the uniform one, `start` an optional start vector.
    pub fn solve(&mut self, opts: Options, reset: Option<&[f64]>, start: Option<&[f64]>)
    -> IgraphResult<(Vec<f64>, SolveStats)> {
        let n = self.n as usize;
        for v in [reset, start].into_iter().flatten() {
            if v.len() != n {
                return Err(IgraphError::InvalidArgument(format!("vector length {} must equal vcount {n}", v.len())));
            }
        }
        let c = opts.to_c(start.map_or(std::ptr::null(), |s| s.as_ptr()));
        let mut out = vec![0.0; n];
        let mut st = SolveStats::default();
        // SAFETY: reset / start are null or hold n doubles; out holds n.
        check(unsafe {
            ffi::prg_solve(self.h, &c, reset.map_or(std::ptr::null(), |r| r.as_ptr()), out.as_mut_ptr(), &mut st)
        })?;
        Ok((out, st))
    }

    /// The allocation-free FP64 solve (`prg_solve_noalloc`) for callers that
    /// must not allocate device memory while they solve.
    ///
    /// # Safety
    /// `d_reset` (null or n doubles, normalised) and `d_out` (n doubles) must
    /// be device memory of the graph's GPU; calls must not overlap.
    pub unsafe fn solve_noalloc(&mut self, opts: Options, d_reset: *const f64, d_out: *mut f64)
    -> IgraphResult<SolveStats> {
        let c = opts.to_c(std::ptr::null());
        let mut st = SolveStats::default();
        // SAFETY: the caller upholds the pointer contract above.
        check(unsafe { ffi::prg_solve_noalloc(self.h, &c, d_reset, d_out, &mut st) })?;
        Ok(st)
    }

    pub fn vcount(&self) -> u32 {
        self.n
    }
}

impl Drop for DeviceGraph {
    fn drop(&mut self) {
        // SAFETY: h came from prg_graph_create and is destroyed once.
        unsafe { ffi::prg_graph_destroy(self.h) };
    }
}
