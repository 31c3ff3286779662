// api.cu — the extern "C" boundary (include/prg_b200.h).
//
// Validation order and messages follow rust-igraph so a binding can hand
// the status/message pair straight to IgraphError:
//   pagerank            pagerank.rs:52-101
//   pagerank_weighted   pagerank_weighted.rs:52-79
//   personalized        personalized_pagerank.rs:65-107
//   _vs                 personalized_pagerank.rs:241-268
// There is no CPU fallback: every solve runs the CUDA kernels, and a missing
// or unusable GPU is reported as PRG_ERR_CUDA.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/prg_b200.h"
#include "autotune.cuh"
#include "gnn.cuh"
#include "graph.cuh"
#include "edgelist.cuh"
#include "eigen.cuh"
#include "handle.cuh"
#include "ppr_batch.cuh"
#include "solver.cuh"

namespace {

thread_local std::string g_err;

int32_t fail(int32_t code, const std::string &msg) {
    g_err = msg;
    return code;
}

}  // namespace

namespace prg {
// Lets entry points defined in other files report through prg_last_error().
void set_last_error(const std::string &msg) { g_err = msg; }
}  // namespace prg

namespace {

int32_t from_cuda(const prg::CudaError &e) {
    if (e.err == cudaErrorMemoryAllocation) return fail(PRG_ERR_OUT_OF_MEMORY, "cuda: out of memory");
    return fail(PRG_ERR_CUDA, std::string("cuda: ") + cudaGetErrorString(e.err) + " (" + e.what + ")");
}

// Display of an f64 the way Rust's `{}` formats it: shortest round-trip
// digits, never exponent notation, "NaN"/"inf"/"-inf".
std::string rust_f64(double v) {
    if (std::isnan(v)) return "NaN";
    if (std::isinf(v)) return v > 0 ? "inf" : "-inf";
    char buf[64];
    int prec = 1;
    for (; prec <= 17; prec++) {
        std::snprintf(buf, sizeof buf, "%.*e", prec - 1, v);
        if (std::strtod(buf, nullptr) == v) break;
    }
    // buf = d.ddddde[+-]XX ; expand to plain decimal
    std::string s(buf);
    bool neg = false;
    if (s[0] == '-') {
        neg = true;
        s = s.substr(1);
    }
    size_t epos = s.find('e');
    int ex = std::atoi(s.c_str() + epos + 1);
    std::string digits;
    for (size_t i = 0; i < epos; i++)
        if (s[i] != '.') digits += s[i];
    while (digits.size() > 1 && digits.back() == '0') digits.pop_back();
    std::string out;
    int point = ex + 1;  // digits before the decimal point
    if (point <= 0) {
        out = "0." + std::string(-point, '0') + digits;
    } else if ((size_t)point >= digits.size()) {
        out = digits + std::string(point - digits.size(), '0');
    } else {
        out = digits.substr(0, point) + "." + digits.substr(point);
    }
    if (v == 0.0) out = "0";
    return (neg ? "-" : "") + out;
}

bool ensure_pool_config() {
    static bool done = false;
    if (done) return true;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return false;
    cudaMemPool_t pool;
    if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        uint64_t thr = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
    }
    done = true;
    return true;
}

// Checks that every endpoint is < n (Graph::add_edges rejects others with
// IgraphError::VertexOutOfRange, graph.rs:756-785).
__global__ void max_endpoint_kernel(const uint32_t *a, const uint32_t *b, uint64_t m, uint32_t *out) {
    uint32_t mx = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < m; i += (uint64_t)gridDim.x * blockDim.x)
        mx = max(mx, max(a[i], b[i]));
    for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, mx);
}

// Size checks shared by both ways of creating a handle.
static int32_t check_sizes(uint32_t n, uint64_t m, int32_t directed) {
    if (m > 0xFFFFFFFFull) return fail(PRG_ERR_INTERNAL, "ecount overflows u32");
    const uint64_t arcs = directed ? m : 2 * m;
    if (arcs + prg::kColPad >= 0xFFFFFFFFull)
        return fail(PRG_ERR_INTERNAL, "arc count exceeds the u32 CSR index range");
    if (n >= prg::kChunkFlag) return fail(PRG_ERR_INTERNAL, "vertex count exceeds 2^31 - 1");
    return PRG_OK;
}

// A handle with the process-wide tuning applied and nothing built yet.
static prg_graph *new_handle(uint32_t n, uint64_t m, int32_t directed, cudaStream_t s, int relabel) {
    prg_graph *h = new prg_graph();
    h->stream = s;
    h->g.n = n;
    h->g.m = m;
    h->g.directed = directed != 0;
    const prg::Tuning &t = prg::tuning();
    h->g.capw = t.capw;
    h->g.shortmax = t.shortmax;
    h->g.split = t.split;
    h->g.blocks_per_sm = t.blocks_per_sm;
    h->g.relabel = relabel >= 0 ? relabel : t.relabel;
    h->g.hot_cache = t.hot_cache;
    h->g.hot_cache64 = t.hot_cache64;
    h->g.hot_threads = t.hot_threads;
    h->g.seg_kry32 = t.seg_kry32;
    h->g.seg_hot = t.seg_hot;
    h->g.seg_res64 = t.seg_res64;
    h->g.seg_hot64 = t.seg_hot64;
    h->g.seg_plain64 = t.seg_plain64;
    h->g.seg_eig64 = t.seg_eig64;
    h->g.seg_prefetch = t.seg_prefetch;
    h->g.seg_threads = t.seg_threads;
    h->g.seg_pipe = t.seg_pipe;
    h->g.l1_hot32 = t.l1_hot32;
    h->g.l1_hot64 = t.l1_hot64;
    h->ws.unroll = t.unroll;
    PRG_CUDA(cudaGetDevice(&h->g.device));
    return h;
}

static std::string range_message(uint32_t mx, uint32_t n) {
    return "vertex id " + std::to_string(mx) + " out of range (vcount = " + std::to_string(n) + ")";
}

// Creates a handle from device edge arrays (copies nothing on the host).
int32_t create_from_device(uint32_t n, uint64_t m, const uint32_t *d_from, const uint32_t *d_to, const double *d_w,
                           int32_t directed, cudaStream_t s, prg_graph **out, int relabel = -1) {
    const int32_t rc = check_sizes(n, m, directed);
    if (rc != PRG_OK) return rc;
    prg_graph *h = new_handle(n, m, directed, s, relabel);
    if (m > 0) {
        uint32_t *d_mx = nullptr, mx = 0;
        PRG_CUDA(cudaMallocAsync((void **)&d_mx, 4, s));
        PRG_CUDA(cudaMemsetAsync(d_mx, 0, 4, s));
        max_endpoint_kernel<<<148 * 8, 256, 0, s>>>(d_from, d_to, m, d_mx);
        PRG_CUDA(cudaGetLastError());
        PRG_CUDA(cudaMemcpyAsync(&mx, d_mx, 4, cudaMemcpyDeviceToHost, s));
        PRG_CUDA(cudaFreeAsync(d_mx, s));
        PRG_CUDA(cudaStreamSynchronize(s));
        if (mx >= n) {
            delete h;
            return fail(PRG_ERR_VERTEX_OUT_OF_RANGE, range_message(mx, n));
        }
    }
    prg::build_graph(h->g, d_from, d_to, d_w, s);
    *out = h;
    return PRG_OK;
}

void destroy(prg_graph *h);

int32_t create_from_host(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to, const double *w,
                         int32_t directed, prg_graph **out, int relabel = -1) {
    if (!ensure_pool_config()) return fail(PRG_ERR_CUDA, "cuda: no usable device");
    cudaStream_t s;
    PRG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    if (m > 0xFFFFFFFFull) {
        cudaStreamDestroy(s);
        return fail(PRG_ERR_INTERNAL, "ecount overflows u32");
    }
    if (m >= prg::kStreamMinEdges && !(w && directed)) {
        // large edge lists: chunked copies overlapped with the build
        int32_t rc = check_sizes(n, m, directed);
        if (rc == PRG_OK) {
            prg_graph *h = new_handle(n, m, directed, s, relabel);
            uint32_t mx = 0;
            bool ok = false;
            try {
                ok = prg::build_graph_host(h->g, from, to, w, s, &mx);
            } catch (...) {
                destroy(h);
                throw;
            }
            if (ok) {
                *out = h;
                return PRG_OK;
            }
            destroy(h);  // what was built, and the stream
            return fail(PRG_ERR_VERTEX_OUT_OF_RANGE, range_message(mx, n));
        }
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
        return rc;
    }
    uint32_t *d_f = nullptr, *d_t = nullptr;
    double *d_w = nullptr;
    const uint64_t mm = m ? m : 1;
    PRG_CUDA(cudaMallocAsync((void **)&d_f, mm * 4, s));
    PRG_CUDA(cudaMallocAsync((void **)&d_t, mm * 4, s));
    if (m) {
        PRG_CUDA(cudaMemcpyAsync(d_f, from, m * 4, cudaMemcpyHostToDevice, s));
        PRG_CUDA(cudaMemcpyAsync(d_t, to, m * 4, cudaMemcpyHostToDevice, s));
    }
    if (w) {
        PRG_CUDA(cudaMallocAsync((void **)&d_w, mm * 8, s));
        if (m) PRG_CUDA(cudaMemcpyAsync(d_w, w, m * 8, cudaMemcpyHostToDevice, s));
    }
    int32_t rc = create_from_device(n, m, d_f, d_t, w ? d_w : nullptr, directed, s, out, relabel);
    cudaFreeAsync(d_f, s);
    cudaFreeAsync(d_t, s);
    if (d_w) cudaFreeAsync(d_w, s);
    if (rc != PRG_OK) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
    }
    return rc;
}

// Set-up for a handle returned to the caller: the allocation-free solve's
// scratch and kernels are loaded now, while allocating is allowed.  A
// failure destroys the handle and propagates.
static void prepare_handle(prg_graph *&h) {
    try {
        prg::noalloc_prepare(h->g);
    } catch (...) {
        cudaStreamSynchronize(h->stream);
        destroy(h);
        h = nullptr;
        throw;
    }
}

void destroy(prg_graph *h) {
    if (!h) return;
    cudaStream_t s = h->stream;
    prg::workspace_free(h->ws, s);
    auto f = [&](void *p) {
        if (p) cudaFreeAsync(p, s);
    };
    f(h->g.row_ptr);
    f(h->g.col);
    f(h->g.w64);
    f(h->g.w32);
    f(h->g.deg);
    f(h->g.dval);
    f(h->g.inv32);
    f(h->g.rb);
    f(h->g.hubs);
    f(h->g.perm);
    f(h->g.iperm);
    f(h->d_reset);
    f(h->d_out);
    f(h->d_start);
    cudaStreamSynchronize(s);
    cudaStreamDestroy(s);
    delete h;
}

prg::SolveOpts to_solve_opts(const prg_options *o) {
    prg::SolveOpts so;
    so.refine_switch = prg::tuning().refine_switch;
    if (o) {
        so.damping = o->damping;
        so.eps = o->eps;
        so.max_iter = o->max_iter;
        so.precision = o->precision;
        so.inner = o->inner;
        so.stop = o->stop;
        so.normalise = o->normalise;
    }
    return so;
}

void fill_stats(prg_stats *st, const prg::SolveStats &s, const prg_graph *h) {
    if (!st) return;
    std::memset(st, 0, sizeof(*st));
    st->iterations = s.iterations;
    st->fp64_passes = s.fp64_passes;
    st->fp32_passes = s.fp32_passes;
    st->residual_passes = s.residual_passes;
    st->last_diff = s.last_diff;
    st->residual_l1 = s.residual_l1;
    st->error_bound = s.error_bound;
    st->solve_ms = s.solve_ms;
    st->build_ms = h->g.build_ms;
    st->arcs = h->g.arcs;
    st->n_dangling = h->g.n_dangling;
    st->kernel_launches = s.kernel_launches;
    st->fp32_ms = s.fp32_ms;
    st->fp64_ms = s.fp64_ms;
    st->spmv_ms = s.spmv_ms;
    st->spmv_launches = s.spmv_launches;
}

// Host-side solve: stages the (already normalised) reset and start vectors,
// runs, copies the result into `out`.
int32_t solve_host(prg_graph *h, const prg::SolveOpts &so_in, const double *norm_reset, const double *start,
                   double *out, prg_stats *st) {
    cudaStream_t s = h->stream;
    const uint64_t n = h->g.n;
    prg::SolveOpts so = so_in;
    if (!h->d_out) PRG_CUDA(cudaMallocAsync((void **)&h->d_out, n * 8, s));
    const double *d_t = nullptr;
    if (norm_reset) {
        if (!h->d_reset) PRG_CUDA(cudaMallocAsync((void **)&h->d_reset, n * 8, s));
        PRG_CUDA(cudaMemcpyAsync(h->d_reset, norm_reset, n * 8, cudaMemcpyHostToDevice, s));
        d_t = h->d_reset;
    }
    if (start) {
        if (!h->d_start) PRG_CUDA(cudaMallocAsync((void **)&h->d_start, n * 8, s));
        PRG_CUDA(cudaMemcpyAsync(h->d_start, start, n * 8, cudaMemcpyHostToDevice, s));
        so.d_start = h->d_start;
    }
    prg::SolveStats ss;
    prg::solve(h->g, h->ws, so, d_t, h->d_out, ss, s);
    PRG_CUDA(cudaMemcpyAsync(out, h->d_out, n * 8, cudaMemcpyDeviceToHost, s));
    PRG_CUDA(cudaStreamSynchronize(s));
    fill_stats(st, ss, h);
    return PRG_OK;
}

int32_t check_options(const prg_options &o) {
    if (o.precision < PRG_PRECISION_FP64 || o.precision > PRG_PRECISION_LINSYS)
        return fail(PRG_ERR_INVALID_ARGUMENT, "unknown precision " + std::to_string(o.precision));
    if (o.inner != PRG_INNER_KRYLOV && o.inner != PRG_INNER_RICHARDSON)
        return fail(PRG_ERR_INVALID_ARGUMENT, "unknown inner solver " + std::to_string(o.inner));
    if (o.stop != PRG_STOP_SUCCESSIVE && o.stop != PRG_STOP_ERROR_BOUND)
        return fail(PRG_ERR_INVALID_ARGUMENT, "unknown stop rule " + std::to_string(o.stop));
    if (!(o.eps > 0.0)) return fail(PRG_ERR_INVALID_ARGUMENT, "eps must be positive (got " + rust_f64(o.eps) + ")");
    return PRG_OK;
}

// One-shot drop-in: build, solve with the reference's constants, download.
int32_t dropin(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to, int32_t directed, const double *w,
               const double *norm_reset, double damping, double *out, int precision = PRG_PRECISION_FP64) {
    prg_graph *h = nullptr;
    int32_t rc = create_from_host(n, m, from, to, w, directed, &h);
    if (rc != PRG_OK) return rc;
    prg::SolveOpts so;
    so.damping = damping;
    so.precision = precision;
    try {
        rc = solve_host(h, so, norm_reset, nullptr, out, nullptr);
    } catch (...) {
        destroy(h);
        throw;
    }
    destroy(h);
    return rc;
}

}  // namespace

#define PRG_GUARD_BEGIN try {
#define PRG_GUARD_END                                                   \
    }                                                                   \
    catch (const prg::CudaError &e) {                                   \
        return from_cuda(e);                                            \
    }                                                                   \
    catch (const std::bad_alloc &) {                                    \
        return fail(PRG_ERR_OUT_OF_MEMORY, "host: out of memory");      \
    }                                                                   \
    catch (...) {                                                       \
        return fail(PRG_ERR_INTERNAL, "unexpected exception");          \
    }

extern "C" {

void prg_default_options(prg_options *o) {
    if (!o) return;
    o->damping = 0.85;
    o->eps = 1e-10;
    o->max_iter = 1000;
    o->precision = PRG_PRECISION_FP64;
    o->stop = PRG_STOP_SUCCESSIVE;
    o->normalise = 1;
    o->start = nullptr;
    o->inner = PRG_INNER_KRYLOV;
}

const char *prg_last_error(void) { return g_err.c_str(); }

uint64_t prg_last_error_len(void) { return g_err.size(); }

int32_t prg_pagerank(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to, int32_t directed,
                     double *out) {
    g_err.clear();
    PRG_GUARD_BEGIN
    if (n == 0) return PRG_OK;  // pagerank.rs:55-57
    if (n == 1) {               // pagerank.rs:58-60
        out[0] = 1.0;
        return PRG_OK;
    }
    return dropin(n, m, from, to, directed, nullptr, nullptr, 0.85, out);
    PRG_GUARD_END
}

int32_t prg_eigenvector_centrality(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to, int32_t directed,
                                   double *out, double *eigenvalue) {
    g_err.clear();
    PRG_GUARD_BEGIN
    if (eigenvalue) *eigenvalue = 0.0;
    if (directed)  // eigenvector.rs:118-123
        return fail(PRG_ERR_UNSUPPORTED,
                    "directed eigenvector_centrality \xe2\x80\x94 use eigenvector_centrality_directed or _full");
    if (n == 0) return PRG_OK;
    if (m == 0 || n == 1) {  // eigenvector.rs:296-307: ones, eigenvalue 0
        for (uint32_t i = 0; i < n; i++) out[i] = 1.0;
        return PRG_OK;
    }
    prg_graph *h = nullptr;
    int32_t rc = create_from_host(n, m, from, to, nullptr, 0, &h);
    if (rc != PRG_OK) return rc;
    try {
        cudaStream_t s = h->stream;
        if (!h->d_out) PRG_CUDA(cudaMallocAsync((void **)&h->d_out, (uint64_t)n * 8, s));
        const prg::eig::Result r = prg::eig::eigenvector_centrality(h->g, h->ws, h->d_out, s);
        PRG_CUDA(cudaMemcpyAsync(out, h->d_out, (uint64_t)n * 8, cudaMemcpyDeviceToHost, s));
        PRG_CUDA(cudaStreamSynchronize(s));
        if (eigenvalue) *eigenvalue = r.eigenvalue;
    } catch (...) {
        destroy(h);
        throw;
    }
    destroy(h);
    return PRG_OK;
    PRG_GUARD_END
}

int32_t prg_hub_and_authority_scores(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to,
                                     int32_t directed, double *hub, double *authority, double *eigenvalue) {
    g_err.clear();
    PRG_GUARD_BEGIN
    if (eigenvalue) *eigenvalue = 0.0;
    if (n == 0) return PRG_OK;
    if (!directed) {
        // hits.rs:131-141: eigenvector centrality, eigenvalue = (x.Ax / x.x)^2
        double lam = 0.0;
        int32_t rc = prg_eigenvector_centrality(n, m, from, to, 0, hub, &lam);
        if (rc != PRG_OK) return rc;
        if (n == 1 && m > 0) lam = 2.0 * (double)m;  // x = [1]; every edge is a loop seen twice
        for (uint32_t i = 0; i < n; i++) authority[i] = hub[i];
        if (eigenvalue) *eigenvalue = lam * lam;
        return PRG_OK;
    }
    if (m == 0) {  // hits.rs:144-150
        for (uint32_t i = 0; i < n; i++) hub[i] = authority[i] = 1.0;
        return PRG_OK;
    }
    prg_graph *g = nullptr, *rev = nullptr;
    int32_t rc = create_from_host(n, m, from, to, nullptr, 1, &g, 0);
    if (rc != PRG_OK) return rc;
    rc = create_from_host(n, m, to, from, nullptr, 1, &rev, 0);
    if (rc != PRG_OK) {
        destroy(g);
        return rc;
    }
    try {
        cudaStream_t s = g->stream;
        PRG_CUDA(cudaStreamSynchronize(rev->stream));  // rev's build runs on its own stream
        double *d_h = nullptr, *d_a = nullptr;
        PRG_CUDA(cudaMallocAsync((void **)&d_h, (uint64_t)n * 8, s));
        PRG_CUDA(cudaMallocAsync((void **)&d_a, (uint64_t)n * 8, s));
        const prg::eig::Result r = prg::eig::hits_directed(g->g, g->ws, rev->g, rev->ws, d_h, d_a, s);
        PRG_CUDA(cudaMemcpyAsync(hub, d_h, (uint64_t)n * 8, cudaMemcpyDeviceToHost, s));
        PRG_CUDA(cudaMemcpyAsync(authority, d_a, (uint64_t)n * 8, cudaMemcpyDeviceToHost, s));
        cudaFreeAsync(d_h, s);
        cudaFreeAsync(d_a, s);
        PRG_CUDA(cudaStreamSynchronize(s));
        if (eigenvalue) *eigenvalue = r.eigenvalue;
    } catch (...) {
        destroy(g);
        destroy(rev);
        throw;
    }
    destroy(g);
    destroy(rev);
    return PRG_OK;
    PRG_GUARD_END
}

// Weighted eigen variants; the checks come in the reference's order.  A
// negative weight switches the iterations to the reference's signed rules
// (signed pivot, no clamping, no DAG or zero-eigenvalue shortcut).
static bool any_negative(const double *w, uint64_t m) {
    for (uint64_t e = 0; e < m; e++)
        if (w[e] < 0.0) return true;
    return false;
}
static bool all_zero(const double *w, uint64_t m) {
    for (uint64_t e = 0; e < m; e++)
        if (w[e] != 0.0) return false;
    return true;
}

int32_t prg_eigenvector_centrality_weighted(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to,
                                            int32_t directed, const double *weights, uint64_t weights_len,
                                            double *out, double *eigenvalue) {
    g_err.clear();
    PRG_GUARD_BEGIN
    if (eigenvalue) *eigenvalue = 0.0;
    if (directed)  // eigenvector.rs:157-168
        return fail(PRG_ERR_UNSUPPORTED, "directed eigenvector_centrality_weighted \xe2\x80\x94 use "
                                         "eigenvector_centrality_directed_weighted");
    if (weights_len != m)  // eigenvector.rs:272-283
        return fail(PRG_ERR_INVALID_ARGUMENT, "weights vector length (" + std::to_string(weights_len) +
                                                  ") not equal to number of edges (" + std::to_string(m) + ")");
    if (n == 0) return PRG_OK;
    if (m == 0 || all_zero(weights, m) || n == 1) {  // eigenvector.rs:379-405
        for (uint32_t i = 0; i < n; i++) out[i] = 1.0;
        return PRG_OK;
    }
    prg::eig::EigOpts o;  // eigenvector.rs:375-538
    o.rowsum_seed = true;
    o.eps = 1e-12;
    o.negative = any_negative(weights, m);
    prg_graph *h = nullptr;
    int32_t rc = create_from_host(n, m, from, to, weights, 0, &h);
    if (rc != PRG_OK) return rc;
    try {
        cudaStream_t s = h->stream;
        if (!h->d_out) PRG_CUDA(cudaMallocAsync((void **)&h->d_out, (uint64_t)n * 8, s));
        const prg::eig::Result r = prg::eig::eigenvector_centrality(h->g, h->ws, h->d_out, s, o);
        PRG_CUDA(cudaMemcpyAsync(out, h->d_out, (uint64_t)n * 8, cudaMemcpyDeviceToHost, s));
        PRG_CUDA(cudaStreamSynchronize(s));
        if (eigenvalue) *eigenvalue = r.eigenvalue;
    } catch (...) {
        destroy(h);
        throw;
    }
    destroy(h);
    return PRG_OK;
    PRG_GUARD_END
}

int32_t prg_eigenvector_centrality_full(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to,
                                        int32_t directed, int32_t mode, const double *weights, uint64_t weights_len,
                                        double *out, double *eigenvalue) {
    g_err.clear();
    PRG_GUARD_BEGIN
    if (eigenvalue) *eigenvalue = 0.0;
    if (weights && weights_len != m)  // eigenvector.rs:272-283
        return fail(PRG_ERR_INVALID_ARGUMENT, "weights vector length (" + std::to_string(weights_len) +
                                                  ") not equal to number of edges (" + std::to_string(m) + ")");
    if (mode < PRG_EIG_OUT || mode > PRG_EIG_ALL) return fail(PRG_ERR_INVALID_ARGUMENT, "unknown eigenvector mode");
    if (!directed) {  // eigenvector.rs:252-264: undirected input takes the symmetric path
        if (weights) return prg_eigenvector_centrality_weighted(n, m, from, to, 0, weights, m, out, eigenvalue);
        return prg_eigenvector_centrality(n, m, from, to, 0, out, eigenvalue);
    }
    if (n == 0) return PRG_OK;
    const bool all = mode == PRG_EIG_ALL;
    if (m == 0 || (all && n == 1) || (weights && all_zero(weights, m))) {
        for (uint32_t i = 0; i < n; i++) out[i] = 1.0;
        return PRG_OK;
    }
    const bool neg = weights && any_negative(weights, m);
    // Out walks the in-edges of v: the graph's own in-CSR.  In, and All on a
    // directed graph (graph.neighbors / incident give out-edges there), walk
    // the out-edges: the in-CSR of the reversed graph.
    const bool reverse = mode != PRG_EIG_OUT;
    prg_graph *h = nullptr;
    int32_t rc = create_from_host(n, m, reverse ? to : from, reverse ? from : to, weights, 1, &h);
    if (rc != PRG_OK) return rc;
    try {
        cudaStream_t s = h->stream;
        if (!h->d_out) PRG_CUDA(cudaMallocAsync((void **)&h->d_out, (uint64_t)n * 8, s));
        prg::eig::Result r;
        if (!all) {
            r = prg::eig::eigenvector_directed(h->g, h->ws, h->d_out, s, neg);
        } else if (weights) {
            prg::eig::EigOpts o;  // eigenvector.rs:375-538
            o.rowsum_seed = true;
            o.eps = 1e-12;
            o.negative = neg;
            r = prg::eig::eigenvector_centrality(h->g, h->ws, h->d_out, s, o);
        } else {
            r = prg::eig::eigenvector_centrality(h->g, h->ws, h->d_out, s);  // eigenvector.rs:286-372
        }
        PRG_CUDA(cudaMemcpyAsync(out, h->d_out, (uint64_t)n * 8, cudaMemcpyDeviceToHost, s));
        PRG_CUDA(cudaStreamSynchronize(s));
        if (eigenvalue) *eigenvalue = r.eigenvalue;
    } catch (...) {
        destroy(h);
        throw;
    }
    destroy(h);
    return PRG_OK;
    PRG_GUARD_END
}

int32_t prg_hub_and_authority_scores_weighted(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to,
                                              int32_t directed, const double *weights, uint64_t weights_len,
                                              double *hub, double *authority, double *eigenvalue) {
    g_err.clear();
    PRG_GUARD_BEGIN
    if (eigenvalue) *eigenvalue = 0.0;
    if (weights_len != m)  // hits.rs:294-300
        return fail(PRG_ERR_INVALID_ARGUMENT, "weights length " + std::to_string(weights_len) +
                                                  " does not match edge count " + std::to_string(m));
    if (n == 0) return PRG_OK;
    if (m == 0 || all_zero(weights, m)) {  // hits.rs:310-332
        for (uint32_t i = 0; i < n; i++) hub[i] = authority[i] = 1.0;
        return PRG_OK;
    }
    const bool neg = any_negative(weights, m);
    if (!directed) {
        // hits.rs:334-341, 470-553: the weighted iteration with a signed
        // strength seed, eigenvalue (x.Wx / x.x)^2
        prg::eig::EigOpts o;
        o.rowsum_seed = true;
        o.signed_seed = true;
        o.eps = 1e-12;
        o.negative = neg;
        prg_graph *h = nullptr;
        int32_t rc = create_from_host(n, m, from, to, weights, 0, &h);
        if (rc != PRG_OK) return rc;
        try {
            cudaStream_t s = h->stream;
            if (!h->d_out) PRG_CUDA(cudaMallocAsync((void **)&h->d_out, (uint64_t)n * 8, s));
            const prg::eig::Result r = prg::eig::eigenvector_centrality(h->g, h->ws, h->d_out, s, o);
            PRG_CUDA(cudaMemcpyAsync(hub, h->d_out, (uint64_t)n * 8, cudaMemcpyDeviceToHost, s));
            PRG_CUDA(cudaStreamSynchronize(s));
            for (uint32_t i = 0; i < n; i++) authority[i] = hub[i];
            if (eigenvalue) *eigenvalue = r.eigenvalue * r.eigenvalue;
        } catch (...) {
            destroy(h);
            throw;
        }
        destroy(h);
        return PRG_OK;
    }
    prg_graph *g = nullptr, *rev = nullptr;
    int32_t rc = create_from_host(n, m, from, to, weights, 1, &g, 0);
    if (rc != PRG_OK) return rc;
    rc = create_from_host(n, m, to, from, weights, 1, &rev, 0);
    if (rc != PRG_OK) {
        destroy(g);
        return rc;
    }
    try {
        cudaStream_t s = g->stream;
        PRG_CUDA(cudaStreamSynchronize(rev->stream));
        double *d_h = nullptr, *d_a = nullptr;
        PRG_CUDA(cudaMallocAsync((void **)&d_h, (uint64_t)n * 8, s));
        PRG_CUDA(cudaMallocAsync((void **)&d_a, (uint64_t)n * 8, s));
        const prg::eig::Result r = prg::eig::hits_directed(g->g, g->ws, rev->g, rev->ws, d_h, d_a, s, neg);
        PRG_CUDA(cudaMemcpyAsync(hub, d_h, (uint64_t)n * 8, cudaMemcpyDeviceToHost, s));
        PRG_CUDA(cudaMemcpyAsync(authority, d_a, (uint64_t)n * 8, cudaMemcpyDeviceToHost, s));
        cudaFreeAsync(d_h, s);
        cudaFreeAsync(d_a, s);
        PRG_CUDA(cudaStreamSynchronize(s));
        if (eigenvalue) *eigenvalue = r.eigenvalue;
    } catch (...) {
        destroy(g);
        destroy(rev);
        throw;
    }
    destroy(g);
    destroy(rev);
    return PRG_OK;
    PRG_GUARD_END
}

int32_t prg_infomap_flow(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to, int32_t directed,
                         const double *edge_weights, uint64_t edge_weights_len, const double *vertex_weights,
                         uint64_t vertex_weights_len, double *node_flow, uint32_t *iterations) {
    g_err.clear();
    PRG_GUARD_BEGIN
    if (iterations) *iterations = 0;
    if (edge_weights) {  // infomap.rs:175-193
        if (edge_weights_len != m)
            return fail(PRG_ERR_INVALID_ARGUMENT, "edge weight vector length " + std::to_string(edge_weights_len) +
                                                      " does not match edge count " + std::to_string(m));
        for (uint64_t e = 0; e < m; e++) {
            const double w = edge_weights[e];
            if (w < 0.0 || !std::isfinite(w))
                return fail(PRG_ERR_INVALID_ARGUMENT, "edge weight[" + std::to_string(e) + "] = " + rust_f64(w) +
                                                          " is invalid (must be non-negative and finite)");
        }
    }
    std::vector<double> tele;
    if (vertex_weights) {  // infomap.rs:195-218
        if (vertex_weights_len != n)
            return fail(PRG_ERR_INVALID_ARGUMENT, "vertex weight vector length " +
                                                      std::to_string(vertex_weights_len) +
                                                      " does not match vertex count " + std::to_string(n));
        bool any = false;
        for (uint32_t i = 0; i < n; i++) {
            const double w = vertex_weights[i];
            if (w < 0.0 || !std::isfinite(w))
                return fail(PRG_ERR_INVALID_ARGUMENT,
                            "vertex weight[" + std::to_string(i) + "] = " + rust_f64(w) + " is invalid");
            any |= w > 0.0;
        }
        if (!any && n > 0) return fail(PRG_ERR_INVALID_ARGUMENT, "all vertex weights are zero");
        // infomap.rs:261-270: tele = vw / sum(vw), summed in index order
        double sum = 0.0;
        for (uint32_t i = 0; i < n; i++) sum += vertex_weights[i];
        tele.resize(n);
        for (uint32_t i = 0; i < n; i++) tele[i] = vertex_weights[i] / sum;
    }
    if (n == 0) return PRG_OK;
    if (n == 1) {  // infomap.rs:308-310
        node_flow[0] = 1.0;
        return PRG_OK;
    }
    prg_graph *h = nullptr;
    int32_t rc = create_from_host(n, m, from, to, edge_weights, directed, &h);
    if (rc != PRG_OK) return rc;
    double *d_t = nullptr, *d_ti = nullptr;
    try {
        cudaStream_t s = h->stream;
        if (!h->d_out) PRG_CUDA(cudaMallocAsync((void **)&h->d_out, (uint64_t)n * 8, s));
        if (!tele.empty()) {
            PRG_CUDA(cudaMallocAsync((void **)&d_t, (uint64_t)n * 8, s));
            PRG_CUDA(cudaMemcpyAsync(d_t, tele.data(), (uint64_t)n * 8, cudaMemcpyHostToDevice, s));
            if (h->g.perm) {
                PRG_CUDA(cudaMallocAsync((void **)&d_ti, (uint64_t)n * 8, s));
                prg::gather_f64(d_ti, d_t, h->g.perm, n, s);
            }
        }
        const prg::eig::Result r = prg::eig::infomap_flow(h->g, h->ws, d_ti ? d_ti : d_t, h->d_out, s);
        PRG_CUDA(cudaMemcpyAsync(node_flow, h->d_out, (uint64_t)n * 8, cudaMemcpyDeviceToHost, s));
        if (d_t) cudaFreeAsync(d_t, s);
        if (d_ti) cudaFreeAsync(d_ti, s);
        d_t = d_ti = nullptr;
        PRG_CUDA(cudaStreamSynchronize(s));
        if (iterations) *iterations = r.iterations;
    } catch (...) {
        if (d_t) cudaFreeAsync(d_t, h->stream);
        if (d_ti) cudaFreeAsync(d_ti, h->stream);
        destroy(h);
        throw;
    }
    destroy(h);
    return PRG_OK;
    PRG_GUARD_END
}

int32_t prg_pagerank_linsys(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to, int32_t directed,
                            double *out) {
    g_err.clear();
    PRG_GUARD_BEGIN
    if (n == 0) return PRG_OK;  // pagerank_linsys.rs:102-104
    if (n == 1) {               // pagerank_linsys.rs:105-107
        out[0] = 1.0;
        return PRG_OK;
    }
    return dropin(n, m, from, to, directed, nullptr, nullptr, 0.85, out, PRG_PRECISION_LINSYS);
    PRG_GUARD_END
}

int32_t prg_pagerank_weighted(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to, int32_t directed,
                              const double *weights, uint64_t weights_len, double *out) {
    g_err.clear();
    PRG_GUARD_BEGIN
    if (n == 0) return PRG_OK;  // pagerank_weighted.rs:55-57
    if (n == 1) {
        out[0] = 1.0;
        return PRG_OK;
    }
    if (weights_len != m)  // :62-68
        return fail(PRG_ERR_INVALID_ARGUMENT, "weights vector size (" + std::to_string(weights_len) +
                                                  ") differs from edge count (" + std::to_string(m) + ")");
    for (uint64_t e = 0; e < m; e++) {  // :69-76
        const double w = weights[e];
        if (std::isnan(w) || w < 0.0 || !std::isfinite(w))
            return fail(PRG_ERR_INVALID_ARGUMENT, "weight at edge " + std::to_string(e) +
                                                      " must be non-negative and finite (got " + rust_f64(w) + ")");
    }
    return dropin(n, m, from, to, directed, weights, nullptr, 0.85, out);
    PRG_GUARD_END
}

// personalized_pagerank.rs:65-111: validation, n==1, reset normalisation.
static int32_t ppr_validate(uint32_t n, const double *reset, uint64_t reset_len, double damping,
                            std::vector<double> &norm, bool *trivial) {
    *trivial = false;
    if (n == 0) {
        if (reset_len == 0) {
            *trivial = true;
            return PRG_OK;
        }
        return fail(PRG_ERR_INVALID_ARGUMENT,
                    "personalized_pagerank: reset vector non-empty but graph has no vertices");
    }
    if (reset_len != n)
        return fail(PRG_ERR_INVALID_ARGUMENT, "personalized_pagerank: reset length (" + std::to_string(reset_len) +
                                                  ") does not match vcount (" + std::to_string(n) + ")");
    if (damping <= 0.0 || damping >= 1.0)
        return fail(PRG_ERR_INVALID_ARGUMENT,
                    "personalized_pagerank: damping (" + rust_f64(damping) + ") must be in (0, 1)");
    double sum = 0.0;
    for (uint32_t i = 0; i < n; i++) sum += reset[i];
    if (sum <= 0.0)
        return fail(PRG_ERR_INVALID_ARGUMENT, "personalized_pagerank: reset vector must sum to a positive value");
    for (uint32_t i = 0; i < n; i++)
        if (reset[i] < 0.0)
            return fail(PRG_ERR_INVALID_ARGUMENT, "personalized_pagerank: negative reset value (" +
                                                      rust_f64(reset[i]) + ") at index " + std::to_string(i));
    if (n == 1) {
        *trivial = true;
        return PRG_OK;
    }
    const double inv = 1.0 / sum;
    norm.resize(n);
    for (uint32_t i = 0; i < n; i++) norm[i] = reset[i] * inv;
    return PRG_OK;
}

int32_t prg_personalized_pagerank(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to,
                                  int32_t directed, const double *reset, uint64_t reset_len, double damping,
                                  double *out) {
    g_err.clear();
    PRG_GUARD_BEGIN
    std::vector<double> norm;
    bool trivial = false;
    int32_t rc = ppr_validate(n, reset, reset_len, damping, norm, &trivial);
    if (rc != PRG_OK) return rc;
    if (trivial) {
        if (n == 1) out[0] = 1.0;
        return PRG_OK;
    }
    return dropin(n, m, from, to, directed, nullptr, norm.data(), damping, out);
    PRG_GUARD_END
}

int32_t prg_personalized_pagerank_vs(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to,
                                     int32_t directed, const uint32_t *reset_vids, uint64_t nvids, double damping,
                                     double *out) {
    g_err.clear();
    PRG_GUARD_BEGIN
    if (nvids == 0) return fail(PRG_ERR_INVALID_ARGUMENT, "reset_vids must not be empty");
    std::vector<double> reset(n, 0.0);
    const double weight = 1.0 / (double)nvids;
    for (uint64_t i = 0; i < nvids; i++) {
        const uint32_t v = reset_vids[i];
        if (v >= n)
            return fail(PRG_ERR_INVALID_ARGUMENT, "reset vertex " + std::to_string(v) + " out of range (vcount = " +
                                                      std::to_string(n) + ")");
        reset[v] += weight;
    }
    return prg_personalized_pagerank(n, m, from, to, directed, reset.data(), n, damping, out);
    PRG_GUARD_END
}

int32_t prg_graph_create(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to, const double *weights,
                         int32_t directed, prg_graph **out) {
    g_err.clear();
    PRG_GUARD_BEGIN
    if (!out) return fail(PRG_ERR_INVALID_ARGUMENT, "null output handle");
    *out = nullptr;
    if (weights) {
        for (uint64_t e = 0; e < m; e++) {
            const double w = weights[e];
            if (std::isnan(w) || w < 0.0 || !std::isfinite(w))
                return fail(PRG_ERR_INVALID_ARGUMENT, "weight at edge " + std::to_string(e) +
                                                          " must be non-negative and finite (got " + rust_f64(w) +
                                                          ")");
        }
    }
    const int32_t rc = create_from_host(n, m, from, to, weights, directed, out);
    if (rc == PRG_OK) prepare_handle(*out);
    return rc;
    PRG_GUARD_END
}

int32_t prg_graph_create_device(uint32_t n, uint64_t m, const uint32_t *d_from, const uint32_t *d_to,
                                const double *d_weights, int32_t directed, prg_graph **out) {
    g_err.clear();
    PRG_GUARD_BEGIN
    if (!out) return fail(PRG_ERR_INVALID_ARGUMENT, "null output handle");
    *out = nullptr;
    if (!ensure_pool_config()) return fail(PRG_ERR_CUDA, "cuda: no usable device");
    cudaStream_t s;
    PRG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    int32_t rc = create_from_device(n, m, d_from, d_to, d_weights, directed, s, out);
    if (rc != PRG_OK) cudaStreamDestroy(s);
    else prepare_handle(*out);
    return rc;
    PRG_GUARD_END
}

// Copies the text to the device and parses it there (edgelist.cu).  On
// success the result owns device edge arrays on stream s.
static int32_t edgelist_common(const char *text, uint64_t len, cudaStream_t s, prg::el::ParseResult &r,
                               uint64_t *err_line) {
    if (err_line) *err_line = 0;
    if (len && !text) return fail(PRG_ERR_INVALID_ARGUMENT, "null text");
    uint8_t *d_text = nullptr;
    if (len) {
        PRG_CUDA(cudaMallocAsync((void **)&d_text, len, s));
        PRG_CUDA(cudaMemcpyAsync(d_text, text, len, cudaMemcpyHostToDevice, s));
    }
    try {
        r = prg::el::parse(d_text, reinterpret_cast<const uint8_t *>(text), len, s);
    } catch (...) {
        if (d_text) cudaFreeAsync(d_text, s);
        throw;
    }
    if (d_text) cudaFreeAsync(d_text, s);
    if (r.status != PRG_OK) {
        if (err_line) *err_line = r.err_line;
        return fail(r.status, r.message);
    }
    return PRG_OK;
}

int32_t prg_parse_edgelist(const char *text, uint64_t len, uint32_t *from, uint32_t *to, uint64_t capacity,
                           uint64_t *m, uint32_t *n, uint64_t *err_line) {
    g_err.clear();
    PRG_GUARD_BEGIN
    if (m) *m = 0;
    if (n) *n = 0;
    if (!ensure_pool_config()) return fail(PRG_ERR_CUDA, "cuda: no usable device");
    cudaStream_t s;
    PRG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    prg::el::ParseResult r;
    int32_t rc = PRG_OK;
    try {
        rc = edgelist_common(text, len, s, r, err_line);
        if (rc == PRG_OK) {
            if (m) *m = r.m;
            if (n) *n = r.n;
            if (r.m > capacity) {
                rc = fail(PRG_ERR_INVALID_ARGUMENT, "edge arrays hold " + std::to_string(capacity) + " edges, the text has " +
                                                        std::to_string(r.m));
            } else if (r.m) {
                if (!from || !to) {
                    rc = fail(PRG_ERR_INVALID_ARGUMENT, "null edge arrays");
                } else {
                    PRG_CUDA(cudaMemcpyAsync(from, r.d_from, r.m * 4, cudaMemcpyDeviceToHost, s));
                    PRG_CUDA(cudaMemcpyAsync(to, r.d_to, r.m * 4, cudaMemcpyDeviceToHost, s));
                }
            }
        }
        prg::el::free_result(r, s);
        PRG_CUDA(cudaStreamSynchronize(s));
    } catch (...) {
        prg::el::free_result(r, s);
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
        throw;
    }
    cudaStreamDestroy(s);
    return rc;
    PRG_GUARD_END
}

int32_t prg_read_edgelist(const char *text, uint64_t len, prg_graph **out, uint32_t *n, uint64_t *m,
                          uint64_t *err_line) {
    g_err.clear();
    PRG_GUARD_BEGIN
    if (!out) return fail(PRG_ERR_INVALID_ARGUMENT, "null output handle");
    *out = nullptr;
    if (m) *m = 0;
    if (n) *n = 0;
    if (!ensure_pool_config()) return fail(PRG_ERR_CUDA, "cuda: no usable device");
    cudaStream_t s;
    PRG_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    prg::el::ParseResult r;
    int32_t rc = PRG_OK;
    try {
        rc = edgelist_common(text, len, s, r, err_line);
        if (rc == PRG_OK) {
            if (m) *m = r.m;
            if (n) *n = r.n;
            if (r.m > 0) {
                rc = create_from_device(r.n, r.m, r.d_from, r.d_to, nullptr, 0, s, out);
                if (rc == PRG_OK) {
                    prg::el::free_result(r, s);  // the graph owns the stream from here on
                    prepare_handle(*out);
                    return PRG_OK;
                }
            }
        }
        prg::el::free_result(r, s);
        PRG_CUDA(cudaStreamSynchronize(s));
    } catch (...) {
        prg::el::free_result(r, s);
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
        throw;
    }
    cudaStreamDestroy(s);
    return rc;
    PRG_GUARD_END
}

void prg_graph_destroy(prg_graph *g) {
    try {
        destroy(g);
    } catch (...) {
    }
}

int32_t prg_graph_relabelled(const prg_graph *h) { return h && h->g.perm ? 1 : 0; }

int32_t prg_graph_device_csr(const prg_graph *h, const uint32_t **row_ptr, const uint32_t **col,
                             const uint32_t **perm, const float **inv32) {
    if (!h) return fail(PRG_ERR_INVALID_ARGUMENT, "null graph handle");
    if (row_ptr) *row_ptr = h->g.row_ptr;
    if (col) *col = h->g.col;
    if (perm) *perm = h->g.perm;
    if (inv32) *inv32 = h->g.inv32;
    return PRG_OK;
}

int32_t prg_graph_info(const prg_graph *h, uint32_t *n, uint64_t *arcs, uint32_t *n_dangling, uint32_t *nrb,
                       uint32_t *nhub, double *build_ms) {
    if (!h) return fail(PRG_ERR_INVALID_ARGUMENT, "null graph handle");
    if (n) *n = h->g.n;
    if (arcs) *arcs = h->g.arcs;
    if (n_dangling) *n_dangling = h->g.n_dangling;
    if (nrb) *nrb = h->g.nrb;
    if (nhub) *nhub = h->g.nhub;
    if (build_ms) *build_ms = h->g.build_ms;
    return PRG_OK;
}

void *prg_graph_stream(prg_graph *h) { return h ? (void *)h->stream : nullptr; }

int32_t prg_graph_gather_probe(prg_graph *h, int32_t reps, double *ms_per_pass) {
    g_err.clear();
    PRG_GUARD_BEGIN
    if (!h) return fail(PRG_ERR_INVALID_ARGUMENT, "null graph handle");
    if (reps < 1 || reps > 10000) return fail(PRG_ERR_INVALID_ARGUMENT, "reps must be in 1..=10000");
    const float ms = prg::gather_probe(h->g, reps, h->stream);
    if (ms_per_pass) *ms_per_pass = (double)ms;
    return PRG_OK;
    PRG_GUARD_END
}

int32_t prg_graph_matvec32(prg_graph *h, int32_t kernel, const float *d_p, const float *d_pt, double dz,
                           double damping, float *d_y, double *dots, double *ms) {
    g_err.clear();
    PRG_GUARD_BEGIN
    if (!h) return fail(PRG_ERR_INVALID_ARGUMENT, "null graph handle");
    if (kernel < 0 || kernel > 2) return fail(PRG_ERR_INVALID_ARGUMENT, "kernel must be 0, 1 or 2");
    if (kernel != 0 && h->g.weighted)
        return fail(PRG_ERR_UNSUPPORTED, "the tile-segmented matvec serves unweighted graphs");
    if (!(damping >= 0.0 && damping <= 1.0)) return fail(PRG_ERR_INVALID_ARGUMENT, "damping must be in [0, 1]");
    if (h->g.n == 0 || h->g.arcs == 0) return fail(PRG_ERR_INVALID_ARGUMENT, "the graph has no arcs");
    if (!d_p || !d_pt || !d_y) return fail(PRG_ERR_INVALID_ARGUMENT, "null vector");
    double d[3];
    float t = 0.f;
    prg::matvec32_probe(h->g, h->ws, kernel, d_p, d_pt, dz, damping, d_y, d, &t, h->stream);
    if (dots) std::memcpy(dots, d, sizeof(d));
    if (ms) *ms = (double)t;
    return PRG_OK;
    PRG_GUARD_END
}

int32_t prg_solve(prg_graph *h, const prg_options *opt, const double *reset, double *out, prg_stats *st) {
    g_err.clear();
    PRG_GUARD_BEGIN
    if (!h) return fail(PRG_ERR_INVALID_ARGUMENT, "null graph handle");
    prg_options o;
    prg_default_options(&o);
    if (opt) o = *opt;
    if (int32_t rc = check_options(o)) return rc;
    const uint32_t n = h->g.n;
    if (n == 0) return PRG_OK;
    if (reset) {
        std::vector<double> norm;
        bool trivial = false;
        int32_t rc = ppr_validate(n, reset, n, o.damping, norm, &trivial);
        if (rc != PRG_OK) return rc;
        if (trivial) {
            out[0] = 1.0;
            return PRG_OK;
        }
        return solve_host(h, to_solve_opts(&o), norm.data(), o.start, out, st);
    }
    if (o.damping <= 0.0 || o.damping >= 1.0)
        return fail(PRG_ERR_INVALID_ARGUMENT, "damping (" + rust_f64(o.damping) + ") must be in (0, 1)");
    if (n == 1) {
        out[0] = 1.0;
        return PRG_OK;
    }
    return solve_host(h, to_solve_opts(&o), nullptr, o.start, out, st);
    PRG_GUARD_END
}

int32_t prg_solve_device(prg_graph *h, const prg_options *opt, const double *d_reset, double *d_out,
                         prg_stats *st) {
    g_err.clear();
    PRG_GUARD_BEGIN
    if (!h) return fail(PRG_ERR_INVALID_ARGUMENT, "null graph handle");
    prg_options o;
    prg_default_options(&o);
    if (opt) o = *opt;
    if (int32_t rc = check_options(o)) return rc;
    if (!(o.damping > 0.0 && o.damping < 1.0))
        return fail(PRG_ERR_INVALID_ARGUMENT, "damping (" + rust_f64(o.damping) + ") must be in (0, 1)");
    if (h->g.n < 2) return fail(PRG_ERR_INVALID_ARGUMENT, "device solve needs vcount >= 2");
    prg::SolveOpts so = to_solve_opts(&o);
    so.d_start = o.start;  // device pointer on this entry point
    cudaStream_t s = h->stream;
    const double *d_t = nullptr;
    if (d_reset) {
        if (!h->d_reset) PRG_CUDA(cudaMallocAsync((void **)&h->d_reset, (uint64_t)h->g.n * 8, s));
        PRG_CUDA(cudaMemcpyAsync(h->d_reset, d_reset, (uint64_t)h->g.n * 8, cudaMemcpyDeviceToDevice, s));
        d_t = h->d_reset;
    }
    prg::SolveStats ss;
    prg::solve(h->g, h->ws, so, d_t, d_out, ss, s);
    fill_stats(st, ss, h);
    return PRG_OK;
    PRG_GUARD_END
}

static int32_t batch_common(prg_graph *h, uint32_t K, const uint64_t *off, const uint32_t *seeds, double damping,
                            double tol, uint32_t max_iter, uint32_t vec, float *d_out, uint32_t *column_iters,
                            prg_batch_stats *st) {
    if (!h) return fail(PRG_ERR_INVALID_ARGUMENT, "null graph handle");
    if (K == 0) return fail(PRG_ERR_INVALID_ARGUMENT, "batch needs at least one column");
    if (!(damping > 0.0 && damping < 1.0))
        return fail(PRG_ERR_INVALID_ARGUMENT,
                    "personalized_pagerank: damping (" + rust_f64(damping) + ") must be in (0, 1)");
    const uint32_t n = h->g.n;
    if (n < 2) return fail(PRG_ERR_INVALID_ARGUMENT, "batched solve needs vcount >= 2");
    if (off[0] != 0) return fail(PRG_ERR_INVALID_ARGUMENT, "seed_offsets[0] must be 0");
    for (uint32_t k = 0; k < K; k++) {
        if (off[k + 1] <= off[k]) return fail(PRG_ERR_INVALID_ARGUMENT, "reset_vids must not be empty");
        for (uint64_t i = off[k]; i < off[k + 1]; i++)
            if (seeds[i] >= n)
                return fail(PRG_ERR_INVALID_ARGUMENT, "reset vertex " + std::to_string(seeds[i]) +
                                                          " out of range (vcount = " + std::to_string(n) + ")");
    }
    if (vec == 0) vec = h->g.batch_vec ? h->g.batch_vec : prg::tuning().batch_vec;
    prg::BatchStats bs;
    const int rc = prg::ppr_batch(h->g, K, off, seeds, damping, tol, max_iter, vec, d_out, bs, h->stream);
    if (column_iters)
        for (uint32_t k = 0; k < K; k++) column_iters[k] = bs.column_iters[k];
    if (st) {
        st->column_iterations = bs.column_iterations;
        st->max_iters = bs.max_iters;
        st->tiles = bs.tiles;
        st->tile_width = 32 * bs.vec;
        st->kernel_launches = bs.kernel_launches;
        st->ms = bs.ms;
        st->chebyshev = bs.chebyshev;
        st->pad = 0;
    }
    if (rc == PRG_ERR_TIMEOUT) return fail(PRG_ERR_TIMEOUT, "batched solve: a grid barrier timed out");
    if (rc != 0) return fail(PRG_ERR_INTERNAL, "batched solve: device status " + std::to_string(rc));
    return PRG_OK;
}

int32_t prg_ppr_batch_device(prg_graph *h, uint32_t K, const uint64_t *off, const uint32_t *seeds, double damping,
                             double tol, uint32_t max_iter, uint32_t vec, float *d_out, uint32_t *column_iters,
                             prg_batch_stats *st) {
    g_err.clear();
    PRG_GUARD_BEGIN
    return batch_common(h, K, off, seeds, damping, tol, max_iter, vec, d_out, column_iters, st);
    PRG_GUARD_END
}

int32_t prg_ppr_batch(prg_graph *h, uint32_t K, const uint64_t *off, const uint32_t *seeds, double damping,
                      double tol, uint32_t max_iter, uint32_t vec, float *out, uint32_t *column_iters,
                      prg_batch_stats *st) {
    g_err.clear();
    PRG_GUARD_BEGIN
    if (!h) return fail(PRG_ERR_INVALID_ARGUMENT, "null graph handle");
    float *d_out = nullptr;
    const size_t bytes = (size_t)h->g.n * K * 4;
    PRG_CUDA(cudaMallocAsync((void **)&d_out, std::max<size_t>(bytes, 16), h->stream));
    int32_t rc = batch_common(h, K, off, seeds, damping, tol, max_iter, vec, d_out, column_iters, st);
    if (rc == PRG_OK) PRG_CUDA(cudaMemcpyAsync(out, d_out, bytes, cudaMemcpyDeviceToHost, h->stream));
    cudaFreeAsync(d_out, h->stream);
    PRG_CUDA(cudaStreamSynchronize(h->stream));
    return rc;
    PRG_GUARD_END
}

int32_t prg_autotune(prg_graph *h, int32_t tune_batch, const char *cache_path, prg_tune_result *out) {
    g_err.clear();
    PRG_GUARD_BEGIN
    if (!h) return fail(PRG_ERR_INVALID_ARGUMENT, "null graph handle");
    if (h->g.n < 2) return fail(PRG_ERR_INVALID_ARGUMENT, "autotune needs vcount >= 2");
    prg::TuneResult r;
    prg::autotune(h->g, h->ws, h->stream, tune_batch != 0, cache_path, r);
    if (out) {
        out->capw = r.capw;
        out->shortmax = r.shortmax;
        out->split = r.split;
        out->blocks_per_sm = r.blocks_per_sm;
        out->batch_tile_width = 32 * r.batch_vec;
        out->candidates = r.tried;
        out->from_cache = r.from_cache ? 1 : 0;
        out->default_ms = r.default_ms;
        out->best_ms = r.best_ms;
        out->seg_hot = r.seg_hot;
        out->seg_hot64 = r.seg_hot64;
        out->seg_default_ms = r.seg_default_ms;
        out->seg_best_ms = r.seg_best_ms;
    }
    return PRG_OK;
    PRG_GUARD_END
}

// ---- learned warm start ----------------------------------------------------

struct prg_gnn {
    prg::gnn::Net net;
    double *tmp = nullptr;  // n doubles (target / prediction in internal ids)
    uint32_t tmp_n = 0;
};

static double *gnn_tmp(prg_gnn *net, uint32_t n, cudaStream_t s) {
    if (net->tmp_n < n) {
        if (net->tmp) cudaFreeAsync(net->tmp, s);
        PRG_CUDA(cudaMallocAsync((void **)&net->tmp, (size_t)n * 8, s));
        net->tmp_n = n;
    }
    return net->tmp;
}

uint32_t prg_gnn_param_count(void) { return (uint32_t)prg::gnn::param_count(); }

int32_t prg_gnn_create(uint64_t seed, prg_gnn **out) {
    g_err.clear();
    PRG_GUARD_BEGIN
    if (!out) return fail(PRG_ERR_INVALID_ARGUMENT, "null output handle");
    if (!ensure_pool_config()) return fail(PRG_ERR_CUDA, "cuda: no usable device");
    prg_gnn *net = new prg_gnn();
    net->net.init(seed, 0);
    PRG_CUDA(cudaStreamSynchronize(0));
    *out = net;
    return PRG_OK;
    PRG_GUARD_END
}

void prg_gnn_destroy(prg_gnn *net) {
    if (!net) return;
    try {
        net->net.free(0);
        if (net->tmp) cudaFreeAsync(net->tmp, 0);
        cudaStreamSynchronize(0);
    } catch (...) {
    }
    delete net;
}

int32_t prg_gnn_get_params(const prg_gnn *net, float *host) {
    g_err.clear();
    PRG_GUARD_BEGIN
    if (!net || !host) return fail(PRG_ERR_INVALID_ARGUMENT, "null argument");
    net->net.get_params(host, 0);
    return PRG_OK;
    PRG_GUARD_END
}

int32_t prg_gnn_set_params(prg_gnn *net, const float *host) {
    g_err.clear();
    PRG_GUARD_BEGIN
    if (!net || !host) return fail(PRG_ERR_INVALID_ARGUMENT, "null argument");
    for (int i = 0; i < prg::gnn::param_count(); i++)
        if (!std::isfinite(host[i])) return fail(PRG_ERR_INVALID_ARGUMENT, "parameters must be finite");
    net->net.set_params(host, 0);
    return PRG_OK;
    PRG_GUARD_END
}

int32_t prg_gnn_predict(prg_gnn *net, prg_graph *h, double *d_start, double *ms) {
    g_err.clear();
    PRG_GUARD_BEGIN
    if (!net || !h || !d_start) return fail(PRG_ERR_INVALID_ARGUMENT, "null argument");
    if (h->g.n < 2) return fail(PRG_ERR_INVALID_ARGUMENT, "prediction needs vcount >= 2");
    cudaStream_t s = h->stream;
    PRG_CUDA(cudaStreamSynchronize(0));
    cudaEvent_t e0, e1;
    PRG_CUDA(cudaEventCreate(&e0));
    PRG_CUDA(cudaEventCreate(&e1));
    PRG_CUDA(cudaEventRecord(e0, s));
    if (h->g.iperm) {
        double *x = gnn_tmp(net, h->g.n, s);
        net->net.predict(h->g, x, s);
        prg::gather_f64(d_start, x, h->g.iperm, h->g.n, s);
    } else {
        net->net.predict(h->g, d_start, s);
    }
    PRG_CUDA(cudaEventRecord(e1, s));
    PRG_CUDA(cudaEventSynchronize(e1));
    float t = 0.f;
    PRG_CUDA(cudaEventElapsedTime(&t, e0, e1));
    if (ms) *ms = t;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return PRG_OK;
    PRG_GUARD_END
}

static int32_t gnn_loss(prg_gnn *net, prg_graph *h, const double *d_target, double *loss) {
    cudaStream_t s = h->stream;
    PRG_CUDA(cudaStreamSynchronize(0));
    const double *t = d_target;
    if (h->g.perm) {
        double *tt = gnn_tmp(net, h->g.n, s);
        prg::gather_f64(tt, d_target, h->g.perm, h->g.n, s);
        t = tt;
    }
    const double l = net->net.loss_grad(h->g, t, s);
    if (loss) *loss = l;
    return PRG_OK;
}

int32_t prg_gnn_loss_grad(prg_gnn *net, prg_graph *h, const double *d_target, double *loss, float *host_grad) {
    g_err.clear();
    PRG_GUARD_BEGIN
    if (!net || !h || !d_target) return fail(PRG_ERR_INVALID_ARGUMENT, "null argument");
    if (h->g.n < 2) return fail(PRG_ERR_INVALID_ARGUMENT, "training needs vcount >= 2");
    int32_t rc = gnn_loss(net, h, d_target, loss);
    if (rc == PRG_OK && host_grad) {
        PRG_CUDA(cudaMemcpyAsync(host_grad, net->net.G, (size_t)prg::gnn::param_count() * 4, cudaMemcpyDeviceToHost,
                                 h->stream));
        PRG_CUDA(cudaStreamSynchronize(h->stream));
    }
    return rc;
    PRG_GUARD_END
}

int32_t prg_gnn_train_step(prg_gnn *net, prg_graph *h, const double *d_target, float lr, double *loss) {
    g_err.clear();
    PRG_GUARD_BEGIN
    if (!net || !h || !d_target) return fail(PRG_ERR_INVALID_ARGUMENT, "null argument");
    if (h->g.n < 2) return fail(PRG_ERR_INVALID_ARGUMENT, "training needs vcount >= 2");
    if (!(lr > 0.0f)) return fail(PRG_ERR_INVALID_ARGUMENT, "learning rate must be > 0");
    int32_t rc = gnn_loss(net, h, d_target, loss);
    if (rc == PRG_OK) {
        net->net.adam(lr, h->stream);
        PRG_CUDA(cudaStreamSynchronize(h->stream));
    }
    return rc;
    PRG_GUARD_END
}

int32_t prg_set_tuning(const char *key, int64_t value) {
    g_err.clear();
    if (!key) return fail(PRG_ERR_INVALID_ARGUMENT, "null tuning key");
    prg::Tuning &t = prg::tuning();
    const std::string k(key);
    if (value < 0) return fail(PRG_ERR_INVALID_ARGUMENT, "tuning value must be >= 0");
    if (k == "defaults") t = prg::Tuning{};  // every key back to its default
    else if (k == "capw") t.capw = (uint32_t)value;
    else if (k == "shortmax") t.shortmax = (uint32_t)value;
    else if (k == "split") t.split = (uint32_t)value;
    else if (k == "blocks_per_sm") t.blocks_per_sm = (uint32_t)value;
    else if (k == "relabel") {
        if (value > 2) return fail(PRG_ERR_INVALID_ARGUMENT, "relabel must be 0, 1 or 2");
        t.relabel = (int)value;
    } else if (k == "batch_vec") {
        if (value != 1 && value != 2 && value != 4) return fail(PRG_ERR_INVALID_ARGUMENT, "batch_vec must be 1, 2 or 4");
        t.batch_vec = (uint32_t)value;
    } else if (k == "refine_switch_e12") {
        t.refine_switch = (double)value * 1e-12;
    } else if (k == "batch_cheb") {
        if (value != 0 && value != 1) return fail(PRG_ERR_INVALID_ARGUMENT, "batch_cheb must be 0 or 1");
        t.batch_cheb = (uint32_t)value;
    } else if (k == "batch_barrier_extra") {
        if (value > 1) return fail(PRG_ERR_INVALID_ARGUMENT, "batch_barrier_extra must be 0 or 1");
        t.batch_barrier_extra = (uint32_t)value;
    } else if (k == "l1_hot32") {
        t.l1_hot32 = (uint32_t)std::min<int64_t>(value, 0xFFFFFFFFll);
    } else if (k == "l1_hot64") {
        t.l1_hot64 = (uint32_t)std::min<int64_t>(value, 0xFFFFFFFFll);
    } else if (k == "krylov_floor_pct") {
        if (value < 1 || value > 90) return fail(PRG_ERR_INVALID_ARGUMENT, "krylov_floor_pct must be in [1, 90]");
        t.krylov_floor = (double)value / 100.0;
    } else if (k == "krylov_rel_e12") {
        t.krylov_rel = (double)value * 1e-12;
    } else if (k == "hot_cache" || k == "hot_cache32" || k == "hot_cache64") {
        if (value > 65536) return fail(PRG_ERR_INVALID_ARGUMENT, k + " must be at most 65536 entries");
        if (k != "hot_cache64") t.hot_cache = (uint32_t)value;
        if (k != "hot_cache32") t.hot_cache64 = (uint32_t)value;
    } else if (k == "seg_kry32") {
        if (value > 2) return fail(PRG_ERR_INVALID_ARGUMENT, "seg_kry32 must be 0, 1 or 2");
        t.seg_kry32 = (uint32_t)value;
    } else if (k == "seg_res64") {
        if (value > 1) return fail(PRG_ERR_INVALID_ARGUMENT, "seg_res64 must be 0 or 1");
        t.seg_res64 = (uint32_t)value;
    } else if (k == "seg_plain64") {
        if (value > 1) return fail(PRG_ERR_INVALID_ARGUMENT, "seg_plain64 must be 0 or 1");
        t.seg_plain64 = (uint32_t)value;
    } else if (k == "seg_eig64") {
        if (value > 1) return fail(PRG_ERR_INVALID_ARGUMENT, "seg_eig64 must be 0 or 1");
        t.seg_eig64 = (uint32_t)value;
    } else if (k == "seg_threads") {
        if (value != 1024 && value != 768 && value != 512)
            return fail(PRG_ERR_INVALID_ARGUMENT, "seg_threads must be 1024, 768 or 512");
        t.seg_threads = (uint32_t)value;
    } else if (k == "seg_pipe") {
        if (value > 1) return fail(PRG_ERR_INVALID_ARGUMENT, "seg_pipe must be 0 or 1");
        t.seg_pipe = (uint32_t)value;
    } else if (k == "seg_prefetch") {
        if (value > 1) return fail(PRG_ERR_INVALID_ARGUMENT, "seg_prefetch must be 0 or 1");
        t.seg_prefetch = (uint32_t)value;
    } else if (k == "seg_hot64") {
        if (value > 20480) return fail(PRG_ERR_INVALID_ARGUMENT, "seg_hot64 must be at most 20480 entries");
        t.seg_hot64 = (uint32_t)value;
    } else if (k == "seg_hot") {
        if (value > 49152) return fail(PRG_ERR_INVALID_ARGUMENT, "seg_hot must be at most 49152 entries");
        t.seg_hot = (uint32_t)value;
    } else if (k == "hot_threads") {
        if (value != 256 && value != 512 && value != 1024)
            return fail(PRG_ERR_INVALID_ARGUMENT, "hot_threads must be 256, 512 or 1024");
        t.hot_threads = (uint32_t)value;
    } else if (k == "unroll") {
        if (value < 1 || value > 64) return fail(PRG_ERR_INVALID_ARGUMENT, "unroll must be in 1..=64");
        t.unroll = (int)value;
    } else {
        return fail(PRG_ERR_INVALID_ARGUMENT, "unknown tuning key: " + k);
    }
    return PRG_OK;
}

int32_t prg_generate_device(int32_t kind, uint32_t n, uint64_t m, double p0, double p1, double p2, uint64_t seed,
                            uint32_t *d_from, uint32_t *d_to, void *stream) {
    g_err.clear();
    PRG_GUARD_BEGIN
    if (kind < 0 || kind > 2) return fail(PRG_ERR_INVALID_ARGUMENT, "generator kind must be 0, 1 or 2");
    if (n < 2) return fail(PRG_ERR_INVALID_ARGUMENT, "generator needs n >= 2");
    if (kind == 2 && (p0 < 1.0 || (uint32_t)p0 > n)) return fail(PRG_ERR_INVALID_ARGUMENT, "bad block count");
    if (kind == 0 && (n & (n - 1)) != 0) return fail(PRG_ERR_INVALID_ARGUMENT, "R-MAT needs n = 2^scale");
    prg::generate_device(kind, n, m, p0, p1, p2, seed, d_from, d_to, (cudaStream_t)stream);
    return PRG_OK;
    PRG_GUARD_END
}

int32_t prg_rmat_device(uint32_t scale, uint64_t m, double a, double b, double c, uint64_t seed, uint32_t *d_from,
                        uint32_t *d_to, void *stream) {
    g_err.clear();
    PRG_GUARD_BEGIN
    if (scale == 0 || scale > 32) return fail(PRG_ERR_INVALID_ARGUMENT, "scale must be in 1..=32");
    prg::rmat_generate(scale, m, a, b, c, seed, d_from, d_to, (cudaStream_t)stream);
    return PRG_OK;
    PRG_GUARD_END
}

}  // extern "C"
