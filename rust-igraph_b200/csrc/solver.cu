// solver.cu — drives the fused iteration kernels: FP64 power iteration (the
// drop-in) and FP32 iteration with FP64 residual refinement.  Iterations run
// inside captured CUDA graphs of `unroll` iteration pairs; the kernels stop
// themselves (Ctl::done) so the host only polls a pinned copy of Ctl once per
// graph launch.
//
// Refinement (FP32 SpMV, FP64 residual):
//   G(x) = d*P^T(x/s) + d*(sum_dangling x)*t + (1-d)*t  is an L1 contraction
//   with factor d, so ||x - x*||_1 <= ||G(x) - x||_1 / (1-d).
//   repeat: g = G(x) and r = g - x in FP64 (MODE_RESID64);
//           if ||r||_1 <= eps*(1-d)/d: return g (error <= d*||r||/(1-d) <= eps)
//           solve e = d*M e + r approximately in FP32 (MODE_CORR32, seeded
//           with e0 = r) until its successive change <= max(rho*||r||, floor);
//           x <- x + e in FP64.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "solver.cuh"

namespace prg {

template <class T>
static void walloc(T *&p, uint64_t count, cudaStream_t s) {
    PRG_CUDA(cudaMallocAsync((void **)&p, std::max<uint64_t>(count, 1) * sizeof(T), s));
}
template <class T>
static void wfree(T *&p, cudaStream_t s) {
    if (p) cudaFreeAsync(p, s);
    p = nullptr;
}

constexpr uint32_t kPrepParts = 148u * 4u;

void workspace_free(Workspace &ws, cudaStream_t s) {
    for (auto &kv : ws.graphs) cudaGraphExecDestroy(kv.second);
    ws.graphs.clear();
    krylov_free(ws.kry, s);
    seg_free(ws.seg, s);
    for (int i = 0; i < 2; i++) {
        wfree(ws.x64[i], s);
        wfree(ws.xt64[i], s);
        wfree(ws.e32[i], s);
        wfree(ws.et32[i], s);
    }
    wfree(ws.b32, s);
    wfree(ws.t64, s);
    wfree(ws.t32, s);
    wfree(ws.out_tmp, s);
    wfree(ws.ctl, s);
    wfree(ws.blk_part, s);
    wfree(ws.hub_rec, s);
    wfree(ws.chunk_part, s);
    wfree(ws.hub_ticket, s);
    if (ws.h_ctl) cudaFreeHost(ws.h_ctl);
    ws.h_ctl = nullptr;
    for (cudaEvent_t *e : {&ws.ev0, &ws.ev1, &ws.eva, &ws.evb}) {
        if (*e) cudaEventDestroy(*e);
        *e = nullptr;
    }
    ws.ready = false;
}

void workspace_ensure(Workspace &ws, const DeviceGraph &g, cudaStream_t s) {
    if (ws.ready && ws.graphs_rb != (const void *)g.rb) {
        // row-blocks were rebuilt (autotuner): captured graphs hold the old list
        for (auto &kv : ws.graphs) cudaGraphExecDestroy(kv.second);
        ws.graphs.clear();
        ws.graphs_rb = g.rb;
    }
    if (ws.ready && ws.n == g.n && ws.nrb == g.nrb && ws.nhub == g.nhub) return;
    if (ws.ready) workspace_free(ws, s);
    ws.n = g.n;
    ws.nrb = g.nrb;
    ws.nhub = g.nhub;
    unsigned gmax = kPrepParts;
    const bool seg = !g.weighted && g.seg_kry32 != 0 && g.arcs > 0;
    const bool seg_res = !g.weighted && g.seg_res64 != 0 && g.arcs > 0;
    const bool seg_plain = !g.weighted && g.seg_plain64 != 0 && g.arcs > 0;
    const bool seg_eig = !g.weighted && g.seg_eig64 != 0 && g.arcs > 0;
    for (int m = 0; m < kModes; m++) {
        const bool fp32 = m == MODE_CORR32 || m == MODE_KRY32;
        const uint32_t hot = g.perm != nullptr ? (fp32 ? g.hot_cache : g.hot_cache64) : 0u;
        if (m == MODE_KRY32 && seg) ws.cfg[m] = seg_config(g, g.perm != nullptr ? g.seg_hot : 0u, (int)g.seg_kry32);
        else if (m == MODE_KRES64 && seg_res)
            ws.cfg[m] = seg_config(g, g.perm != nullptr ? g.seg_hot64 : 0u, 2, MODE_KRES64);
        else if ((m == MODE_PLAIN64 || m == MODE_PPR64 || m == MODE_KRY64) && seg_plain)
            ws.cfg[m] = seg_config(g, g.perm != nullptr ? g.seg_hot64 : 0u, 2, m);
        else if (m == MODE_EIG64 && seg_eig)
            ws.cfg[m] = seg_config(g, g.perm != nullptr ? g.seg_hot64 : 0u, 2, m);
        else ws.cfg[m] = iteration_config(m, g.weighted, hot, g.blocks_per_sm, g.n, g.hot_threads);
        if (!ws.cfg[m].seg) ws.cfg[m].hub_recs = g.nhub;
        const uint32_t l1 = fp32 ? g.l1_hot32 : g.l1_hot64;
        if (g.perm != nullptr && l1) ws.cfg[m].l1hot = l1;
        gmax = std::max(gmax, ws.cfg[m].grid);
    }
    if (seg || seg_res || seg_plain || seg_eig) seg_build(g, ws.seg, s);
    const uint64_t n = g.n;
    for (int i = 0; i < 2; i++) {
        walloc(ws.x64[i], n, s);
        walloc(ws.xt64[i], n, s);
        walloc(ws.e32[i], n, s);
        walloc(ws.et32[i], n, s);
    }
    walloc(ws.b32, n, s);
    walloc(ws.t64, n, s);
    walloc(ws.t32, n, s);
    if (g.perm) walloc(ws.out_tmp, n, s);
    walloc(ws.ctl, 1, s);
    walloc(ws.blk_part, gmax, s);
    walloc(ws.hub_rec, g.nhub, s);
    walloc(ws.chunk_part, g.nrb, s);
    walloc(ws.hub_ticket, g.nhub, s);
    PRG_CUDA(cudaMemsetAsync(ws.hub_ticket, 0, std::max<uint64_t>(g.nhub, 1) * 4, s));
    PRG_CUDA(cudaMemsetAsync(ws.hub_rec, 0, std::max<uint64_t>(g.nhub, 1) * sizeof(double4), s));
    PRG_CUDA(cudaMallocHost((void **)&ws.h_ctl, sizeof(Ctl)));
    PRG_CUDA(cudaEventCreate(&ws.ev0));
    PRG_CUDA(cudaEventCreate(&ws.ev1));
    PRG_CUDA(cudaEventCreate(&ws.eva));
    PRG_CUDA(cudaEventCreate(&ws.evb));
    ws.graphs_rb = g.rb;
    ws.ready = true;
}

IterArgs base_args(const DeviceGraph &g, Workspace &ws, double damping) {
    IterArgs a;
    std::memset(&a, 0, sizeof(a));
    a.row_ptr = g.row_ptr;
    a.col = g.col;
    a.w64 = g.w64;
    a.w32 = g.w32;
    a.dval = g.dval;
    a.inv32 = g.inv32;
    a.rb = g.rb;
    a.hubs = g.hubs;
    a.nrb = g.nrb;
    a.nhub = g.nhub;
    a.n = g.n;
    a.damping = damping;
    a.inv_n = 1.0 / (double)g.n;
    a.arcs = g.arcs;
    a.seg_mask = ws.seg.mask;
    a.seg_tile_j0 = ws.seg.tile_j0;
    a.seg_meta = ws.seg.meta;
    a.seg_nz = ws.seg.nz_row;
    a.seg_empty = ws.seg.empty_row;
    a.seg_head = ws.seg.head;
    a.seg_tail = ws.seg.tail;
    a.seg_ntiles = ws.seg.ntiles;
    a.seg_nempty = ws.seg.n_empty;
    a.seg_dense = ws.seg.dense;
    a.seg_prefetch = g.seg_prefetch;
    a.seg_span = ws.seg.span;
    a.seg_span_long = ws.seg.span_long;
    a.seg_nspan = ws.seg.n_span;
    a.seg_nlong = ws.seg.n_long;
    a.ctl = ws.ctl;
    a.blk_part = ws.blk_part;
    a.chunk_part = ws.chunk_part;
    a.hub_rec = ws.hub_rec;
    a.hub_ticket = ws.hub_ticket;
    return a;
}

static uint64_t graph_key(int mode, bool has_t, double damping) {
    uint64_t bits;
    std::memcpy(&bits, &damping, 8);
    return (bits * 0x9E3779B97F4A7C15ULL) ^ ((uint64_t)mode << 1) ^ (uint64_t)has_t;
}

// Captured graph of `unroll` (parity 0, parity 1) launch pairs.
static cudaGraphExec_t loop_graph(const DeviceGraph &g, Workspace &ws, int mode, bool has_t, double damping,
                                  const IterArgs &a0, const IterArgs &a1, cudaStream_t s) {
    const uint64_t key = graph_key(mode, has_t, damping);
    auto it = ws.graphs.find(key);
    if (it != ws.graphs.end()) return it->second;
    cudaGraph_t graph;
    PRG_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
    for (int u = 0; u < ws.unroll; u++) {
        launch_iteration(mode, g.weighted, a0, ws.cfg[mode], s);
        launch_iteration(mode, g.weighted, a1, ws.cfg[mode], s);
    }
    PRG_CUDA(cudaStreamEndCapture(s, &graph));
    cudaGraphExec_t exec;
    PRG_CUDA(cudaGraphInstantiate(&exec, graph, 0));
    cudaGraphDestroy(graph);
    ws.graphs[key] = exec;
    return exec;
}

// Launches the loop graph until the kernels raise Ctl::done.  Adds the
// device time of the graph launches (CUDA events on `s`) to *ms and the
// kernels they contain to *launches.
static void run_loop(Workspace &ws, cudaGraphExec_t exec, uint32_t max_iter, cudaStream_t s, double *ms,
                     uint32_t *launches) {
    const uint64_t max_launches = (uint64_t)max_iter / (2u * ws.unroll) + 2u;
    for (uint64_t k = 0; k < max_launches; k++) {
        PRG_CUDA(cudaEventRecord(ws.eva, s));
        PRG_CUDA(cudaGraphLaunch(exec, s));
        PRG_CUDA(cudaEventRecord(ws.evb, s));
        PRG_CUDA(cudaMemcpyAsync(ws.h_ctl, ws.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
        PRG_CUDA(cudaStreamSynchronize(s));
        float t = 0.f;
        PRG_CUDA(cudaEventElapsedTime(&t, ws.eva, ws.evb));
        *ms += t;
        *launches += 2u * ws.unroll;
        if (ws.h_ctl->done) return;
    }
}

void read_ctl(Workspace &ws, cudaStream_t s) {
    PRG_CUDA(cudaMemcpyAsync(ws.h_ctl, ws.ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, s));
    PRG_CUDA(cudaStreamSynchronize(s));
}

__global__ void to_f32_kernel(const double *a, float *b, uint32_t n) {
    for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < n; v += gridDim.x * blockDim.x) b[v] = (float)a[v];
}

void to_f32(const double *a, float *b, uint32_t n, cudaStream_t s) {
    to_f32_kernel<<<148 * 4, kThreads, 0, s>>>(a, b, n);
    PRG_CUDA(cudaGetLastError());
}

// FP64 power iteration (PLAIN64 / PPR64) from the start vector until the
// successive L1 change is < thr or max_iter iterations ran.  Returns the
// buffer holding the newest iterate.
const double *fp64_loop(const DeviceGraph &g, Workspace &ws, const SolveOpts &o, const double *d_t, double thr,
                        uint32_t max_iter, SolveStats &st, cudaStream_t s) {
    const bool ppr = d_t != nullptr;
    if (o.d_start) {
        if (o.d_start != ws.x64[0])
            PRG_CUDA(cudaMemcpyAsync(ws.x64[0], o.d_start, (uint64_t)g.n * 8, cudaMemcpyDeviceToDevice, s));
    } else {
        launch_fill_start(ws.x64[0], d_t, g.n, s);
    }
    Ctl c;
    std::memset(&c, 0, sizeof(c));
    c.thr = thr;
    c.max_iter = max_iter;
    PRG_CUDA(cudaMemcpyAsync(ws.ctl, &c, sizeof(Ctl), cudaMemcpyHostToDevice, s));
    launch_prepare64(g, ws.x64[0], nullptr, ws.xt64[0], ws.ctl, 0, ws.blk_part, s);
    st.kernel_launches += (o.d_start ? 0u : 1u) + 2u;
    IterArgs a0 = base_args(g, ws, o.damping), a1 = a0;
    a0.t64 = a1.t64 = d_t;
    a0.parity = 0;
    a0.x64_in = ws.x64[0];
    a0.xt64_in = ws.xt64[0];
    a0.x64_out = ws.x64[1];
    a0.xt64_out = ws.xt64[1];
    a1.parity = 1;
    a1.x64_in = ws.x64[1];
    a1.xt64_in = ws.xt64[1];
    a1.x64_out = ws.x64[0];
    a1.xt64_out = ws.xt64[0];
    const int mode = ppr ? MODE_PPR64 : MODE_PLAIN64;
    if (max_iter > 0) {
        cudaGraphExec_t ex = loop_graph(g, ws, mode, ppr, o.damping, a0, a1, s);
        const double before = st.fp64_ms;
        run_loop(ws, ex, max_iter, s, &st.fp64_ms, &st.kernel_launches);
        st.spmv_ms += st.fp64_ms - before;
    } else {
        read_ctl(ws, s);
    }
    const Ctl &h = *ws.h_ctl;
    st.spmv_launches += h.iters;
    st.fp64_passes += h.iters;
    st.iterations += h.iters;
    st.last_diff = h.diff;
    return (h.iters == 0) ? ws.x64[0] : (h.parity_last == 0 ? ws.x64[1] : ws.x64[0]);
}

static void solve_fp64(const DeviceGraph &g, Workspace &ws, const SolveOpts &o, const double *d_t, double *d_out,
                       SolveStats &st, cudaStream_t s) {
    const double thr = o.stop == 1 ? o.eps * (1.0 - o.damping) / o.damping : o.eps;
    const double *res = fp64_loop(g, ws, o, d_t, thr, o.max_iter, st, s);
    PRG_CUDA(cudaMemcpyAsync(d_out, res, (uint64_t)g.n * 8, cudaMemcpyDeviceToDevice, s));
    st.residual_l1 = st.last_diff;
    st.error_bound = st.last_diff * o.damping / (1.0 - o.damping);
}

// Refined solve.  FP32 corrections carry a rounding error of ~1e-7 of the
// correction's size, spread over every eigen-direction of the operator, and
// slow directions decay only at the rate d.  Corrections therefore start
// once the FP64 power iteration has brought the successive change below
// `refine_switch` (so that noise sits far under the tolerance); above it the
// iteration stays in FP64.
static void solve_refined(const DeviceGraph &g, Workspace &ws, const SolveOpts &o, const double *d_t,
                          double *d_out, SolveStats &st, cudaStream_t s) {
    const bool ppr = d_t != nullptr;
    const double thr_final = o.eps * (1.0 - o.damping) / o.damping;
    const double sw = std::max(o.refine_switch, thr_final);
    const double *xa = fp64_loop(g, ws, o, d_t, sw, o.max_iter, st, s);
    if (!(st.last_diff >= thr_final) && st.fp64_passes > 0) {
        // the FP64 phase already met the error bound
        PRG_CUDA(cudaMemcpyAsync(d_out, xa, (uint64_t)g.n * 8, cudaMemcpyDeviceToDevice, s));
        st.residual_l1 = st.last_diff;
        st.error_bound = st.last_diff * o.damping / (1.0 - o.damping);
        return;
    }
    if (xa != ws.x64[0]) PRG_CUDA(cudaMemcpyAsync(ws.x64[0], xa, (uint64_t)g.n * 8, cudaMemcpyDeviceToDevice, s));
    if (ppr) {
        to_f32_kernel<<<148 * 4, kThreads, 0, s>>>(d_t, ws.t32, g.n);
        st.kernel_launches += 1u;
    }
    Ctl c;
    std::memset(&c, 0, sizeof(c));
    c.rho = 4e-6;
    c.floor_abs = 0.05 * thr_final;
    const uint32_t inner_cap = std::max<uint32_t>(16u, std::min<uint32_t>(o.max_iter, 400u));
    c.max_iter = inner_cap;
    PRG_CUDA(cudaMemcpyAsync(ws.ctl, &c, sizeof(Ctl), cudaMemcpyHostToDevice, s));
    launch_prepare64(g, ws.x64[0], nullptr, ws.xt64[0], ws.ctl, 1, ws.blk_part, s);
    st.kernel_launches += 2u;

    IterArgs r = base_args(g, ws, o.damping);
    r.t64 = d_t;
    r.parity = 1;
    r.x64_in = ws.x64[0];
    r.xt64_in = ws.xt64[0];
    r.x64_out = ws.x64[1];
    r.b32_out = ws.b32;
    r.x32_out = ws.e32[0];
    r.xt32_out = ws.et32[0];

    IterArgs a0 = base_args(g, ws, o.damping), a1 = a0;
    a0.t32 = a1.t32 = ppr ? ws.t32 : nullptr;
    a0.b32 = a1.b32 = ws.b32;
    a0.parity = 0;
    a0.x32_in = ws.e32[0];
    a0.xt32_in = ws.et32[0];
    a0.x32_out = ws.e32[1];
    a0.xt32_out = ws.et32[1];
    a1.parity = 1;
    a1.x32_in = ws.e32[1];
    a1.xt32_in = ws.et32[1];
    a1.x32_out = ws.e32[0];
    a1.xt32_out = ws.et32[0];
    cudaGraphExec_t ex = loop_graph(g, ws, MODE_CORR32, ppr, o.damping, a0, a1, s);

    const uint32_t pass_cap = std::max<uint32_t>(o.max_iter, 64u);
    uint32_t fp32 = 0, fp64 = st.fp64_passes;
    for (int outer = 0; outer < 64; outer++) {
        PRG_CUDA(cudaEventRecord(ws.eva, s));
        launch_iteration(MODE_RESID64, g.weighted, r, ws.cfg[MODE_RESID64], s);
        PRG_CUDA(cudaEventRecord(ws.evb, s));
        fp64++;
        st.kernel_launches += 1u;
        read_ctl(ws, s);
        {
            float t = 0.f;
            PRG_CUDA(cudaEventElapsedTime(&t, ws.eva, ws.evb));
            st.fp64_ms += t;
        }
        const double rn = ws.h_ctl->rnorm;
        st.residual_l1 = rn;
        if (std::getenv("PRG_TRACE"))
            std::fprintf(stderr, "[prg] residual pass %u: ||r||_1 = %.3e (after %u fp32 passes)\n", fp64, rn, fp32);
        if (!(rn > thr_final) || fp32 + fp64 >= pass_cap) break;
        const double before = st.fp32_ms;
        run_loop(ws, ex, inner_cap, s, &st.fp32_ms, &st.kernel_launches);
        st.spmv_ms += st.fp32_ms - before;
        st.spmv_launches += ws.h_ctl->iters;
        fp32 += ws.h_ctl->iters;
        const float *e_fin = ws.h_ctl->parity_last == 0 ? ws.e32[1] : ws.e32[0];
        launch_prepare64(g, ws.x64[0], e_fin, ws.xt64[0], ws.ctl, 1, ws.blk_part, s);
        st.kernel_launches += 2u;
    }
    if (o.normalise) {
        // result = g / sum(g) (FP64), sum taken by the last residual pass
        PRG_CUDA(cudaMemcpyAsync(d_out, ws.x64[1], (uint64_t)g.n * 8, cudaMemcpyDeviceToDevice, s));
        launch_normalise(d_out, g.n, ws.ctl, s);
        st.kernel_launches += 1u;
    } else {
        PRG_CUDA(cudaMemcpyAsync(d_out, ws.x64[1], (uint64_t)g.n * 8, cudaMemcpyDeviceToDevice, s));
    }
    st.fp32_passes = fp32;
    st.residual_passes = fp64 - st.fp64_passes;
    st.fp64_passes = fp64;
    st.iterations = fp32 + fp64;
    st.last_diff = ws.h_ctl->diff;
    st.error_bound = st.residual_l1 * o.damping / (1.0 - o.damping);
}

double time_iterations(const DeviceGraph &g, Workspace &ws, int mode, uint32_t iters, cudaStream_t s) {
    workspace_ensure(ws, g, s);
    PRG_CUDA(cudaMemsetAsync(ws.hub_ticket, 0, std::max<uint64_t>(g.nhub, 1) * 4, s));
    const uint64_t n = g.n;
    launch_fill_start(ws.x64[0], nullptr, g.n, s);
    for (int i = 0; i < 2; i++) {
        PRG_CUDA(cudaMemsetAsync(ws.e32[i], 0, n * 4, s));
        PRG_CUDA(cudaMemsetAsync(ws.et32[i], 0, n * 4, s));
    }
    PRG_CUDA(cudaMemsetAsync(ws.b32, 0, n * 4, s));
    Ctl c;
    std::memset(&c, 0, sizeof(c));
    c.thr = -1.0;  // never converges: every launch does the full work
    c.max_iter = 0xFFFFFFFFu;
    PRG_CUDA(cudaMemcpyAsync(ws.ctl, &c, sizeof(Ctl), cudaMemcpyHostToDevice, s));
    launch_prepare64(g, ws.x64[0], nullptr, ws.xt64[0], ws.ctl, 0, ws.blk_part, s);
    IterArgs a[2];
    a[0] = base_args(g, ws, 0.85);
    a[1] = a[0];
    for (int p = 0; p < 2; p++) {
        a[p].parity = p;
        a[p].x64_in = ws.x64[p];
        a[p].xt64_in = ws.xt64[p];
        a[p].x64_out = ws.x64[p ^ 1];
        a[p].xt64_out = ws.xt64[p ^ 1];
        a[p].x32_in = ws.e32[p];
        a[p].xt32_in = ws.et32[p];
        a[p].x32_out = ws.e32[p ^ 1];
        a[p].xt32_out = ws.et32[p ^ 1];
        a[p].b32 = ws.b32;
        a[p].b32_out = ws.b32;
    }
    const int m = mode == MODE_RESID64 ? MODE_PLAIN64 : mode;
    for (int k = 0; k < 2; k++) launch_iteration(m, g.weighted, a[k & 1], ws.cfg[m], s);
    PRG_CUDA(cudaEventRecord(ws.eva, s));
    for (uint32_t k = 0; k < iters; k++) launch_iteration(m, g.weighted, a[k & 1], ws.cfg[m], s);
    PRG_CUDA(cudaEventRecord(ws.evb, s));
    PRG_CUDA(cudaEventSynchronize(ws.evb));
    float ms = 0.f;
    PRG_CUDA(cudaEventElapsedTime(&ms, ws.eva, ws.evb));
    return (double)ms / (double)std::max<uint32_t>(iters, 1u);
}

void solve(const DeviceGraph &g, Workspace &ws, const SolveOpts &o_in, const double *d_t, double *d_out,
           SolveStats &st, cudaStream_t s) {
    st = SolveStats{};
    workspace_ensure(ws, g, s);
    PRG_CUDA(cudaMemsetAsync(ws.hub_ticket, 0, std::max<uint64_t>(g.nhub, 1) * 4, s));
    PRG_CUDA(cudaEventRecord(ws.ev0, s));
    // Vectors cross into internal ids here: the teleport vector always lives
    // in ws.t64 (so captured graphs stay valid), a start vector goes straight
    // into x64[0], and the result is gathered back to caller ids at the end.
    SolveOpts o = o_in;
    const double *t = nullptr;
    if (d_t) {
        if (g.perm) {
            gather_f64(ws.t64, d_t, g.perm, g.n, s);
            st.kernel_launches += 1u;
        } else if (d_t != ws.t64) {
            PRG_CUDA(cudaMemcpyAsync(ws.t64, d_t, (uint64_t)g.n * 8, cudaMemcpyDeviceToDevice, s));
        }
        t = ws.t64;
    }
    if (o.d_start) {
        if (g.perm) {
            gather_f64(ws.x64[1], o.d_start, g.perm, g.n, s);
            st.kernel_launches += 1u;
            o.d_start = ws.x64[1];
        }
    }
    double *out = g.perm ? ws.out_tmp : d_out;
    if (o.precision == 1 && o.inner == 1) solve_refined(g, ws, o, t, out, st, s);
    else if (o.precision == 1) solve_krylov(g, ws, o, t, out, st, s, false, false);
    else if (o.precision == 2) solve_krylov(g, ws, o, t, out, st, s, true, false);
    else if (o.precision == 3) solve_krylov(g, ws, o, t, out, st, s, true, true);
    else solve_fp64(g, ws, o, t, out, st, s);
    if (g.perm) {
        gather_f64(d_out, ws.out_tmp, g.iperm, g.n, s);
        st.kernel_launches += 1u;
    }
    PRG_CUDA(cudaEventRecord(ws.ev1, s));
    PRG_CUDA(cudaEventSynchronize(ws.ev1));
    float ms = 0.f;
    PRG_CUDA(cudaEventElapsedTime(&ms, ws.ev0, ws.ev1));
    st.solve_ms = ms;
    PRG_CUDA(cudaGetLastError());
}

}  // namespace prg
