// noalloc.cu — an allocation-free FP64 solve on a resident graph.
//
// Who needs it: code that must not allocate device memory at solve time —
// a real-time loop that reserves all memory up front, a host thread running
// under a memory budget enforced by another framework's caching allocator,
// or a process that calls in while the device is nearly full.  A
// cudaMalloc (or stream-ordered allocation) there either fails, stalls the
// device, or steps outside the caller's accounting.
//
// Every piece of solve scratch (iterate ping-pong buffers, teleport copy,
// reduction partials, hub tickets, control block) lives in one file-scope
// __device__ array of kNaBytes (about 26.6 MiB) that every GPU loading the
// library holds until the process exits.  The caller passes the graph
// handle (created earlier, when allocating was allowed), an optional
// normalised teleport vector and the output buffer, all in device memory.
// Limits: n <= 524,288 vertices, <= 262,144 row-blocks, <= 8,192 hub rows,
// and the FP64 path only; larger inputs are rejected with
// PRG_ERR_INVALID_ARGUMENT.
//
// CUDA loads a module lazily, on the first use of anything in it, and that
// load is when the device allocates the module's code and its __device__
// arrays.  So the set-up happens when a graph within the limits below is
// created (prg_graph_create*, prg_read_edgelist), a point where the caller
// is allocating anyway: noalloc_prepare() looks up the array's device
// address with cudaGetSymbolAddress (host code cannot use the symbol
// itself: in host code its name is only a stand-in), which loads this
// module and its array, and it loads every kernel the solve launches.  The
// solve itself then allocates nothing, its first call on a device
// included.  It still looks the address up on every call (cheap once the
// module is loaded), so a context torn down and made again is never handed
// a stale address.  All calls share the one array and it keeps the last
// call's contents, so the parts that must start at zero (control block, hub
// tickets) are cleared at the start of each call, and calls that overlap on
// the GPU — on two streams, or from two threads — race on the array.
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstring>
#include <string>

#include "../../include/prg_b200.h"
#include "handle.cuh"
#include "spmv.cuh"

namespace prg {
void set_last_error(const std::string &msg);
}

namespace {

constexpr uint32_t kNaMaxN = 1u << 19;      // vertices
constexpr uint32_t kNaMaxRb = 1u << 18;     // row-blocks
constexpr uint32_t kNaMaxHub = 8192;        // hub rows
constexpr uint32_t kNaMaxBlocks = 4096;     // persistent-grid / prepare blocks
constexpr size_t kOffCtl = 0;
constexpr size_t kOffBlk = 256;
constexpr size_t kOffHubRec = kOffBlk + (size_t)kNaMaxBlocks * 32;
constexpr size_t kOffHubTk = kOffHubRec + (size_t)kNaMaxHub * 32;
constexpr size_t kOffChunk = kOffHubTk + (size_t)kNaMaxHub * 4;
constexpr size_t kOffVec = kOffChunk + (size_t)kNaMaxRb * 8;
constexpr size_t kVec = (size_t)kNaMaxN * 8;  // one FP64 vector slot
constexpr size_t kNaBytes = kOffVec + 6 * kVec;
static_assert(sizeof(prg::Ctl) <= 256, "control block slot");

}  // namespace

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNaBytes];

namespace {

int32_t na_fail(int32_t code, const std::string &m) {
    prg::set_last_error(m);
    return code;
}

// Device address of the scratch array on the current device.  The host-side
// name is not a device pointer; the lookup also loads this module (and so
// the array) if nothing has loaded it yet.
void *scratch_address(cudaError_t *err) {
    void *p = nullptr;
    *err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    return *err == cudaSuccess ? p : nullptr;
}

bool within_limits(const prg::DeviceGraph &g) {
    return g.n <= kNaMaxN && g.nrb <= kNaMaxRb && g.nhub <= kNaMaxHub;
}

}  // namespace

namespace prg {

// Called when a graph handle is created (api.cu), while allocating is
// allowed: loads this module's scratch array and every kernel the
// allocation-free solve launches, so that solve allocates nothing later.
// Graphs beyond the limits skip it (the solve rejects them anyway).
void noalloc_prepare(const DeviceGraph &g) {
    if (!within_limits(g) || g.n < 2) return;
    cudaError_t e = cudaSuccess;
    if (!scratch_address(&e)) throw CudaError(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    iteration_config(MODE_PLAIN64, g.weighted, 0, g.blocks_per_sm, g.n);
    iteration_config(MODE_PPR64, g.weighted, 0, g.blocks_per_sm, g.n);
    preload_fp64_support();
}

}  // namespace prg

extern "C" int32_t prg_solve_noalloc(prg_graph *h, const prg_options *opt, const double *d_reset, double *d_out,
                                     prg_stats *st) {
    prg::set_last_error("");
    if (st) std::memset(st, 0, sizeof(*st));
    if (!h) return na_fail(PRG_ERR_INVALID_ARGUMENT, "null graph handle");
    prg_options o;
    prg_default_options(&o);
    if (opt) o = *opt;
    const prg::DeviceGraph &g = h->g;
    const uint32_t n = g.n;
    // the checks prg_solve_device makes, then this entry point's own limits
    if (o.precision < PRG_PRECISION_FP64 || o.precision > PRG_PRECISION_LINSYS)
        return na_fail(PRG_ERR_INVALID_ARGUMENT, "unknown precision " + std::to_string(o.precision));
    if (o.stop != PRG_STOP_SUCCESSIVE && o.stop != PRG_STOP_ERROR_BOUND)
        return na_fail(PRG_ERR_INVALID_ARGUMENT, "unknown stop rule " + std::to_string(o.stop));
    if (!(o.eps > 0.0)) return na_fail(PRG_ERR_INVALID_ARGUMENT, "eps must be positive");
    if (o.precision != PRG_PRECISION_FP64)
        return na_fail(PRG_ERR_INVALID_ARGUMENT, "the allocation-free solve runs the FP64 path only");
    if (!(o.damping > 0.0 && o.damping < 1.0))
        return na_fail(PRG_ERR_INVALID_ARGUMENT, "damping must be in (0, 1)");
    if (n > kNaMaxN)
        return na_fail(PRG_ERR_INVALID_ARGUMENT, "graph has " + std::to_string(n) +
                                                     " vertices; the allocation-free solve supports at most " +
                                                     std::to_string(kNaMaxN));
    if (g.nrb > kNaMaxRb || g.nhub > kNaMaxHub)
        return na_fail(PRG_ERR_INVALID_ARGUMENT, "graph has " + std::to_string(g.nrb) + " row-blocks and " +
                                                     std::to_string(g.nhub) +
                                                     " hub rows; the allocation-free solve supports at most " +
                                                     std::to_string(kNaMaxRb) + " and " + std::to_string(kNaMaxHub));
    cudaStream_t s = h->stream;
    try {
        int dev = 0;
        PRG_CUDA(cudaGetDevice(&dev));
        if (dev != g.device) return na_fail(PRG_ERR_INVALID_ARGUMENT, "the graph lives on another device");
        if (n == 0) return PRG_OK;
        if (n == 1) {
            // a single vertex holds all the mass (pagerank.rs:62-64); the copy
            // is ordered after earlier work on the graph's stream
            static const double one = 1.0;
            PRG_CUDA(cudaMemcpyAsync(d_out, &one, 8, cudaMemcpyHostToDevice, s));
            PRG_CUDA(cudaStreamSynchronize(s));
            return PRG_OK;
        }
        cudaError_t e = cudaSuccess;
        unsigned char *base = static_cast<unsigned char *>(scratch_address(&e));
        if (!base) return na_fail(PRG_ERR_CUDA, std::string("cuda: scratch lookup: ") + cudaGetErrorString(e));
        prg::Ctl *ctl = reinterpret_cast<prg::Ctl *>(base + kOffCtl);
        double4 *blk = reinterpret_cast<double4 *>(base + kOffBlk);
        double4 *hub_rec = reinterpret_cast<double4 *>(base + kOffHubRec);
        uint32_t *hub_tk = reinterpret_cast<uint32_t *>(base + kOffHubTk);
        double *chunk = reinterpret_cast<double *>(base + kOffChunk);
        double *x0 = reinterpret_cast<double *>(base + kOffVec);
        double *x1 = reinterpret_cast<double *>(base + kOffVec + kVec);
        double *xt0 = reinterpret_cast<double *>(base + kOffVec + 2 * kVec);
        double *xt1 = reinterpret_cast<double *>(base + kOffVec + 3 * kVec);
        double *t64 = reinterpret_cast<double *>(base + kOffVec + 4 * kVec);
        double *res_tmp = reinterpret_cast<double *>(base + kOffVec + 5 * kVec);

        const bool ppr = d_reset != nullptr;
        const int mode = ppr ? prg::MODE_PPR64 : prg::MODE_PLAIN64;
        const prg::LaunchCfg cfg = prg::iteration_config(mode, g.weighted, false, g.blocks_per_sm, n);
        if (cfg.grid > kNaMaxBlocks)
            return na_fail(PRG_ERR_INVALID_ARGUMENT, "device needs more persistent blocks than the scratch holds");

        // zero what the kernels expect at zero; then the control block
        PRG_CUDA(cudaMemsetAsync(base, 0, 256, s));
        PRG_CUDA(cudaMemsetAsync(hub_tk, 0, (size_t)kNaMaxHub * 4, s));
        prg::Ctl c;
        std::memset(&c, 0, sizeof(c));
        c.thr = o.stop == PRG_STOP_ERROR_BOUND ? o.eps * (1.0 - o.damping) / o.damping : o.eps;
        c.max_iter = o.max_iter;
        PRG_CUDA(cudaMemcpyAsync(ctl, &c, sizeof(c), cudaMemcpyHostToDevice, s));

        const double *t = nullptr;
        if (ppr) {
            if (g.perm) {
                prg::gather_f64(t64, d_reset, g.perm, n, s);
                t = t64;
            } else {
                t = d_reset;
            }
        }
        if (o.start) {
            // a caller-supplied start vector in device memory, used as given
            // (as prg_solve_device does), mapped to internal ids
            if (g.perm) prg::gather_f64(x0, o.start, g.perm, n, s);
            else PRG_CUDA(cudaMemcpyAsync(x0, o.start, (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
        } else {
            prg::launch_fill_start(x0, t, n, s);
        }
        prg::launch_prepare64(g, x0, nullptr, xt0, ctl, 0, blk, s);

        prg::IterArgs a0;
        std::memset(&a0, 0, sizeof(a0));
        a0.row_ptr = g.row_ptr;
        a0.col = g.col;
        a0.w64 = g.w64;
        a0.w32 = g.w32;
        a0.dval = g.dval;
        a0.inv32 = g.inv32;
        a0.rb = g.rb;
        a0.hubs = g.hubs;
        a0.nrb = g.nrb;
        a0.nhub = g.nhub;
        a0.n = n;
        a0.damping = o.damping;
        a0.inv_n = 1.0 / (double)n;
        a0.ctl = ctl;
        a0.blk_part = blk;
        a0.chunk_part = chunk;
        a0.hub_rec = hub_rec;
        a0.hub_ticket = hub_tk;
        a0.t64 = t;
        prg::IterArgs a1 = a0;
        a0.parity = 0;
        a0.x64_in = x0;
        a0.xt64_in = xt0;
        a0.x64_out = x1;
        a0.xt64_out = xt1;
        a1.parity = 1;
        a1.x64_in = x1;
        a1.xt64_in = xt1;
        a1.x64_out = x0;
        a1.xt64_out = xt0;

        // iterations launched in groups of 8; the kernels stop themselves
        // (Ctl::done), the host reads the control block between groups
        prg::Ctl hc;
        std::memset(&hc, 0, sizeof(hc));
        uint32_t launched = 0;
        while (launched < o.max_iter) {
            for (int k = 0; k < 4; k++) {
                prg::launch_iteration(mode, g.weighted, a0, cfg, s);
                prg::launch_iteration(mode, g.weighted, a1, cfg, s);
            }
            launched += 8;
            PRG_CUDA(cudaMemcpyAsync(&hc, ctl, sizeof(hc), cudaMemcpyDeviceToHost, s));
            PRG_CUDA(cudaStreamSynchronize(s));
            if (hc.done) break;
        }
        if (o.max_iter == 0) {
            PRG_CUDA(cudaMemcpyAsync(&hc, ctl, sizeof(hc), cudaMemcpyDeviceToHost, s));
            PRG_CUDA(cudaStreamSynchronize(s));
        }
        const double *res = hc.iters == 0 ? x0 : (hc.parity_last == 0 ? x1 : x0);
        if (g.perm) {
            PRG_CUDA(cudaMemcpyAsync(res_tmp, res, (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
            prg::gather_f64(d_out, res_tmp, g.iperm, n, s);
        } else {
            PRG_CUDA(cudaMemcpyAsync(d_out, res, (size_t)n * 8, cudaMemcpyDeviceToDevice, s));
        }
        PRG_CUDA(cudaStreamSynchronize(s));
        if (st) {
            std::memset(st, 0, sizeof(*st));
            st->iterations = st->fp64_passes = hc.iters;
            st->last_diff = hc.diff;
            st->residual_l1 = hc.diff;
            st->error_bound = hc.diff * o.damping / (1.0 - o.damping);
            st->arcs = g.arcs;
            st->n_dangling = g.n_dangling;
            st->build_ms = g.build_ms;
        }
        return PRG_OK;
    } catch (const prg::CudaError &ce) {
        return na_fail(PRG_ERR_CUDA, std::string("cuda: ") + cudaGetErrorString(ce.err) + " (" + ce.what + ")");
    } catch (...) {
        return na_fail(PRG_ERR_INTERNAL, "unexpected exception");
    }
}
