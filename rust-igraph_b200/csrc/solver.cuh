// solver.cuh — host orchestration of a PageRank solve on a resident graph.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <map>

#include "graph.cuh"
#include "spmv.cuh"

namespace prg {

struct SolveOpts {
    double damping = 0.85;
    double eps = 1e-10;
    uint32_t max_iter = 1000;
    int precision = 0;      // 0 FP64 power, 1 FP32-refined, 2 FP64 Krylov, 3 pagerank_linsys
    int stop = 0;           // 0 successive (reference), 1 error bound
    int normalise = 1;
    const double *d_start = nullptr;  // device start vector (warm start) or null
    double refine_switch = 5e-7;      // refined (Richardson inner): FP64 steps until the successive change is below this
    int inner = 0;                    // refined: 0 BiCGStab inner solve, 1 Richardson (power-style) correction
};

struct KrylovWs;  // krylov.cu

struct SolveStats {
    uint32_t iterations = 0, fp64_passes = 0, fp32_passes = 0, residual_passes = 0;
    double last_diff = 0, residual_l1 = 0, error_bound = 0, solve_ms = 0;
    uint32_t kernel_launches = 0;
    double fp32_ms = 0, fp64_ms = 0;
    double spmv_ms = 0;          // SpMV launches that did work (power graphs / Krylov matvecs)
    uint32_t spmv_launches = 0;
};

// Reusable per-handle solve buffers and captured CUDA graphs.
struct Workspace {
    bool ready = false;
    uint32_t n = 0, nrb = 0, nhub = 0;
    LaunchCfg cfg[kModes];  // persistent launch shape per iteration mode
    double *x64[2] = {nullptr, nullptr};
    double *xt64[2] = {nullptr, nullptr};
    float *e32[2] = {nullptr, nullptr};
    float *et32[2] = {nullptr, nullptr};
    float *b32 = nullptr;
    double *t64 = nullptr;
    float *t32 = nullptr;
    double *out_tmp = nullptr;  // result in internal ids before un-permuting
    Ctl *ctl = nullptr;
    Ctl *h_ctl = nullptr;  // pinned mirror
    double4 *blk_part = nullptr;   // per-block records (iteration and prepare kernels)
    double4 *hub_rec = nullptr;
    double *chunk_part = nullptr;
    uint32_t *hub_ticket = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr, eva = nullptr, evb = nullptr;
    std::map<uint64_t, cudaGraphExec_t> graphs;
    const void *graphs_rb = nullptr;  // row-block list the cached graphs were captured with
    int unroll = 8;  // iteration pairs per graph launch
    KrylovWs *kry = nullptr;  // Krylov vectors, allocated on first use
    SegIndex seg;             // row-end index of the tile-segmented FP32 Krylov matvec (when used)
};

void workspace_ensure(Workspace &ws, const DeviceGraph &g, cudaStream_t s);

// Device time of one iteration of `mode` (ms), averaged over `iters`
// back-to-back launches that never converge (autotuner probe).
double time_iterations(const DeviceGraph &g, Workspace &ws, int mode, uint32_t iters, cudaStream_t s);
void workspace_free(Workspace &ws, cudaStream_t s);

// Solves on graph g.  d_t: normalised teleport/reset vector on the device
// (null = uniform 1/n).  d_out: device double[n].
void solve(const DeviceGraph &g, Workspace &ws, const SolveOpts &o, const double *d_t, double *d_out,
           SolveStats &st, cudaStream_t s);

// Linear-system solve (krylov.cu): BiCGStab inner solves against FP64
// residual passes.  fp64_inner = false is the FP32-refined form; linsys
// applies pagerank_linsys()'s 2-norm stop rule and returns the iterate.
void solve_krylov(const DeviceGraph &g, Workspace &ws, const SolveOpts &o, const double *d_t, double *d_out,
                  SolveStats &st, cudaStream_t s, bool fp64_inner, bool linsys);
void krylov_free(KrylovWs *&k, cudaStream_t s);
// One FP32 Krylov matvec through kernel 0 (row-block), 1 or 2 (tile-segmented),
// for tests and measurement (krylov.cu).
void matvec32_probe(const DeviceGraph &g, Workspace &ws, int kernel, const float *p, const float *pt, double dz,
                    double damping, float *y, double dots[3], float *ms, cudaStream_t s);

// Pieces of the power-iteration driver the Krylov driver reuses (solver.cu).
IterArgs base_args(const DeviceGraph &g, Workspace &ws, double damping);
void read_ctl(Workspace &ws, cudaStream_t s);
const double *fp64_loop(const DeviceGraph &g, Workspace &ws, const SolveOpts &o, const double *d_t, double thr,
                        uint32_t max_iter, SolveStats &st, cudaStream_t s);
void to_f32(const double *a, float *b, uint32_t n, cudaStream_t s);

}  // namespace prg
