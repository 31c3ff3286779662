// handle.cuh — the object behind the opaque prg_graph handle of the C ABI.
#pragma once
#include <cuda_runtime.h>

#include "graph.cuh"
#include "solver.cuh"

namespace prg {
// Loads the allocation-free solve's static scratch and kernels (noalloc.cu);
// called when a handle is created, while allocating is allowed.
void noalloc_prepare(const DeviceGraph &g);
}  // namespace prg

struct prg_graph {
    prg::DeviceGraph g;
    prg::Workspace ws;
    cudaStream_t stream = nullptr;
    double *d_reset = nullptr;  // normalised reset staging (n doubles)
    double *d_out = nullptr;    // output staging (n doubles)
    double *d_start = nullptr;  // warm-start staging
};
