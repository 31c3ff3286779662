// handle.cuh — the object behind the opaque prg_graph handle of the C ABI.
#pragma once
#include <cuda_runtime.h>

#include "graph.cuh"
#include "solver.cuh"

struct prg_graph {
    prg::DeviceGraph g;
    prg::Workspace ws;
    cudaStream_t stream = nullptr;
    double *d_reset = nullptr;  // normalised reset staging (n doubles)
    double *d_out = nullptr;    // output staging (n doubles)
    double *d_start = nullptr;  // warm-start staging
};
