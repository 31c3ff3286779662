// ppr_batch.cuh — batched personalized PageRank (FP32 SpMM, per-column freeze).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "graph.cuh"

namespace prg {

struct BatchStats {
    std::vector<uint32_t> column_iters;  // iterations each column ran before it froze
    std::vector<double> column_diff;     // its last successive L1 change
    uint64_t column_iterations = 0;      // sum of column_iters
    uint32_t max_iters = 0;
    uint32_t tiles = 0;
    uint32_t vec = 1;  // tile width = 32 * vec columns
    uint32_t grid = 0;
    uint32_t chebyshev = 0;  // 1: Chebyshev steps (undirected graph), 0: plain power steps
    uint32_t kernel_launches = 0;
    float ms = 0.f;
};

// K columns; seeds of column k are seeds[seed_offsets[k] .. seed_offsets[k+1])
// (caller vertex ids).  d_out: device float[n * K], row-major by caller id.
// Returns 0 or a prg status code (7 = a grid barrier timed out).
int ppr_batch(const DeviceGraph &g, uint32_t K, const uint64_t *seed_offsets, const uint32_t *seeds, double damping,
              double tol, uint32_t max_iter, uint32_t vec, float *d_out, BatchStats &st, cudaStream_t s);

}  // namespace prg
