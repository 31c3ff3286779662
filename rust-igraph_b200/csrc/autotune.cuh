// autotune.cuh — per-graph autotuner (row-block shape, grid occupancy, batched tile width).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "graph.cuh"
#include "solver.cuh"

namespace prg {

struct TuneResult {
    uint32_t capw = 0, shortmax = 0, split = 0, blocks_per_sm = 0, batch_vec = 1;
    double default_ms = 0, best_ms = 0;  // FP64 + FP32 iteration time, before / after
    uint32_t tried = 0;
    bool from_cache = false;
    uint32_t seg_hot = 0, seg_hot64 = 0;  // segmented passes' hot prefixes (unweighted graphs)
    double seg_default_ms = 0, seg_best_ms = 0;
};

int autotune(DeviceGraph &g, Workspace &ws, cudaStream_t s, bool tune_batch, const char *cache_path, TuneResult &r);

}  // namespace prg
