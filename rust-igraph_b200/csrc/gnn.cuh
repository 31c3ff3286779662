// gnn.cuh — learned warm start network (see gnn.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "graph.cuh"

namespace prg {
namespace gnn {

int param_count();

struct Net {
    float *P = nullptr;  // FP32 master parameters
    float *G = nullptr;  // gradient
    float *m = nullptr, *v = nullptr;  // Adam moments
    void *w = nullptr;   // BF16 weight copies read by the forward pass
    unsigned char *buf = nullptr;  // per-vertex activations and gradients
    uint32_t buf_n = 0;
    int step = 0;

    void alloc(cudaStream_t s);
    void init(uint64_t seed, cudaStream_t s);
    void set_params(const float *host, cudaStream_t s);
    void get_params(float *host, cudaStream_t s) const;
    void ensure(uint32_t n, cudaStream_t s);
    void forward(const DeviceGraph &g, cudaStream_t s);
    // start vector in internal ids (sums to 1)
    void predict(const DeviceGraph &g, double *x_internal, cudaStream_t s);
    // loss and gradient (into G) for a target PageRank vector in internal ids
    double loss_grad(const DeviceGraph &g, const double *target_internal, cudaStream_t s);
    void adam(float lr, cudaStream_t s);
    void free(cudaStream_t s);
};

}  // namespace gnn
}  // namespace prg
