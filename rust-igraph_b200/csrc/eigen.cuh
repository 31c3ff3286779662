// eigen.cuh — eigenvector centrality and HITS on the resident CSR.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "graph.cuh"

namespace prg {
struct Workspace;
namespace eig {

struct Result {
    uint32_t iterations = 0;
    double eigenvalue = 0.0;
};

// Undirected graph g: x (caller ids) into d_out[n]; eigenvalue = x.Ax / x.x.
Result eigenvector_centrality(const DeviceGraph &g, Workspace &ws, double *d_out, cudaStream_t s);

// Directed graph g and its reverse rev (both without relabelling):
// hub and authority vectors into d_hub / d_auth; eigenvalue of A A^T.
Result hits_directed(const DeviceGraph &g, Workspace &ws, const DeviceGraph &rev, Workspace &wsr, double *d_hub,
                     double *d_auth, cudaStream_t s);

}  // namespace eig
}  // namespace prg
