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

// Undirected graph g: x (caller ids) into d_out[n]; eigenvalue = x.Ax / x.x
// (A weighted when g is).  strength_seed: start from the vertex strengths
// (all ones when they are all zero) instead of ones; eps: L1 stop.
Result eigenvector_centrality(const DeviceGraph &g, Workspace &ws, double *d_out, cudaStream_t s,
                              bool strength_seed = false, double eps = 1e-14);

// Directed graph g and its reverse rev (both without relabelling):
// hub and authority vectors into d_hub / d_auth; eigenvalue of A A^T.
// The seed is the out-degree, or the out-strength when g is weighted.
Result hits_directed(const DeviceGraph &g, Workspace &ws, const DeviceGraph &rev, Workspace &wsr, double *d_hub,
                     double *d_auth, cudaStream_t s);

// Infomap's flow model (infomap.rs:299-355) on g (directed or undirected,
// arc weights when g is weighted): node flows into d_out[n] (caller ids).
// d_t: teleport weights in g's internal ids, summing to 1 (null = 1/n).
// Requires n >= 2.
Result infomap_flow(const DeviceGraph &g, Workspace &ws, const double *d_t, double *d_out, cudaStream_t s);

}  // namespace eig
}  // namespace prg
