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

// Options of the shifted power iteration x' = shift x + A x over g's in-CSR.
struct EigOpts {
    bool rowsum_seed = false;    // start from |row sums| of A (all ones when zero) instead of ones
    double eps = 1e-14;          // L1 stop
    bool auto_shift = false;     // shift = max(max row sum of |A|, 1) + 1 (else 1)
    bool zero_fallback = false;  // eigenvalue <= 1e-12 -> zero vector, eigenvalue 0
    bool negative = false;       // some weight < 0: signed pivot, a zero row sum over a non-empty row seeds 1,
                                 // no clamping and no zero fallback
    bool signed_seed = false;    // keep the sign of the row sums in the seed (the HITS form)
};

// Power iteration on g: x (caller ids) into d_out[n]; eigenvalue = x.Ax / x.x
// (A weighted when g is), negatives clamped.  For an undirected g the row
// sums are the vertex strengths.
Result eigenvector_centrality(const DeviceGraph &g, Workspace &ws, double *d_out, cudaStream_t s, const EigOpts &o);
Result eigenvector_centrality(const DeviceGraph &g, Workspace &ws, double *d_out, cudaStream_t s,
                              bool strength_seed = false, double eps = 1e-14);

// True when the directed graph g has no cycle.
bool is_dag(const DeviceGraph &g, cudaStream_t s);

// Directed eigenvector centrality over g's in-CSR (eigenvector.rs:539-756,
// non-negative weights): Out mode on a graph is this on the graph itself, In
// mode this on its reverse.  A DAG gives 1 where g's out-strength is 0.
Result eigenvector_directed(const DeviceGraph &g, Workspace &ws, double *d_out, cudaStream_t s, bool negative = false);

// Directed graph g and its reverse rev (both without relabelling):
// hub and authority vectors into d_hub / d_auth; eigenvalue of A A^T.
// The seed is the out-degree, or the out-strength when g is weighted.
Result hits_directed(const DeviceGraph &g, Workspace &ws, const DeviceGraph &rev, Workspace &wsr, double *d_hub,
                     double *d_auth, cudaStream_t s, bool negative = false);

// Infomap's flow model (infomap.rs:299-355) on g (directed or undirected,
// arc weights when g is weighted): node flows into d_out[n] (caller ids).
// d_t: teleport weights in g's internal ids, summing to 1 (null = 1/n).
// Requires n >= 2.
Result infomap_flow(const DeviceGraph &g, Workspace &ws, const double *d_t, double *d_out, cudaStream_t s);

}  // namespace eig
}  // namespace prg
