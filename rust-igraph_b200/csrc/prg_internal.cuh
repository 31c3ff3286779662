// prg_internal.cuh — shared definitions for the B200 PageRank library.
//
// Device layout of a graph (pull / in-arc CSR, built once per handle):
//   row_ptr  u32[n+1]      arcs of row v are [row_ptr[v], row_ptr[v+1])
//   col      u32[arcs+pad] source vertex of each in-arc, rows in edge-id order
//   w64/w32  f64/f32[arcs] per-arc weight (weighted graphs only)
//   deg      u32[n]        out-degree as rust-igraph counts it (graph.rs:877-900)
//   dval     f64[n]        out-degree or out-strength as a double (divisor)
//   inv32    f32[n]        1/dval in FP32 (0 for dangling vertices)
//   rb       uint4[nrb]    row-blocks, the SpMV work units of one warp:
//                          {row_begin, row_end | 0x80000000|hub, arc_begin, arc_end}
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

namespace prg {

constexpr int kThreads = 256;         // threads per block for all hot kernels
constexpr int kWarps = kThreads / 32;
constexpr uint32_t kWarpBuf = 512;    // products staged per warp (shared memory)
constexpr uint32_t kRowCap = 32;      // rows per stream row-block (one lane per row)
constexpr uint32_t kCapW = 256;       // default stream window: a new row-block starts when a row's
                                      // first arc crosses a multiple of kCapW
constexpr uint32_t kShortMax = 256;   // default: rows with more arcs are handled by a whole warp
constexpr uint32_t kSplit = 8192;     // default: rows with more arcs are split into chunks
constexpr uint32_t kColPad = 16;      // extra u32 slots after col[] for aligned vector loads
constexpr uint32_t kChunkFlag = 0x80000000u;

// Per-solve device control block.  Scalars that an iteration reads and the
// next one writes are double-buffered by launch parity.
struct Ctl {
    double dsum[2];       // dangling mass of the vector a launch of parity p reads
    double diff;          // L1 change of the last completed loop iteration
    double thr;           // loop iterations stop once diff < thr
    double rnorm;         // L1 norm of the last FP64 residual
    double gsum;          // sum of the last residual pass's g = G(x) (or of x in prepare)
    double rho;           // inner threshold = max(rho * rnorm, floor_abs)
    double floor_abs;
    uint32_t groups_done; // reduction groups finished in the current launch
    uint32_t iters;       // loop iterations completed since the last reset
    uint32_t max_iter;    // loop iteration cap
    int32_t done;         // 1 once converged or capped: later loop launches return at once
    int32_t parity_last;  // parity of the launch that produced the newest vector
    int32_t status;       // 0 ok; nonzero = device-detected error
    uint32_t total_iters; // all loop iterations (never reset by the kernels)
    uint32_t resid_passes;
};

struct Hub {
    uint32_t row;
    uint32_t nchunks;
    uint32_t first_rb;
    uint32_t pad;
};

std::string cuda_msg(cudaError_t e, const char *what);

}  // namespace prg

#define PRG_CUDA(call)                                                 \
    do {                                                               \
        cudaError_t e_ = (call);                                       \
        if (e_ != cudaSuccess) throw prg::CudaError(e_, #call);        \
    } while (0)

namespace prg {
struct CudaError {
    cudaError_t err;
    const char *what;
    CudaError(cudaError_t e, const char *w) : err(e), what(w) {}
};
}  // namespace prg
