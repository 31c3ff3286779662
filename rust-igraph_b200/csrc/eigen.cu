// eigen.cu — eigenvector centrality and HITS hub/authority scores
// (unweighted) as max-normalised power iterations over the resident CSR.
//
//   eigenvector_centrality (undirected; eigenvector.rs:286-372):
//     x = 1; repeat x' = (A + I) x, x' /= max|x'| until sum|x' - x| < 1e-14
//     or 5000 iterations; eigenvalue = x.Ax / x.x; negatives clamped.
//   hub_and_authority_scores (hits.rs:122-230): directed graphs iterate
//     h' = A (A^T h) from the out-degrees (max-normalised), the eigenvalue is
//     max|h'|, until sum|h' - h| < 1e-12; authority = A^T h rescaled;
//     undirected graphs take the eigenvector centrality and (x.Ax/x.x)^2.
//
// One iteration is the adjacency product (iter_kernel<MODE_EIG64>, which
// also leaves per-block max |y| records), a normalise kernel (every block
// reduces the records in the same order, divides, and records its part of
// the L1 change) and a one-block check kernel that sums the parts and
// raises `done`.  All kernels return at once once `done` is set, so the
// host enqueues iterations ahead and polls a pinned copy of the state.
// A^T products gather over the in-CSR of the graph; A products over the
// in-CSR of the reversed graph (both built without relabelling, so they
// share vertex ids).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "eigen.cuh"
#include "prims.cuh"
#include "solver.cuh"

namespace prg {
namespace eig {

struct State {
    int32_t done;
    uint32_t iters;
    uint32_t max_iter;
    int32_t final_buf;  // buffer index holding the newest normalised iterate
    double diff, eps;
    double maxv;        // max |y| of the newest product (HITS eigenvalue)
    double pad;
};

constexpr unsigned kNB = 148u * 4u;
constexpr int kNT = 256;

__device__ __forceinline__ double3 recs3(const double4 *a, uint32_t na, const double4 *b, uint32_t nb) {
    // (max .x, sum .y, sum .z) in a fixed order; result in every thread
    __shared__ double sm[3][kNT / 32];
    __shared__ double out[3];
    double mx = 0.0, y = 0.0, z = 0.0;
    for (uint32_t i = threadIdx.x; i < na; i += kNT) {
        const double4 q = a[i];
        mx = fmax(mx, q.x);
        y += q.y;
        z += q.z;
    }
    for (uint32_t i = threadIdx.x; i < nb; i += kNT) {
        const double4 q = b[i];
        mx = fmax(mx, q.x);
        y += q.y;
        z += q.z;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
        y += __shfl_xor_sync(0xffffffffu, y, o);
        z += __shfl_xor_sync(0xffffffffu, z, o);
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) {
        sm[0][w] = mx;
        sm[1][w] = y;
        sm[2][w] = z;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < kNT / 32; k++) {
            mx = fmax(mx, sm[0][k]);
            y += sm[1][k];
            z += sm[2][k];
        }
        out[0] = mx;
        out[1] = y;
        out[2] = z;
    }
    __syncthreads();
    return make_double3(out[0], out[1], out[2]);
}

// x /= max (records of the product that wrote x), sum |x - xold| per block.
__global__ void __launch_bounds__(kNT) normalise_kernel(uint32_t n, const double4 *recs, uint32_t nrec,
                                                        const double4 *hub_rec, uint32_t nhub, double *x,
                                                        const double *xold, double4 *part, const State *st) {
    if (st && *(volatile const int32_t *)&st->done) return;
    const double mx = recs3(recs, nrec, hub_rec, nhub).x;
    double d = 0.0;
    for (uint32_t v = blockIdx.x * kNT + threadIdx.x; v < n; v += gridDim.x * kNT) {
        double xv = x[v];
        if (mx > 0.0) {
            xv /= mx;
            x[v] = xv;
        }
        if (xold) d += fabs(xv - xold[v]);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
    __shared__ double sh[kNT / 32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sh[w] = d;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < kNT / 32; k++) d += sh[k];
        part[blockIdx.x] = make_double4(d, mx, 0.0, 0.0);
    }
}

__global__ void check_kernel(const double4 *part, uint32_t nb, State *st, int32_t buf) {
    if (st->done) return;
    __shared__ double sh[32];
    double d = 0.0;
    for (uint32_t i = threadIdx.x; i < nb; i += blockDim.x) d += part[i].x;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) d += __shfl_xor_sync(0xffffffffu, d, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sh[w] = d;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < (int)(blockDim.x >> 5); k++) d += sh[k];
        const double mx = part[0].y;
        st->iters += 1u;
        st->diff = d;
        if (mx != 0.0) st->maxv = mx;  // the last non-zero scale (signed with negative weights)
        st->final_buf = buf;
        if (d < st->eps || st->iters >= st->max_iter) st->done = 1;
    }
}

__global__ void fill_kernel(double *x, uint32_t n, double v) {
    for (uint32_t i = blockIdx.x * kNT + threadIdx.x; i < n; i += gridDim.x * kNT) x[i] = v;
}

// x = out-degree (deg) or out-strength (dval; with negative weights (neg) a
// zero strength on a vertex with out-arcs gives 1) and block records
// (max |x|, 0, 0) for the normalisation
__global__ void degree_seed_kernel(const uint32_t *deg, const double *dval, uint32_t n, bool neg, double *x,
                                   double4 *recs) {
    double mx = 0.0;
    for (uint32_t i = blockIdx.x * kNT + threadIdx.x; i < n; i += gridDim.x * kNT) {
        x[i] = dval ? (dval[i] != 0.0 ? dval[i] : ((neg && deg[i] > 0u) ? 1.0 : 0.0)) : (double)deg[i];
        mx = fmax(mx, fabs(x[i]));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    __shared__ double sh[kNT / 32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sh[w] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < kNT / 32; k++) mx = fmax(mx, sh[k]);
        recs[blockIdx.x] = make_double4(mx, 0.0, 0.0, 0.0);
    }
}

// ---- signed pivot (negative weights; eigenvector.rs:464-476, hits.rs:399-411)
// The component of greatest |y|, the one with the smallest caller id (perm[i],
// or i) on ties, as the reference scans caller ids in order and keeps the
// first strict maximum.  (mag, id, value) records: a total order, so any
// reduction order gives the same pivot.
__device__ __forceinline__ bool pv_better(double m1, double i1, double m2, double i2) {
    return m1 > m2 || (m1 == m2 && i1 < i2);
}

__device__ __forceinline__ void pv_reduce_block(double &mag, double &id, double &val, double (*sm)[kNT / 32]) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double m2 = __shfl_xor_sync(0xffffffffu, mag, o), i2 = __shfl_xor_sync(0xffffffffu, id, o);
        const double v2 = __shfl_xor_sync(0xffffffffu, val, o);
        if (pv_better(m2, i2, mag, id)) {
            mag = m2;
            id = i2;
            val = v2;
        }
    }
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) {
        sm[0][w] = mag;
        sm[1][w] = id;
        sm[2][w] = val;
    }
    __syncthreads();
    if (threadIdx.x == 0)
        for (int k = 1; k < kNT / 32; k++)
            if (pv_better(sm[0][k], sm[1][k], mag, id)) {
                mag = sm[0][k];
                id = sm[1][k];
                val = sm[2][k];
            }
}

__global__ void __launch_bounds__(kNT) pivot_kernel(const double *y, uint32_t n, const uint32_t *perm, double4 *recs,
                                                    const State *st) {
    if (st && *(volatile const int32_t *)&st->done) return;
    __shared__ double sm[3][kNT / 32];
    double mag = -1.0, id = 4294967296.0, val = 0.0;
    for (uint32_t i = blockIdx.x * kNT + threadIdx.x; i < n; i += gridDim.x * kNT) {
        const double m = fabs(y[i]), c = (double)(perm ? perm[i] : i);
        if (pv_better(m, c, mag, id)) {
            mag = m;
            id = c;
            val = y[i];
        }
    }
    pv_reduce_block(mag, id, val, sm);
    if (threadIdx.x == 0) recs[blockIdx.x] = make_double4(mag, id, val, 0.0);
}

// x /= pivot (when the pivot is not 0), sum |x - xold| per block; records
// (change, pivot, 0, 0) as normalise_kernel's.
__global__ void __launch_bounds__(kNT) normalise_signed_kernel(uint32_t n, const double4 *recs, uint32_t nrec,
                                                               double *x, const double *xold, double4 *part,
                                                               const State *st) {
    if (st && *(volatile const int32_t *)&st->done) return;
    __shared__ double sm[3][kNT / 32];
    __shared__ double s_piv;
    double mag = -1.0, id = 4294967296.0, val = 0.0;
    for (uint32_t i = threadIdx.x; i < nrec; i += kNT) {
        const double4 q = recs[i];
        if (pv_better(q.x, q.y, mag, id)) {
            mag = q.x;
            id = q.y;
            val = q.z;
        }
    }
    pv_reduce_block(mag, id, val, sm);
    if (threadIdx.x == 0) s_piv = val;
    __syncthreads();
    const double piv = s_piv;
    double d = 0.0;
    for (uint32_t v = blockIdx.x * kNT + threadIdx.x; v < n; v += gridDim.x * kNT) {
        double xv = x[v];
        if (piv != 0.0) {
            xv /= piv;
            x[v] = xv;
        }
        if (xold) d += fabs(xv - xold[v]);
    }
    d = warp_sum(d);
    __shared__ double sh[kNT / 32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sh[w] = d;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < kNT / 32; k++) d += sh[k];
        part[blockIdx.x] = make_double4(d, piv, 0.0, 0.0);
    }
}

// ---- directed eigenvector centrality (eigenvector.rs:539-756)

// x[v] = |sum of row v's arc weights| (row length when unweighted; the sum
// itself when keep_sign), and with negative weights (neg) 1 for a zero sum
// over a non-empty row; one warp per row; records (max |x|, max sum of |w|
// over a row, 0, 0).
__global__ void __launch_bounds__(kNT) rowsum_seed_kernel(const uint32_t *row_ptr, const double *w64, uint32_t n,
                                                          bool keep_sign, bool neg, double *x, double4 *recs) {
    __shared__ double sm[2][kNT / 32];
    const uint32_t lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double mx = 0.0, mnorm = 0.0;
    for (uint32_t v = (blockIdx.x * kNT + threadIdx.x) >> 5; v < n; v += (gridDim.x * kNT) >> 5) {
        const uint32_t lo = row_ptr[v], hi = row_ptr[v + 1];
        double s = 0.0, sa = 0.0;
        if (w64) {
            for (uint32_t p = lo + lane; p < hi; p += 32) {
                s += w64[p];
                sa += fabs(w64[p]);
            }
            s = warp_sum(s);
            sa = warp_sum(sa);
        } else {
            s = sa = (double)(hi - lo);
        }
        if (lane == 0) {
            const double xv = s != 0.0 ? (keep_sign ? s : fabs(s)) : ((neg && hi > lo) ? 1.0 : 0.0);
            x[v] = xv;
            mx = fmax(mx, fabs(xv));
            mnorm = fmax(mnorm, sa);
        }
    }
    if (lane == 0) {
        sm[0][wid] = mx;
        sm[1][wid] = mnorm;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 1; k < kNT / 32; k++) {
            mx = fmax(mx, sm[0][k]);
            mnorm = fmax(mnorm, sm[1][k]);
        }
        recs[blockIdx.x] = make_double4(mx, mnorm, 0.0, 0.0);
    }
}

// DAG test: sinks are peeled round by round over the in-CSR (a vertex whose
// remaining out-degree reaches 0 joins the next frontier); every vertex is
// peeled exactly when the graph has no cycle.  A self-loop keeps its vertex.
__global__ void peel_init(const uint32_t *deg, uint32_t n, uint32_t *odeg, uint32_t *front, uint32_t *cnt) {
    for (uint32_t v = blockIdx.x * kNT + threadIdx.x; v < n; v += gridDim.x * kNT) {
        odeg[v] = deg[v];
        if (deg[v] == 0u) front[atomicAdd(cnt, 1u)] = v;
    }
}

__global__ void peel_round(const uint32_t *row_ptr, const uint32_t *col, uint32_t n, uint32_t *odeg,
                           const uint32_t *front_in, const uint32_t *cnt_in, uint32_t *front_out, uint32_t *cnt_out,
                           unsigned long long *removed) {
    const uint32_t k = *cnt_in;
    if (blockIdx.x == 0 && threadIdx.x == 0) *removed += k;
    for (uint32_t i = blockIdx.x * kNT + threadIdx.x; i < k; i += gridDim.x * kNT) {
        const uint32_t v = front_in[i];
        for (uint32_t p = row_ptr[v]; p < row_ptr[v + 1]; p++) {
            const uint32_t u = col[p];
            if (atomicSub(&odeg[u], 1u) == 1u) {
                const uint32_t slot = atomicAdd(cnt_out, 1u);
                if (slot < n) front_out[slot] = u;
            }
        }
    }
}

__global__ void zero_u32_kernel(uint32_t *p) { *p = 0u; }

// x[v] = 1 where the graph's own out-strength (dval) is 0, else 0.
__global__ void sentinel_kernel(const double *dval, uint32_t n, double *x) {
    for (uint32_t v = blockIdx.x * kNT + threadIdx.x; v < n; v += gridDim.x * kNT) x[v] = dval[v] == 0.0 ? 1.0 : 0.0;
}

// ---- Infomap flow model (infomap.rs:299-355)
constexpr double kTau = 0.15;

__device__ __forceinline__ double block_total(double v, double *sh) {
    v = warp_sum(v);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) sh[w] = v;
    __syncthreads();
    if (threadIdx.x == 0)
        for (int k = 1; k < kNT / 32; k++) v += sh[k];
    return v;  // valid in thread 0
}

// pr = 1/n, xt = pr / strength (0 for dangling), records (0, dangling sum).
__global__ void flow_init_kernel(uint32_t n, const double *dval, double *pr, double *xt, double4 *part) {
    __shared__ double sh[kNT / 32];
    const double p = 1.0 / (double)n;
    double ds = 0.0;
    for (uint32_t v = blockIdx.x * kNT + threadIdx.x; v < n; v += gridDim.x * kNT) {
        pr[v] = p;
        const double s = dval[v];
        xt[v] = s > 0.0 ? p / s : 0.0;
        if (s <= 0.0) ds += p;
    }
    ds = block_total(ds, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = make_double4(0.0, ds, 0.0, 0.0);
}

// buf[v] = tau t[v] + (1 - tau) link[v] + dangling t[v] in place over the
// product y = link, with the dangling sum from the last normalisation's
// records; records (0, sum of buf).
__global__ void __launch_bounds__(kNT) flow_epi_kernel(uint32_t n, double *y, const double *t, const double4 *dpart,
                                                       uint32_t ndp, double4 *spart, const State *st) {
    if (*(volatile const int32_t *)&st->done) return;
    __shared__ double sh[kNT / 32];
    const double ds = recs3(dpart, ndp, nullptr, 0).y;
    const double inv_n = 1.0 / (double)n;
    double sum = 0.0;
    for (uint32_t v = blockIdx.x * kNT + threadIdx.x; v < n; v += gridDim.x * kNT) {
        const double tv = t ? t[v] : inv_n;
        const double b = __dadd_rn(__dadd_rn(__dmul_rn(kTau, tv), __dmul_rn(1.0 - kTau, y[v])), __dmul_rn(ds, tv));
        y[v] = b;
        sum += b;
    }
    sum = block_total(sum, sh);
    if (threadIdx.x == 0) spart[blockIdx.x] = make_double4(0.0, sum, 0.0, 0.0);
}

// pr_new = buf / sum(buf) (unscaled when the sum is not positive), the L1
// change from pr_old, xt = pr_new / strength; records (change, dangling sum).
__global__ void __launch_bounds__(kNT) flow_norm_kernel(uint32_t n, const double *buf, const double4 *spart,
                                                        uint32_t nsp, const double *pr_old, double *pr_new, double *xt,
                                                        const double *dval, double4 *dpart, const State *st) {
    if (*(volatile const int32_t *)&st->done) return;
    __shared__ double sh[kNT / 32];
    const double s = recs3(spart, nsp, nullptr, 0).y;
    double d = 0.0, ds = 0.0;
    for (uint32_t v = blockIdx.x * kNT + threadIdx.x; v < n; v += gridDim.x * kNT) {
        const double p = s > 0.0 ? __ddiv_rn(buf[v], s) : buf[v];
        d += fabs(pr_old[v] - p);
        pr_new[v] = p;
        const double sv = dval[v];
        xt[v] = sv > 0.0 ? __ddiv_rn(p, sv) : 0.0;
        if (sv <= 0.0) ds += p;
    }
    d = block_total(d, sh);
    __syncthreads();
    ds = block_total(ds, sh);
    if (threadIdx.x == 0) dpart[blockIdx.x] = make_double4(d, ds, 0.0, 0.0);
}

__global__ void clamp_kernel(double *x, uint32_t n) {
    for (uint32_t i = blockIdx.x * kNT + threadIdx.x; i < n; i += gridDim.x * kNT)
        if (x[i] < 0.0) x[i] = 0.0;
}

// ---------------------------------------------------------------- host side

struct Product {
    const DeviceGraph *g;
    Workspace *ws;
};

static IterArgs product_args(const Product &pr, const double *x, double *y, double shift, double4 *recs,
                             const int32_t *done) {
    IterArgs a = base_args(*pr.g, *pr.ws, 0.0);
    a.x64_in = x;
    a.xt64_in = x;
    a.x64_out = y;
    a.shift = shift;
    a.kpart_out = recs;
    a.kdone = done;
    return a;
}

static void product(const Product &pr, const double *x, double *y, double shift, double4 *recs, const int32_t *done,
                    cudaStream_t s) {
    launch_iteration(MODE_EIG64, pr.g->weighted, product_args(pr, x, y, shift, recs, done), pr.ws->cfg[MODE_EIG64],
                     s);
}

template <class T>
static T *alloc(uint64_t count, cudaStream_t s) {
    void *p = nullptr;
    PRG_CUDA(cudaMallocAsync(&p, std::max<uint64_t>(count, 1) * sizeof(T), s));
    return (T *)p;
}
template <class T>
static void release(T *&p, cudaStream_t s) {
    if (p) cudaFreeAsync(p, s);
    p = nullptr;
}

// Runs iterations of `one(it)` (which enqueues one iteration ending in
// check_kernel) until st->done, polling one batch behind.
template <class F>
static void run_until_done(State *d_st, State *h_st, uint32_t max_iter, cudaStream_t s, F one) {
    cudaEvent_t ev[2];
    for (cudaEvent_t &e : ev) PRG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    const uint32_t per = 8;
    uint32_t it = 0, batch = 0;
    const uint32_t max_batches = max_iter / per + 3u;
    bool stop = false;
    try {
        while (!stop) {
            for (uint32_t i = 0; i < per && it < max_iter + per; i++) one(it++);
            const int slot = (int)(batch & 1u);
            PRG_CUDA(cudaMemcpyAsync(&h_st[slot], d_st, sizeof(State), cudaMemcpyDeviceToHost, s));
            PRG_CUDA(cudaEventRecord(ev[slot], s));
            if (batch > 0) {
                PRG_CUDA(cudaEventSynchronize(ev[slot ^ 1]));
                if (h_st[slot ^ 1].done) stop = true;
            }
            if (++batch >= max_batches) stop = true;
        }
        PRG_CUDA(cudaMemcpyAsync(&h_st[0], d_st, sizeof(State), cudaMemcpyDeviceToHost, s));
        PRG_CUDA(cudaStreamSynchronize(s));
    } catch (...) {
        for (cudaEvent_t &e : ev) cudaEventDestroy(e);
        throw;
    }
    for (cudaEvent_t &e : ev) cudaEventDestroy(e);
}

static double rayleigh(const Product &pr, const double *x, double *tmp, double4 *recs, cudaStream_t s) {
    product(pr, x, tmp, 0.0, recs, nullptr, s);
    const unsigned nb = pr.ws->cfg[MODE_EIG64].grid;
    const uint32_t nh = pr.ws->cfg[MODE_EIG64].hub_recs;  // 0 for the segmented product
    std::vector<double4> h(nb), hh(std::max<uint32_t>(nh, 1));
    PRG_CUDA(cudaMemcpyAsync(h.data(), recs, nb * sizeof(double4), cudaMemcpyDeviceToHost, s));
    if (nh) PRG_CUDA(cudaMemcpyAsync(hh.data(), pr.ws->hub_rec, nh * sizeof(double4), cudaMemcpyDeviceToHost, s));
    PRG_CUDA(cudaStreamSynchronize(s));
    double num = 0.0, den = 0.0;
    for (const double4 &q : h) {
        num += q.y;
        den += q.z;
    }
    for (uint32_t i = 0; i < nh; i++) {
        num += hh[i].y;
        den += hh[i].z;
    }
    return den > 0.0 ? num / den : 0.0;
}

// Seeds x with the absolute row sums of g's in-CSR (the strength the walk
// over each row sees) and max-normalises it; an all-zero seed becomes all
// ones.  Returns the largest row sum of |w| (the shift's row norm).
static double seed(const DeviceGraph &g, bool keep_sign, bool neg, double *x, double4 *recs, double4 *part,
                   cudaStream_t s) {
    rowsum_seed_kernel<<<kNB, kNT, 0, s>>>(g.row_ptr, g.weighted ? g.w64 : nullptr, g.n, keep_sign, neg, x, recs);
    PRG_CUDA(cudaGetLastError());
    std::vector<double4> h(kNB);
    PRG_CUDA(cudaMemcpyAsync(h.data(), recs, kNB * sizeof(double4), cudaMemcpyDeviceToHost, s));
    PRG_CUDA(cudaStreamSynchronize(s));
    double mx = 0.0, norm = 0.0;
    for (const double4 &q : h) {
        mx = std::max(mx, q.x);
        norm = std::max(norm, q.y);
    }
    if (mx == 0.0) fill_kernel<<<kNB, kNT, 0, s>>>(x, g.n, 1.0);
    else normalise_kernel<<<kNB, kNT, 0, s>>>(g.n, recs, kNB, nullptr, 0, x, nullptr, part, nullptr);
    PRG_CUDA(cudaGetLastError());
    return norm;
}

Result eigenvector_centrality(const DeviceGraph &g, Workspace &ws, double *d_out, cudaStream_t s,
                              bool strength_seed, double eps) {
    EigOpts o;
    o.rowsum_seed = strength_seed;
    o.eps = eps;
    return eigenvector_centrality(g, ws, d_out, s, o);
}

Result eigenvector_centrality(const DeviceGraph &g, Workspace &ws, double *d_out, cudaStream_t s, const EigOpts &o) {
    const bool strength_seed = o.rowsum_seed;
    const double eps = o.eps;
    Result r;
    const uint32_t n = g.n;
    workspace_ensure(ws, g, s);
    PRG_CUDA(cudaMemsetAsync(ws.hub_ticket, 0, std::max<uint64_t>(g.nhub, 1) * 4, s));
    const Product pr{&g, &ws};
    const unsigned grid = ws.cfg[MODE_EIG64].grid;
    double *x[2] = {alloc<double>(n, s), alloc<double>(n, s)};
    double4 *recs = alloc<double4>(std::max(grid, kNB), s), *part = alloc<double4>(kNB, s);
    double4 *pvrec = alloc<double4>(kNB, s);
    State *d_st = alloc<State>(1, s), *h_st = nullptr;
    PRG_CUDA(cudaMallocHost((void **)&h_st, 2 * sizeof(State)));
    try {
        State init;
        std::memset(&init, 0, sizeof(init));
        init.max_iter = 5000;
        init.eps = eps;
        PRG_CUDA(cudaMemcpyAsync(d_st, &init, sizeof(State), cudaMemcpyHostToDevice, s));
        double shift = 1.0;
        if (strength_seed) {
            const double norm = seed(g, o.signed_seed, o.negative, x[0], recs, part, s);
            if (o.auto_shift) shift = std::max(norm, 1.0) + 1.0;  // eigenvector.rs:627-643
        } else {
            fill_kernel<<<kNB, kNT, 0, s>>>(x[0], n, 1.0);
            PRG_CUDA(cudaGetLastError());
        }
        run_until_done(d_st, h_st, init.max_iter, s, [&](uint32_t it) {
            const int q = (int)(it & 1u);
            product(pr, x[q], x[q ^ 1], shift, recs, &d_st->done, s);
            if (o.negative) {
                pivot_kernel<<<kNB, kNT, 0, s>>>(x[q ^ 1], n, g.perm, pvrec, d_st);
                normalise_signed_kernel<<<kNB, kNT, 0, s>>>(n, pvrec, kNB, x[q ^ 1], x[q], part, d_st);
            } else {
                normalise_kernel<<<kNB, kNT, 0, s>>>(n, recs, grid, ws.hub_rec, ws.cfg[MODE_EIG64].hub_recs, x[q ^ 1],
                                                     x[q], part, d_st);
            }
            check_kernel<<<1, 256, 0, s>>>(part, kNB, d_st, q ^ 1);
            PRG_CUDA(cudaGetLastError());
        });
        r.iterations = h_st[0].iters;
        const double *xf = h_st[0].iters ? x[h_st[0].final_buf] : x[0];
        double *other = xf == x[0] ? x[1] : x[0];
        r.eigenvalue = rayleigh(pr, xf, other, recs, s);
        if (o.zero_fallback && !o.negative && r.eigenvalue <= 1e-12) {
            // eigenvector.rs:695-699: a (numerically) nilpotent matrix gives zeros
            r.eigenvalue = 0.0;
            fill_kernel<<<kNB, kNT, 0, s>>>(const_cast<double *>(xf), n, 0.0);
        }
        // negatives are numerical drift only with non-negative weights
        if (!o.negative) clamp_kernel<<<kNB, kNT, 0, s>>>(const_cast<double *>(xf), n);
        PRG_CUDA(cudaGetLastError());
        if (g.perm) gather_f64(d_out, xf, g.iperm, n, s);
        else PRG_CUDA(cudaMemcpyAsync(d_out, xf, (uint64_t)n * 8, cudaMemcpyDeviceToDevice, s));
        PRG_CUDA(cudaStreamSynchronize(s));
    } catch (...) {
        cudaStreamSynchronize(s);
        cudaFreeHost(h_st);
        throw;
    }
    cudaFreeHost(h_st);
    release(x[0], s);
    release(x[1], s);
    release(recs, s);
    release(part, s);
    release(pvrec, s);
    release(d_st, s);
    PRG_CUDA(cudaStreamSynchronize(s));
    return r;
}

bool is_dag(const DeviceGraph &g, cudaStream_t s) {
    const uint32_t n = g.n;
    if (n == 0) return true;
    uint32_t *odeg = alloc<uint32_t>(n, s), *front[2] = {alloc<uint32_t>(n, s), alloc<uint32_t>(n, s)};
    uint32_t *cnt = alloc<uint32_t>(2, s);
    unsigned long long *removed = alloc<unsigned long long>(1, s);
    PRG_CUDA(cudaMemsetAsync(cnt, 0, 8, s));
    PRG_CUDA(cudaMemsetAsync(removed, 0, 8, s));
    peel_init<<<kNB, kNT, 0, s>>>(g.deg, n, odeg, front[0], cnt);
    PRG_CUDA(cudaGetLastError());
    uint32_t h_next = 0;
    unsigned long long h_removed = 0;
    // every vertex enters a frontier at most once, so the frontiers are empty
    // after at most n + 1 rounds; the bound only guards against a broken count
    const uint64_t max_rounds = (uint64_t)n + 32u;
    for (uint64_t r = 0; r < max_rounds; r++) {
        const int c = (int)(r & 1u);
        peel_round<<<kNB, kNT, 0, s>>>(g.row_ptr, g.col, n, odeg, front[c], cnt + c, front[c ^ 1], cnt + (c ^ 1),
                                       removed);
        zero_u32_kernel<<<1, 1, 0, s>>>(cnt + c);
        PRG_CUDA(cudaGetLastError());
        if ((r & 15u) == 15u) {  // poll: empty frontier -> done
            PRG_CUDA(cudaMemcpyAsync(&h_next, cnt + (c ^ 1), 4, cudaMemcpyDeviceToHost, s));
            PRG_CUDA(cudaStreamSynchronize(s));
            if (h_next == 0u) break;
        }
    }
    PRG_CUDA(cudaMemcpyAsync(&h_removed, removed, 8, cudaMemcpyDeviceToHost, s));
    PRG_CUDA(cudaStreamSynchronize(s));
    release(odeg, s);
    release(front[0], s);
    release(front[1], s);
    release(cnt, s);
    release(removed, s);
    return h_removed == (unsigned long long)n;
}

Result eigenvector_directed(const DeviceGraph &g, Workspace &ws, double *d_out, cudaStream_t s, bool negative) {
    if (!negative && is_dag(g, s)) {  // eigenvector.rs:570-575, 721-756
        double *x = alloc<double>(g.n, s);
        sentinel_kernel<<<kNB, kNT, 0, s>>>(g.dval, g.n, x);
        PRG_CUDA(cudaGetLastError());
        if (g.perm) gather_f64(d_out, x, g.iperm, g.n, s);
        else PRG_CUDA(cudaMemcpyAsync(d_out, x, (uint64_t)g.n * 8, cudaMemcpyDeviceToDevice, s));
        release(x, s);
        PRG_CUDA(cudaStreamSynchronize(s));
        return Result{};
    }
    EigOpts o;
    o.rowsum_seed = true;
    o.eps = 1e-12;
    o.auto_shift = true;
    o.zero_fallback = true;
    o.negative = negative;
    return eigenvector_centrality(g, ws, d_out, s, o);
}

Result infomap_flow(const DeviceGraph &g, Workspace &ws, const double *d_t, double *d_out, cudaStream_t s) {
    Result r;
    const uint32_t n = g.n;
    workspace_ensure(ws, g, s);
    PRG_CUDA(cudaMemsetAsync(ws.hub_ticket, 0, std::max<uint64_t>(g.nhub, 1) * 4, s));
    const Product pr_{&g, &ws};
    const unsigned grid = ws.cfg[MODE_EIG64].grid;
    double *pr[2] = {alloc<double>(n, s), alloc<double>(n, s)};
    double *xt = alloc<double>(n, s), *y = alloc<double>(n, s);
    double4 *recs = alloc<double4>(std::max(grid, kNB), s), *spart = alloc<double4>(kNB, s);
    double4 *dpart = alloc<double4>(kNB, s);
    State *d_st = alloc<State>(1, s), *h_st = nullptr;
    PRG_CUDA(cudaMallocHost((void **)&h_st, 2 * sizeof(State)));
    try {
        State init;
        std::memset(&init, 0, sizeof(init));
        init.max_iter = 1000;
        init.eps = 1e-10;
        PRG_CUDA(cudaMemcpyAsync(d_st, &init, sizeof(State), cudaMemcpyHostToDevice, s));
        flow_init_kernel<<<kNB, kNT, 0, s>>>(n, g.dval, pr[0], xt, dpart);
        PRG_CUDA(cudaGetLastError());
        run_until_done(d_st, h_st, init.max_iter, s, [&](uint32_t it) {
            const int q = (int)(it & 1u);
            product(pr_, xt, y, 0.0, recs, &d_st->done, s);
            flow_epi_kernel<<<kNB, kNT, 0, s>>>(n, y, d_t, dpart, kNB, spart, d_st);
            flow_norm_kernel<<<kNB, kNT, 0, s>>>(n, y, spart, kNB, pr[q], pr[q ^ 1], xt, g.dval, dpart, d_st);
            check_kernel<<<1, 256, 0, s>>>(dpart, kNB, d_st, q ^ 1);
            PRG_CUDA(cudaGetLastError());
        });
        r.iterations = h_st[0].iters;
        const double *pf = h_st[0].iters ? pr[h_st[0].final_buf] : pr[0];
        if (g.perm) gather_f64(d_out, pf, g.iperm, n, s);
        else PRG_CUDA(cudaMemcpyAsync(d_out, pf, (uint64_t)n * 8, cudaMemcpyDeviceToDevice, s));
        PRG_CUDA(cudaStreamSynchronize(s));
    } catch (...) {
        cudaStreamSynchronize(s);
        cudaFreeHost(h_st);
        throw;
    }
    cudaFreeHost(h_st);
    release(pr[0], s);
    release(pr[1], s);
    release(xt, s);
    release(y, s);
    release(recs, s);
    release(spart, s);
    release(dpart, s);
    release(d_st, s);
    PRG_CUDA(cudaStreamSynchronize(s));
    return r;
}

Result hits_directed(const DeviceGraph &g, Workspace &ws, const DeviceGraph &rev, Workspace &wsr, double *d_hub,
                     double *d_auth, cudaStream_t s, bool negative) {
    Result r;
    const uint32_t n = g.n;
    workspace_ensure(ws, g, s);
    workspace_ensure(wsr, rev, s);
    PRG_CUDA(cudaMemsetAsync(ws.hub_ticket, 0, std::max<uint64_t>(g.nhub, 1) * 4, s));
    PRG_CUDA(cudaMemsetAsync(wsr.hub_ticket, 0, std::max<uint64_t>(rev.nhub, 1) * 4, s));
    const Product pin{&g, &ws};     // A^T h: tmp[v] = sum over in-neighbours u of h[u]
    const Product pout{&rev, &wsr};  // A tmp: h[u] = sum over out-neighbours v of tmp[v]
    const unsigned gin = ws.cfg[MODE_EIG64].grid, gout = wsr.cfg[MODE_EIG64].grid;
    double *h[2] = {alloc<double>(n, s), alloc<double>(n, s)};
    double *tmp = alloc<double>(n, s);
    double4 *rin = alloc<double4>(std::max(gin, kNB), s), *rout = alloc<double4>(std::max(gout, kNB), s);
    double4 *part = alloc<double4>(kNB, s), *pvrec = alloc<double4>(kNB, s);
    State *d_st = alloc<State>(1, s), *h_st = nullptr;
    PRG_CUDA(cudaMallocHost((void **)&h_st, 2 * sizeof(State)));
    try {
        State init;
        std::memset(&init, 0, sizeof(init));
        init.max_iter = 5000;
        init.eps = 1e-12;
        PRG_CUDA(cudaMemcpyAsync(d_st, &init, sizeof(State), cudaMemcpyHostToDevice, s));
        // h = out-degree (out-strength when weighted) / its max: the graph's
        // deg / dval hold out-degree / out-strength
        degree_seed_kernel<<<kNB, kNT, 0, s>>>(g.deg, g.weighted ? g.dval : nullptr, n, negative, h[0], rout);
        normalise_kernel<<<kNB, kNT, 0, s>>>(n, rout, kNB, nullptr, 0, h[0], nullptr, part, nullptr);
        PRG_CUDA(cudaGetLastError());
        run_until_done(d_st, h_st, init.max_iter, s, [&](uint32_t it) {
            const int q = (int)(it & 1u);
            product(pin, h[q], tmp, 0.0, rin, &d_st->done, s);
            product(pout, tmp, h[q ^ 1], 0.0, rout, &d_st->done, s);
            if (negative) {  // hits.rs:399-411: the signed pivot, also the eigenvalue estimate
                pivot_kernel<<<kNB, kNT, 0, s>>>(h[q ^ 1], n, g.perm, pvrec, d_st);
                normalise_signed_kernel<<<kNB, kNT, 0, s>>>(n, pvrec, kNB, h[q ^ 1], h[q], part, d_st);
            } else {
                normalise_kernel<<<kNB, kNT, 0, s>>>(n, rout, gout, wsr.hub_rec, wsr.cfg[MODE_EIG64].hub_recs, h[q ^ 1], h[q], part,
                                                     d_st);
            }
            check_kernel<<<1, 256, 0, s>>>(part, kNB, d_st, q ^ 1);
            PRG_CUDA(cudaGetLastError());
        });
        r.iterations = h_st[0].iters;
        r.eigenvalue = h_st[0].maxv;
        double *hf = h_st[0].iters ? h[h_st[0].final_buf] : h[0];
        if (!negative) clamp_kernel<<<kNB, kNT, 0, s>>>(hf, n);
        // authority = A^T h, rescaled by its max |.|, clamped (non-negative weights)
        product(pin, hf, tmp, 0.0, rin, nullptr, s);
        normalise_kernel<<<kNB, kNT, 0, s>>>(n, rin, gin, ws.hub_rec, ws.cfg[MODE_EIG64].hub_recs, tmp, nullptr, part,
                                             nullptr);
        if (!negative) clamp_kernel<<<kNB, kNT, 0, s>>>(tmp, n);
        PRG_CUDA(cudaGetLastError());
        PRG_CUDA(cudaMemcpyAsync(d_hub, hf, (uint64_t)n * 8, cudaMemcpyDeviceToDevice, s));
        PRG_CUDA(cudaMemcpyAsync(d_auth, tmp, (uint64_t)n * 8, cudaMemcpyDeviceToDevice, s));
        PRG_CUDA(cudaStreamSynchronize(s));
    } catch (...) {
        cudaStreamSynchronize(s);
        cudaFreeHost(h_st);
        throw;
    }
    cudaFreeHost(h_st);
    release(h[0], s);
    release(h[1], s);
    release(tmp, s);
    release(rin, s);
    release(rout, s);
    release(part, s);
    release(pvrec, s);
    release(d_st, s);
    PRG_CUDA(cudaStreamSynchronize(s));
    return r;
}

}  // namespace eig
}  // namespace prg
