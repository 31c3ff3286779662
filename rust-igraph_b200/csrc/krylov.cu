// krylov.cu — PageRank as a linear system, solved with BiCGStab on the GPU.
//
// The fixed point x = G(x) of
//   G(x) = d*P^T(x/s) + d*(sum_dangling x)*t + (1-d)*t
// is the solution of the non-singular system A x = (1-d)*t with
//   A x = x - d*P^T(x/s) - d*(sum_dangling x)*t            (pagerank_linsys.rs:221-238)
// and b - A x = G(x) - x: an FP64 power step that also writes r = G(x) - x
// (MODE_KRES64) computes it.  Two solvers are built on that:
//
//  * refined (FP32 Krylov, FP64 residual): repeat { r = G(x) - x in FP64;
//    stop when ||r||_1 <= eps*(1-d)/d; solve A e = r with BiCGStab in FP32
//    to a relative reduction `rel`; x += e in FP64 }.  Each inner step costs
//    two FP32 matvecs; a handful of FP64 residual passes certify the result.
//  * FP64 Krylov: the same loop with an FP64 inner solve (one outer cycle
//    normally suffices), and the pagerank_linsys() drop-in, which stops on
//    the reference's 2-norm rule ||b - A x||_2 < 1e-13 ||b||_2
//    (pagerank_linsys.rs:54-58, 122-127) and returns x itself.
//
// One BiCGStab step is five kernels: V1 (p = r + beta (p - omega v), p/s),
// M1 (v = A p, fused into the iteration kernel, MODE_KRY*), V2 (s = r - alpha v),
// M2 (t = A s), V3 (e += alpha p + omega s, r = s - omega t).  Every reduction
// is a per-block record; the consuming kernel's blocks each add the records
// in index order, so all blocks derive the same scalars (rho, alpha, omega)
// with no grid-wide barrier, and block 0 stores them (double-buffered by
// step parity) for later kernels.  The kernels return at once when
// KState::done is set, so the host enqueues steps ahead and polls a pinned
// copy of the state one batch behind.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <type_traits>
#include <vector>

#include "solver.cuh"

namespace prg {

struct KState {
    double rho[2], alpha[2], omega[2], rhh[2];  // by step parity
    double rel;        // inner stop: ||r|| <= max(rel * ||r0||, floor_abs)
    double floor_abs;
    double near;       // rel * ||r0|| below near: aim for floor_abs in this solve
    double best;       // smallest ||r|| so far (stagnation guard)
    double tol;        // set by the first V1 from ||r0||
    double rnorm;      // last residual norm V1 saw
    double r0norm;
    uint32_t count;    // completed steps
    uint32_t cap;      // step limit
    int32_t done;      // KDONE_*
    int32_t norm2;     // 0: L1 norms, 1: 2-norms
    uint32_t restarts;
    uint32_t stall;    // consecutive steps without a 2x gain over the best ||r||
    uint32_t half;     // 1: the solve ended at a half step (the last step ran one matvec)
};

enum : int32_t {
    KRUN = 0,
    KDONE_CONVERGED = 1,
    KDONE_BREAKDOWN = 2,
    KDONE_CAP = 3,
    KDONE_NONFINITE = 4,
    KDONE_STALLED = 5  // the residual stopped falling (precision limit of the inner type): keep e
};
constexpr uint32_t kStallSteps = 3;

constexpr unsigned kVB = 148u * 4u;  // blocks of the vector kernels
constexpr uint32_t kEvStep = 6;       // events per BiCGStab step (around each of its five kernels)
constexpr int kVT = 256;

template <class T>
struct KBuf {
    T *rh = nullptr, *p = nullptr, *pt = nullptr, *v = nullptr, *s = nullptr, *st = nullptr, *t = nullptr,
      *e = nullptr, *r = nullptr;
};

struct KrylovWs {
    uint32_t n = 0;
    KBuf<float> f;
    KBuf<double> d;
    double4 *part1 = nullptr, *part2 = nullptr, *part3 = nullptr, *part4 = nullptr, *part5 = nullptr;
    KState *st = nullptr;
    KState *h_st = nullptr;  // pinned, two slots
    cudaEvent_t ev[2] = {nullptr, nullptr};
    std::vector<cudaEvent_t> mv_ev;  // around each matvec launch: 4 per step
};

template <class T>
static void kalloc(T *&p, uint64_t count, cudaStream_t s) {
    if (!p) PRG_CUDA(cudaMallocAsync((void **)&p, std::max<uint64_t>(count, 1) * sizeof(T), s));
}
template <class T>
static void kfree(T *&p, cudaStream_t s) {
    if (p) cudaFreeAsync(p, s);
    p = nullptr;
}
template <class T>
static void kbuf_free(KBuf<T> &b, cudaStream_t s) {
    for (T **q : {&b.rh, &b.p, &b.pt, &b.v, &b.s, &b.st, &b.t, &b.e, &b.r}) kfree(*q, s);
}
template <class T>
static void kbuf_alloc(KBuf<T> &b, uint64_t n, bool own_r, cudaStream_t s) {
    for (T **q : {&b.rh, &b.p, &b.pt, &b.v, &b.s, &b.st, &b.t, &b.e}) kalloc(*q, n, s);
    if (own_r) kalloc(b.r, n, s);
}

void krylov_free(KrylovWs *&k, cudaStream_t s) {
    if (!k) return;
    kbuf_free(k->f, s);
    kbuf_free(k->d, s);
    for (double4 **q : {&k->part1, &k->part2, &k->part3, &k->part4, &k->part5}) kfree(*q, s);
    kfree(k->st, s);
    if (k->h_st) cudaFreeHost(k->h_st);
    for (cudaEvent_t &e : k->ev)
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : k->mv_ev) cudaEventDestroy(e);
    delete k;
    k = nullptr;
}

static KrylovWs &krylov_ws(Workspace &ws, const DeviceGraph &g, unsigned spmv_grid, cudaStream_t s) {
    if (ws.kry && ws.kry->n != g.n) krylov_free(ws.kry, s);
    if (!ws.kry) {
        ws.kry = new KrylovWs();
        KrylovWs &k = *ws.kry;
        k.n = g.n;
        const unsigned np = std::max(kVB, spmv_grid);
        for (double4 **q : {&k.part1, &k.part2, &k.part3, &k.part4, &k.part5}) kalloc(*q, np, s);
        kalloc(k.st, 1, s);
        PRG_CUDA(cudaMallocHost((void **)&k.h_st, 2 * sizeof(KState)));
        for (cudaEvent_t &e : k.ev) PRG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    return *ws.kry;
}

// ---------------------------------------------------------------- device side

__device__ __forceinline__ double kwarp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide sums of three doubles (fixed tree), broadcast to every thread.
__device__ __forceinline__ double3 kblock3(double a, double b, double c) {
    __shared__ double sh[3][kVT / 32];
    __shared__ double out[3];
    a = kwarp_sum(a);
    b = kwarp_sum(b);
    c = kwarp_sum(c);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) {
        sh[0][w] = a;
        sh[1][w] = b;
        sh[2][w] = c;
    }
    __syncthreads();
    if (w == 0) {
        a = l < kVT / 32 ? sh[0][l] : 0.0;
        b = l < kVT / 32 ? sh[1][l] : 0.0;
        c = l < kVT / 32 ? sh[2][l] : 0.0;
        a = kwarp_sum(a);
        b = kwarp_sum(b);
        c = kwarp_sum(c);
        if (l == 0) {
            out[0] = a;
            out[1] = b;
            out[2] = c;
        }
    }
    __syncthreads();
    return make_double3(out[0], out[1], out[2]);
}

// Sum of the records a[0..na) then b[0..nb), in index order per thread and a
// fixed tree across threads: every block obtains the same three values.
__device__ __forceinline__ double3 krecords(const double4 *a, uint32_t na, const double4 *b, uint32_t nb) {
    double x = 0.0, y = 0.0, z = 0.0;
    for (uint32_t i = threadIdx.x; i < na; i += kVT) {
        const double4 q = a[i];
        x += q.x;
        y += q.y;
        z += q.z;
    }
    for (uint32_t i = threadIdx.x; i < nb; i += kVT) {
        const double4 q = b[i];
        x += q.x;
        y += q.y;
        z += q.z;
    }
    return kblock3(x, y, z);
}

__device__ __forceinline__ bool kstopped(const KState *st) { return *(volatile const int32_t *)&st->done != KRUN; }
__device__ __forceinline__ bool kleader() { return blockIdx.x == 0 && threadIdx.x == 0; }

// W-wide loads and stores at an index that is a multiple of W (the vectors
// come from the stream-ordered pool, 256-byte aligned): 16-byte accesses for
// FP32 (W = 4), two 16-byte accesses for FP64; W = 1 for the tail.
template <int W, bool CS, class T>
__device__ __forceinline__ void ldv(const T *p, T (&o)[W]) {
    if constexpr (W == 1) {
        o[0] = CS ? __ldcs(p) : *p;
    } else if constexpr (sizeof(T) == 4) {
        const float4 q = CS ? __ldcs(reinterpret_cast<const float4 *>(p)) : *reinterpret_cast<const float4 *>(p);
        o[0] = q.x; o[1] = q.y; o[2] = q.z; o[3] = q.w;
    } else {
        const double2 a = CS ? __ldcs(reinterpret_cast<const double2 *>(p)) : *reinterpret_cast<const double2 *>(p);
        const double2 b = CS ? __ldcs(reinterpret_cast<const double2 *>(p) + 1)
                             : *(reinterpret_cast<const double2 *>(p) + 1);
        o[0] = a.x; o[1] = a.y; o[2] = b.x; o[3] = b.y;
    }
}
template <int W, bool CS, class T>
__device__ __forceinline__ void stv(T *p, const T (&x)[W]) {
    if constexpr (W == 1) {
        if (CS) __stcs(p, x[0]);
        else *p = x[0];
    } else if constexpr (sizeof(T) == 4) {
        const float4 q = make_float4(x[0], x[1], x[2], x[3]);
        if (CS) __stcs(reinterpret_cast<float4 *>(p), q);
        else *reinterpret_cast<float4 *>(p) = q;
    } else {
        const double2 a = make_double2(x[0], x[1]), b = make_double2(x[2], x[3]);
        if (CS) {
            __stcs(reinterpret_cast<double2 *>(p), a);
            __stcs(reinterpret_cast<double2 *>(p) + 1, b);
        } else {
            *reinterpret_cast<double2 *>(p) = a;
            *(reinterpret_cast<double2 *>(p) + 1) = b;
        }
    }
}

// x / s for W elements at i (the gathered copy) and their dangling flags.
template <int W>
__device__ __forceinline__ void kscale(const float (&x)[W], uint32_t i, const float *inv32, const double *,
                                       float (&o)[W], bool (&dang)[W]) {
    float iv[W];
    ldv<W, false>(inv32 + i, iv);
#pragma unroll
    for (int k = 0; k < W; k++) {
        o[k] = x[k] * iv[k];
        dang[k] = iv[k] == 0.0f;
    }
}
template <int W>
__device__ __forceinline__ void kscale(const double (&x)[W], uint32_t i, const float *, const double *dval,
                                       double (&o)[W], bool (&dang)[W]) {
    double dv[W];
    ldv<W, false>(dval + i, dv);
#pragma unroll
    for (int k = 0; k < W; k++) {
        dang[k] = dv[k] == 0.0;
        o[k] = dang[k] ? 0.0 : x[k] / dv[k];
    }
}

// Runs body<4>(i) over i = 0, 4, ... below n & ~3 (grid-stride), then
// body<1>(i) over the tail.
template <class F4, class F1>
__device__ __forceinline__ void kfor(uint32_t n, F4 body4, F1 body1) {
    const uint32_t tid = blockIdx.x * kVT + threadIdx.x, nt = gridDim.x * kVT;
    const uint32_t n4 = n >> 2;
    for (uint32_t j = tid; j < n4; j += nt) body4(j << 2);
    for (uint32_t i = (n4 << 2) + tid; i < n; i += nt) body1(i);
}

// V0: rh = r, e = 0; records (rh.r, |r|_1, r.r).
template <class T>
__global__ void __launch_bounds__(kVT) kv0(uint32_t n, const T *r, T *rh, T *e, double4 *part5) {
    double a = 0.0, b = 0.0;
    auto body = [&](uint32_t i, auto w) {
        constexpr int W = decltype(w)::value;
        T rv[W], z[W];
        ldv<W, true>(r + i, rv);
#pragma unroll
        for (int k = 0; k < W; k++) {
            z[k] = T(0);
            a += (double)rv[k] * (double)rv[k];
            b += fabs((double)rv[k]);
        }
        stv<W, false>(rh + i, rv);
        stv<W, true>(e + i, z);
    };
    kfor(n, [&](uint32_t i) { body(i, std::integral_constant<int, 4>()); },
         [&](uint32_t i) { body(i, std::integral_constant<int, 1>()); });
    const double3 q = kblock3(a, b, 0.0);
    if (threadIdx.x == 0) part5[blockIdx.x] = make_double4(q.x, q.y, q.x, 0.0);
}

// V1: stop test on ||r||, then p = r + beta (p - omega v) (p = r on the first
// step or a restart), p/s, and the dangling mass of p.
template <class T>
__global__ void __launch_bounds__(kVT) kv1(uint32_t n, int q, KState *st, const double4 *part5, T *rh, const T *r,
                                           T *p, T *pt, const T *v, const float *inv32, const double *dval,
                                           double4 *part1) {
    if (kstopped(st)) return;
    const double3 red = krecords(part5, gridDim.x, nullptr, 0);
    const double rhr = red.x, rn1 = red.y, rr = red.z;
    const uint32_t k = st->count;
    const double norm = st->norm2 ? sqrt(rr) : rn1;
    if (!isfinite(norm) || !isfinite(rhr)) {
        if (kleader()) st->done = KDONE_NONFINITE;
        return;
    }
    // close to the final target already: finish it in this inner solve
    // rather than pay for another outer cycle (residual pass + restart)
    const double rt = st->rel * norm;
    const double tol = k == 0 ? (rt < st->near ? st->floor_abs : fmax(rt, st->floor_abs)) : st->tol;
    if (k == 0 && kleader()) {
        st->tol = tol;
        st->r0norm = norm;
    }
    if (!(norm > tol)) {
        if (kleader()) {
            st->rnorm = norm;
            st->done = KDONE_CONVERGED;
        }
        return;
    }
    if (k >= st->cap) {
        if (kleader()) {
            st->rnorm = norm;
            st->done = KDONE_CAP;
        }
        return;
    }
    // stagnation: kStallSteps steps in a row without halving the best norm
    const double best = k == 0 ? norm : st->best;
    const uint32_t stall = k == 0 ? 0u : (norm < 0.5 * best ? 0u : st->stall + 1u);
    if (stall >= kStallSteps) {
        if (kleader()) {
            st->rnorm = norm;
            st->done = KDONE_STALLED;
        }
        return;
    }
    const int o = q ^ 1;
    const double om = k ? st->omega[o] : 0.0, rho0 = k ? st->rho[o] : 0.0, al = k ? st->alpha[o] : 0.0;
    const double rhh = k ? st->rhh[o] : rr;
    // restart (rh = r) when the shadow residual has become nearly orthogonal
    // to r, or the previous step ended with omega = 0
    const bool restart = k == 0 || om == 0.0 || rho0 == 0.0 || !(fabs(rhr) > 1e-9 * sqrt(rhh * rr));
    const bool write_rh = restart && k != 0;
    const double beta = restart ? 0.0 : (rhr / rho0) * (al / om);
    const T tb = (T)beta, to = (T)om;
    double dz = 0.0;
    auto body = [&](uint32_t i, auto w) {
        constexpr int W = decltype(w)::value;
        T rv[W], pv[W], sc[W];
        bool dang[W];
        ldv<W, true>(r + i, rv);
        if (restart) {
#pragma unroll
            for (int j = 0; j < W; j++) pv[j] = rv[j];
        } else {
            T po[W], vv[W];
            ldv<W, true>(p + i, po);
            ldv<W, true>(v + i, vv);
#pragma unroll
            for (int j = 0; j < W; j++) pv[j] = rv[j] + tb * (po[j] - to * vv[j]);
        }
        stv<W, true>(p + i, pv);  // streamed: only p/s is gathered, keep that in L2
        kscale<W>(pv, i, inv32, dval, sc, dang);
        stv<W, false>(pt + i, sc);
#pragma unroll
        for (int j = 0; j < W; j++)
            if (dang[j]) dz += (double)pv[j];
        if (write_rh) stv<W, false>(rh + i, rv);
    };
    kfor(n, [&](uint32_t i) { body(i, std::integral_constant<int, 4>()); },
         [&](uint32_t i) { body(i, std::integral_constant<int, 1>()); });
    const double3 s3 = kblock3(dz, 0.0, 0.0);
    if (threadIdx.x == 0) part1[blockIdx.x] = make_double4(s3.x, 0.0, 0.0, 0.0);
    if (kleader()) {
        st->rho[q] = restart ? rr : rhr;
        st->rhh[q] = restart ? rr : rhh;
        st->rnorm = norm;
        st->best = fmin(best, norm);
        st->stall = stall;
        if (write_rh) st->restarts += 1u;
    }
}

// V2: alpha = rho / (rh.v); s = r - alpha v, s/s_deg; records (dangling mass
// of s, |s|_1, s.s), the norms for the half-step test in M2.
template <class T>
__global__ void __launch_bounds__(kVT) kv2(uint32_t n, int q, KState *st, const double4 *part2, uint32_t n2,
                                           const double4 *hub_rec, uint32_t nhub, const T *r, const T *v, T *s,
                                           T *sst, const float *inv32, const double *dval, double4 *part3) {
    if (kstopped(st)) return;
    const double3 red = krecords(part2, n2, hub_rec, nhub);
    const double sig = red.x, rho = st->rho[q];
    if (!(fabs(sig) > 0.0) || !isfinite(sig)) {
        if (kleader()) st->done = isfinite(sig) ? KDONE_BREAKDOWN : KDONE_NONFINITE;
        return;
    }
    const double al = rho / sig;
    const T ta = (T)al;
    double dz = 0.0, s1 = 0.0, s2 = 0.0;
    auto body = [&](uint32_t i, auto w) {
        constexpr int W = decltype(w)::value;
        T rv[W], vv[W], sv[W], sc[W];
        bool dang[W];
        ldv<W, true>(r + i, rv);
        ldv<W, true>(v + i, vv);
#pragma unroll
        for (int j = 0; j < W; j++) {
            sv[j] = rv[j] - ta * vv[j];
            s1 += fabs((double)sv[j]);
            s2 += (double)sv[j] * (double)sv[j];
        }
        stv<W, true>(s + i, sv);
        kscale<W>(sv, i, inv32, dval, sc, dang);
        stv<W, false>(sst + i, sc);
#pragma unroll
        for (int j = 0; j < W; j++)
            if (dang[j]) dz += (double)sv[j];
    };
    kfor(n, [&](uint32_t i) { body(i, std::integral_constant<int, 4>()); },
         [&](uint32_t i) { body(i, std::integral_constant<int, 1>()); });
    const double3 s3 = kblock3(dz, s1, s2);
    if (threadIdx.x == 0) part3[blockIdx.x] = make_double4(s3.x, s3.y, s3.z, 0.0);
    if (kleader()) st->alpha[q] = al;
}

// V3: omega = (t.s)/(t.t); e += alpha p + omega s; r = s - omega t;
// records (rh.r, |r|_1, r.r) for the next V1.  When M2 skipped (its marker
// part4[0].w = 1: ||s|| met the target), the step ends at its half:
// e += alpha p and the solve is converged.
template <class T>
__global__ void __launch_bounds__(kVT) kv3(uint32_t n, int q, KState *st, const double4 *part4, uint32_t n4,
                                           const double4 *hub_rec, uint32_t nhub, const double4 *part3,
                                           const T *rh, const T *p, const T *s, const T *t, T *e, T *r,
                                           double4 *part5) {
    if (kstopped(st)) return;
    if (part4[0].w == 1.0) {
        const T ta = (T)st->alpha[q];
        auto half = [&](uint32_t i, auto w) {
            constexpr int W = decltype(w)::value;
            T ev[W], pv[W];
            ldv<W, true>(e + i, ev);
            ldv<W, true>(p + i, pv);
#pragma unroll
            for (int j = 0; j < W; j++) ev[j] = ev[j] + ta * pv[j];
            stv<W, true>(e + i, ev);
        };
        kfor(n, [&](uint32_t i) { half(i, std::integral_constant<int, 4>()); },
             [&](uint32_t i) { half(i, std::integral_constant<int, 1>()); });
        if (blockIdx.x == 0) {  // the block-wide reduction runs in all of block 0's threads
            const double3 sr = krecords(part3, gridDim.x, nullptr, 0);
            if (threadIdx.x == 0) {
                st->rnorm = st->norm2 ? sqrt(sr.z) : sr.y;
                st->count += 1u;
                st->half = 1u;
                st->done = KDONE_CONVERGED;
            }
        }
        return;
    }
    const double3 red = krecords(part4, n4, hub_rec, nhub);
    const double ts = red.y, tt = red.z;
    const double om = tt > 0.0 && isfinite(tt) ? ts / tt : 0.0;
    const T ta = (T)st->alpha[q], to = (T)om;
    double a = 0.0, b = 0.0, c = 0.0;
    auto body = [&](uint32_t i, auto w) {
        constexpr int W = decltype(w)::value;
        T sv[W], ev[W], pv[W], tv[W], hv[W], rv[W];
        ldv<W, true>(s + i, sv);
        ldv<W, true>(e + i, ev);
        ldv<W, true>(p + i, pv);
        ldv<W, true>(t + i, tv);
        ldv<W, true>(rh + i, hv);
#pragma unroll
        for (int j = 0; j < W; j++) {
            ev[j] = ev[j] + ta * pv[j] + to * sv[j];
            rv[j] = sv[j] - to * tv[j];
            a += (double)hv[j] * (double)rv[j];
            b += fabs((double)rv[j]);
            c += (double)rv[j] * (double)rv[j];
        }
        stv<W, true>(e + i, ev);
        stv<W, true>(r + i, rv);
    };
    kfor(n, [&](uint32_t i) { body(i, std::integral_constant<int, 4>()); },
         [&](uint32_t i) { body(i, std::integral_constant<int, 1>()); });
    const double3 s3 = kblock3(a, b, c);
    if (threadIdx.x == 0) part5[blockIdx.x] = make_double4(s3.x, s3.y, s3.z, 0.0);
    if (kleader()) {
        st->omega[q] = om;
        st->count += 1u;
    }
}

// x += e (FP64), xt = x / s, dangling and total mass into Ctl (the same
// bookkeeping as launch_prepare64, for an FP64 correction).
__global__ void __launch_bounds__(kVT) kadd64(uint32_t n, double *x, const double *e) {
    for (uint32_t v = blockIdx.x * kVT + threadIdx.x; v < n; v += gridDim.x * kVT) x[v] += e[v];
}

// ---------------------------------------------------------------- host side

struct InnerResult {
    uint32_t steps = 0;
    uint32_t half = 0;       // 1: the last step stopped after its first matvec
    int32_t done = KRUN;
    double rnorm = 0.0;
    double ms = 0.0;
    double matvec_ms = 0.0;  // the matvec launches of completed steps
    uint32_t launches = 0;
};

template <class T>
static IterArgs matvec_args(const IterArgs &base, const T *in, const T *in_scaled, T *out, const T *rh,
                            const double4 *pin, uint32_t npin, double4 *pout, const KState *st) {
    IterArgs a = base;
    if constexpr (sizeof(T) == 4) {
        a.x32_in = in;
        a.xt32_in = in_scaled;
        a.x32_out = out;
        a.rh32 = rh;
    } else {
        a.x64_in = in;
        a.xt64_in = in_scaled;
        a.x64_out = out;
        a.rh64 = rh;
    }
    a.kpart_in = pin;
    a.kpart_n = npin;
    a.kpart_out = pout;
    a.kdone = &st->done;
    return a;
}

// BiCGStab on A e = r (e0 = 0) in precision T; r is overwritten.
template <class T>
static InnerResult bicgstab(const DeviceGraph &g, Workspace &ws, KrylovWs &k, KBuf<T> &b, const T *r_in,
                            const double *t64, const float *t32, double damping, double rel, double floor_abs,
                            double near, uint32_t cap, bool norm2, cudaStream_t s) {
    InnerResult res;
    constexpr int mode = sizeof(T) == 4 ? MODE_KRY32 : MODE_KRY64;
    const LaunchCfg &cfg = ws.cfg[mode];
    const uint32_t n = g.n;
    T *r = const_cast<T *>(r_in);

    KState init;
    std::memset(&init, 0, sizeof(init));
    init.rel = rel;
    init.floor_abs = floor_abs;
    init.near = near;
    init.cap = cap;
    init.norm2 = norm2 ? 1 : 0;
    PRG_CUDA(cudaMemcpyAsync(k.st, &init, sizeof(KState), cudaMemcpyHostToDevice, s));

    IterArgs base = base_args(g, ws, damping);
    if constexpr (sizeof(T) == 4) base.t32 = t32;
    else base.t64 = t64;
    const IterArgs m1 = matvec_args<T>(base, b.p, b.pt, b.v, b.rh, k.part1, kVB, k.part2, k.st);
    IterArgs m2 = matvec_args<T>(base, b.s, b.st, b.t, (const T *)nullptr, k.part3, kVB, k.part4, k.st);
    m2.ktol = &k.st->tol;  // skip t = A s when ||s|| already meets the target (half step)
    m2.knorm2 = norm2 ? 1 : 0;

    // the matvec launches are bracketed by events (4 per step) so their
    // device time can be reported apart from the vector kernels
    const uint32_t max_steps = (cap / 2u + 3u) * 2u + 2u;
    PRG_CUDA(cudaEventRecord(ws.eva, s));
    kv0<T><<<kVB, kVT, 0, s>>>(n, r, b.rh, b.e, k.part5);
    res.launches += 1u;
    uint32_t it = 0;
    auto step = [&](int q) {
        while (k.mv_ev.size() < kEvStep * (it + 1u)) {
            cudaEvent_t e;
            PRG_CUDA(cudaEventCreate(&e));
            k.mv_ev.push_back(e);
        }
        cudaEvent_t *ev = &k.mv_ev[kEvStep * it];
        PRG_CUDA(cudaEventRecord(ev[0], s));
        kv1<T><<<kVB, kVT, 0, s>>>(n, q, k.st, k.part5, b.rh, r, b.p, b.pt, b.v, g.inv32, g.dval, k.part1);
        PRG_CUDA(cudaEventRecord(ev[1], s));
        launch_iteration(mode, g.weighted, m1, cfg, s);
        PRG_CUDA(cudaEventRecord(ev[2], s));
        kv2<T><<<kVB, kVT, 0, s>>>(n, q, k.st, k.part2, cfg.grid, ws.hub_rec, cfg.hub_recs, r, b.v, b.s, b.st, g.inv32,
                                    g.dval, k.part3);
        PRG_CUDA(cudaEventRecord(ev[3], s));
        launch_iteration(mode, g.weighted, m2, cfg, s);
        PRG_CUDA(cudaEventRecord(ev[4], s));
        kv3<T><<<kVB, kVT, 0, s>>>(n, q, k.st, k.part4, cfg.grid, ws.hub_rec, cfg.hub_recs, k.part3, b.rh, b.p, b.s, b.t,
                                    b.e, r, k.part5);
        PRG_CUDA(cudaEventRecord(ev[5], s));
        res.launches += cfg.seg ? 7u : 5u;  // the segmented matvec is two kernels
    };
    // batches of `per` steps; the state copy of batch j is read while batch
    // j+1 runs (kernels of a finished solve return at once)
    const int per = 2;
    const uint32_t max_batches = cap / per + 3u;
    uint32_t batch = 0;
    bool stop = false;
    while (!stop) {
        for (int i = 0; i < per && it < max_steps; i++) {
            step((int)(it & 1u));
            it++;
        }
        const int slot = (int)(batch & 1u);
        PRG_CUDA(cudaMemcpyAsync(&k.h_st[slot], k.st, sizeof(KState), cudaMemcpyDeviceToHost, s));
        PRG_CUDA(cudaEventRecord(k.ev[slot], s));
        if (batch > 0) {
            const int prev = slot ^ 1;
            PRG_CUDA(cudaEventSynchronize(k.ev[prev]));
            if (k.h_st[prev].done != KRUN) stop = true;
        }
        if (++batch >= max_batches) stop = true;
        PRG_CUDA(cudaGetLastError());
    }
    PRG_CUDA(cudaEventRecord(ws.evb, s));
    PRG_CUDA(cudaMemcpyAsync(&k.h_st[0], k.st, sizeof(KState), cudaMemcpyDeviceToHost, s));
    PRG_CUDA(cudaStreamSynchronize(s));
    float ms = 0.f;
    PRG_CUDA(cudaEventElapsedTime(&ms, ws.eva, ws.evb));
    res.ms = ms;
    res.steps = k.h_st[0].count;
    double vec_ms = 0.0, gap_ms = 0.0;
    for (uint32_t i = 0; i < res.steps && i < it; i++) {
        const cudaEvent_t *ev = &k.mv_ev[kEvStep * i];
        float t[5];
        for (int j = 0; j < 5; j++) PRG_CUDA(cudaEventElapsedTime(&t[j], ev[j], ev[j + 1]));
        res.matvec_ms += (double)t[1] + (double)t[3];
        vec_ms += (double)t[0] + (double)t[2] + (double)t[4];
        if (i + 1 < res.steps && i + 1 < it) {
            float gp = 0.f;
            PRG_CUDA(cudaEventElapsedTime(&gp, ev[5], k.mv_ev[kEvStep * (i + 1)]));
            gap_ms += gp;
        }
    }
    res.done = k.h_st[0].done;
    res.rnorm = k.h_st[0].rnorm;
    res.half = k.h_st[0].half;
    if (std::getenv("PRG_TRACE"))
        std::fprintf(stderr,
                     "[prg] bicgstab<%s>: %u steps (half %u), done=%d, ||r||=%.3e (r0 %.3e), restarts %u, %.3f ms "
                     "(matvecs %.3f, vector kernels %.3f, between steps %.3f)\n",
                     sizeof(T) == 4 ? "f32" : "f64", res.steps, res.half, res.done, res.rnorm, k.h_st[0].r0norm,
                     k.h_st[0].restarts, res.ms, res.matvec_ms, vec_ms, gap_ms);
    return res;
}

// Refined / FP64 Krylov solve (see the file comment).  `fp64_inner` picks the
// inner precision; `linsys` selects the pagerank_linsys() stop rule and
// returns x instead of the normalised G(x).
void solve_krylov(const DeviceGraph &g, Workspace &ws, const SolveOpts &o, const double *d_t, double *d_out,
                  SolveStats &st, cudaStream_t s, bool fp64_inner, bool linsys) {
    const bool ppr = d_t != nullptr;
    const uint32_t n = g.n;
    const int mode = fp64_inner ? MODE_KRY64 : MODE_KRY32;
    KrylovWs &k = krylov_ws(ws, g, ws.cfg[mode].grid, s);
    if (fp64_inner) kbuf_alloc(k.d, n, true, s);
    else kbuf_alloc(k.f, n, false, s);

    const double thr_final = o.eps * (1.0 - o.damping) / o.damping;
    // pagerank_linsys: ||b - A x||_2 < 1e-13 ||b||_2 with b = (1-d)/n * 1
    const double lin_tol = 1e-13 * ((1.0 - o.damping) / (double)n) * std::sqrt((double)n);
    const double rel = linsys ? 0.0 : (fp64_inner ? 1e-14 : tuning().krylov_rel);
    // inner solves aim below the certified threshold by this factor: the
    // FP64 residual pass that follows must land under thr_final, and the
    // FP32 recursive residual drifts a few percent from the true one
    const double floor_abs = linsys ? lin_tol : tuning().krylov_floor * thr_final;

    // x0 (FP64) and its scaled copy / dangling mass for the residual pass
    if (o.d_start) PRG_CUDA(cudaMemcpyAsync(ws.x64[0], o.d_start, (uint64_t)n * 8, cudaMemcpyDeviceToDevice, s));
    else launch_fill_start(ws.x64[0], d_t, n, s);
    Ctl c;
    std::memset(&c, 0, sizeof(c));
    c.rho = 1.0;
    c.floor_abs = 0.0;
    PRG_CUDA(cudaMemcpyAsync(ws.ctl, &c, sizeof(Ctl), cudaMemcpyHostToDevice, s));
    launch_prepare64(g, ws.x64[0], nullptr, ws.xt64[0], ws.ctl, 1, ws.blk_part, s);
    st.kernel_launches += (o.d_start ? 0u : 1u) + 2u;
    if (ppr && !fp64_inner) {
        to_f32(d_t, ws.t32, n, s);
        st.kernel_launches += 1u;
    }

    IterArgs rp = base_args(g, ws, o.damping);
    rp.t64 = d_t;
    rp.parity = 1;
    rp.x64_in = ws.x64[0];
    rp.xt64_in = ws.xt64[0];
    rp.x64_out = ws.x64[1];
    if (fp64_inner) rp.b64_out = k.d.r;
    else rp.b32_out = ws.b32;

    const uint32_t pass_cap = std::max<uint32_t>(o.max_iter, 64u);
    uint32_t mv = 0, fp64 = 0, stalls = 0;
    double prev_rn = INFINITY;
    bool fallback = false;
    for (int outer = 0; outer < 64; outer++) {
        PRG_CUDA(cudaEventRecord(ws.eva, s));
        launch_iteration(MODE_KRES64, g.weighted, rp, ws.cfg[MODE_KRES64], s);
        PRG_CUDA(cudaEventRecord(ws.evb, s));
        fp64++;
        st.kernel_launches += 1u;
        read_ctl(ws, s);
        {
            float t = 0.f;
            PRG_CUDA(cudaEventElapsedTime(&t, ws.eva, ws.evb));
            st.fp64_ms += t;
        }
        const double rn = ws.h_ctl->rnorm;
        st.residual_l1 = rn;
        if (std::getenv("PRG_TRACE"))
            std::fprintf(stderr, "[prg] krylov residual pass %u: ||r||_1 = %.3e (after %u matvecs)\n", fp64, rn, mv);
        if (!std::isfinite(rn)) throw CudaError{cudaErrorUnknown, "non-finite residual in the Krylov solve"};
        if (!linsys && !(rn > thr_final)) break;
        if (mv + fp64 >= pass_cap) break;
        // progress guard: two outer cycles without halving ||r||_1 hand the
        // rest of the solve to the FP64 power iteration
        stalls = rn > 0.5 * prev_rn ? stalls + 1u : 0u;
        prev_rn = rn;
        if (stalls >= 2) {
            fallback = true;
            break;
        }
        const uint32_t cap = std::min<uint32_t>(500u, (pass_cap - mv - fp64) / 2u + 1u);
        InnerResult ir;
        // a relative target within 100x of the final one is replaced by the floor
        const double near = linsys ? 0.0 : 100.0 * thr_final;
        if (fp64_inner)
            ir = bicgstab<double>(g, ws, k, k.d, k.d.r, d_t, nullptr, o.damping, rel, floor_abs, near, cap, linsys,
                                  s);
        else
            ir = bicgstab<float>(g, ws, k, k.f, ws.b32, nullptr, ppr ? ws.t32 : nullptr, o.damping, rel, floor_abs,
                                 near, cap, false, s);
        mv += 2u * ir.steps - ir.half;
        st.spmv_ms += ir.matvec_ms;
        st.spmv_launches += 2u * ir.steps - ir.half;
        st.kernel_launches += ir.launches;
        st.fp32_ms += fp64_inner ? 0.0 : ir.ms;
        st.fp64_ms += fp64_inner ? ir.ms : 0.0;
        if (linsys && ir.steps == 0 && ir.done == KDONE_CONVERGED) break;  // the true residual met the rule
        if (ir.done == KDONE_NONFINITE) {
            fallback = true;
            break;
        }
        if (ir.steps == 0) {
            stalls = 2;
            fallback = true;
            break;
        }
        if (fp64_inner) {
            kadd64<<<kVB, kVT, 0, s>>>(n, ws.x64[0], k.d.e);
            launch_prepare64(g, ws.x64[0], nullptr, ws.xt64[0], ws.ctl, 1, ws.blk_part, s);
            st.kernel_launches += 3u;
        } else {
            launch_prepare64(g, ws.x64[0], k.f.e, ws.xt64[0], ws.ctl, 1, ws.blk_part, s);
            st.kernel_launches += 2u;
        }
    }
    st.fp32_passes = fp64_inner ? 0u : mv;
    st.fp64_passes = fp64 + (fp64_inner ? mv : 0u);
    st.residual_passes = fp64;
    st.iterations = mv + fp64;
    if (fallback) {
        // x64[0] holds the best iterate: finish with the FP64 power iteration
        SolveOpts f = o;
        f.d_start = ws.x64[0];
        f.stop = 1;
        SolveStats fs;
        const double *res = fp64_loop(g, ws, f, d_t, thr_final, o.max_iter, fs, s);
        PRG_CUDA(cudaMemcpyAsync(d_out, res, (uint64_t)n * 8, cudaMemcpyDeviceToDevice, s));
        st.fp64_passes += fs.fp64_passes;
        st.iterations += fs.iterations;
        st.kernel_launches += fs.kernel_launches;
        st.fp64_ms += fs.fp64_ms;
        st.last_diff = fs.last_diff;
        st.residual_l1 = fs.last_diff;
        st.error_bound = fs.last_diff * o.damping / (1.0 - o.damping);
        return;
    }
    if (linsys) {
        // pagerank_linsys returns the iterate itself
        PRG_CUDA(cudaMemcpyAsync(d_out, ws.x64[0], (uint64_t)n * 8, cudaMemcpyDeviceToDevice, s));
    } else {
        PRG_CUDA(cudaMemcpyAsync(d_out, ws.x64[1], (uint64_t)n * 8, cudaMemcpyDeviceToDevice, s));
        if (o.normalise) {
            launch_normalise(d_out, n, ws.ctl, s);
            st.kernel_launches += 1u;
        }
    }
    st.last_diff = ws.h_ctl->diff;
    st.error_bound = st.residual_l1 * o.damping / (1.0 - o.damping);
}

// One FP32 Krylov matvec y = p - d (A pt + dz t), t = 1/n, through the
// row-block kernel (kernel 0) or a tile-segmented one (1, 2), with rh = p:
// dots = the launch's summed records (p.y, y.p, y.y) in record order, ms =
// its device time.  A diagnostic: its inputs live in internal ids.
void matvec32_probe(const DeviceGraph &g, Workspace &ws, int kernel, const float *p, const float *pt, double dz,
                    double damping, float *y, double dots[3], float *ms, cudaStream_t s) {
    workspace_ensure(ws, g, s);
    LaunchCfg c;
    if (kernel == 0) {
        c = iteration_config(MODE_KRY32, g.weighted, g.perm != nullptr ? g.hot_cache : 0u, g.blocks_per_sm, g.n,
                             g.hot_threads);
        c.hub_recs = g.nhub;
    } else {
        if (ws.seg.mask == nullptr) seg_build(g, ws.seg, s);
        c = seg_config(g, g.perm != nullptr ? g.seg_hot : 0u, kernel, MODE_KRY32);
    }
    if (g.perm != nullptr && g.l1_hot32) c.l1hot = g.l1_hot32;
    IterArgs a = base_args(g, ws, damping);
    a.x32_in = p;
    a.xt32_in = pt;
    a.x32_out = y;
    a.rh32 = p;
    // [kdone][record in][records out]
    const uint32_t nrec = c.grid;
    double4 *buf = nullptr;
    PRG_CUDA(cudaMallocAsync((void **)&buf, (2 + (uint64_t)nrec) * sizeof(double4), s));
    PRG_CUDA(cudaMemsetAsync(buf, 0, (2 + (uint64_t)nrec) * sizeof(double4), s));
    const double4 rin = make_double4(dz, 0.0, 0.0, 0.0);
    PRG_CUDA(cudaMemcpyAsync(buf + 1, &rin, sizeof(double4), cudaMemcpyHostToDevice, s));
    a.kdone = reinterpret_cast<const int32_t *>(buf);
    a.kpart_in = buf + 1;
    a.kpart_n = 1;
    a.kpart_out = buf + 2;
    a.ktol = nullptr;
    PRG_CUDA(cudaEventRecord(ws.eva, s));
    launch_iteration(MODE_KRY32, g.weighted, a, c, s);
    PRG_CUDA(cudaEventRecord(ws.evb, s));
    std::vector<double4> rec(nrec), hub(c.hub_recs);
    PRG_CUDA(cudaMemcpyAsync(rec.data(), buf + 2, (uint64_t)nrec * sizeof(double4), cudaMemcpyDeviceToHost, s));
    if (c.hub_recs)
        PRG_CUDA(cudaMemcpyAsync(hub.data(), ws.hub_rec, (uint64_t)c.hub_recs * sizeof(double4),
                                 cudaMemcpyDeviceToHost, s));
    PRG_CUDA(cudaStreamSynchronize(s));
    PRG_CUDA(cudaEventElapsedTime(ms, ws.eva, ws.evb));
    cudaFreeAsync(buf, s);
    dots[0] = dots[1] = dots[2] = 0.0;
    for (const double4 &q : rec) {
        dots[0] += q.x;
        dots[1] += q.y;
        dots[2] += q.z;
    }
    for (const double4 &q : hub) {
        dots[0] += q.x;
        dots[1] += q.y;
        dots[2] += q.z;
    }
}

}  // namespace prg
