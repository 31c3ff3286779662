/*
 * prg_oracle.c — CPU oracle for the PageRank hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product library links or calls
 * this file; only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg load it, and only as the checker (or as the timed CPU baseline).
 *
 * Contents
 *   1. SplitMix64 and the seeded generators used to build identical inputs:
 *        rust-igraph src/core/rng.rs:30-110        (SplitMix64)
 *        src/algorithms/games/erdos_renyi.rs:59-170,328-353  (G(n,m))
 *        src/algorithms/games/barabasi.rs:114-179   (BA, bag variant)
 *        src/algorithms/games/sbm.rs:84-146,224-372 (SBM)
 *      plus a project-defined counter-based R-MAT generator (the reference
 *      has none) that the CUDA generator reproduces bit-for-bit.
 *   2. Line-for-line restatements of the three reference functions:
 *        src/algorithms/properties/pagerank.rs:52-143
 *        src/algorithms/properties/pagerank_weighted.rs:52-161
 *        src/algorithms/properties/personalized_pagerank.rs:65-182
 *      They keep the reference's in-adjacency order (edge-id order), its
 *      per-edge divide, its summation order and its stop rule, so with
 *      -ffp-contract=off they reproduce the reference bit-for-bit.
 *   3. A tight FP64 oracle: the same fixed point iterated with
 *      Neumaier-compensated sums until the successive L1 change is below a
 *      caller tolerance (1e-14 by default), multithreaded over rows.
 *
 * Edges are passed as the reference Graph stores them: edge e is
 * (from[e], to[e]); for undirected graphs Graph::add_edges stores
 * (min, max) (src/core/graph.rs:756-785).  The restatements do not depend
 * on that canonical order (both directions are pushed), but generators emit
 * it so edge lists match the reference's exactly.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

/* Minimal fork-join helper: runs fn(ctx, t, nthreads) on nthreads threads. */
typedef void (*par_fn)(void *ctx, int t, int nt);
typedef struct { par_fn fn; void *ctx; int t, nt; } par_arg;
static void *par_tramp(void *p) {
    par_arg *a = (par_arg *)p;
    a->fn(a->ctx, a->t, a->nt);
    return NULL;
}
static void par_run(int nt, par_fn fn, void *ctx) {
    if (nt < 1) nt = 1;
    if (nt > 256) nt = 256;
    pthread_t th[256];
    int ok[256];
    par_arg args[256];
    for (int t = 0; t < nt; t++) {
        args[t].fn = fn; args[t].ctx = ctx; args[t].t = t; args[t].nt = nt;
        ok[t] = 0;
        if (t > 0) ok[t] = pthread_create(&th[t], NULL, par_tramp, &args[t]) == 0;
    }
    fn(ctx, 0, nt);
    for (int t = 1; t < nt; t++) {
        if (ok[t]) pthread_join(th[t], NULL);
        else fn(ctx, t, nt);
    }
}

/* ------------------------------------------------------------------ */
/* 1. SplitMix64 (rng.rs:30-110)                                       */
/* ------------------------------------------------------------------ */

typedef struct { uint64_t s; } sm64;

/* rng.rs:40-46 */
static inline uint64_t sm64_next(sm64 *r) {
    r->s += 0x9E3779B97F4A7C15ULL;
    uint64_t z = r->s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
/* rng.rs:52-58: straight modulo */
static inline uint64_t sm64_index(sm64 *r, uint64_t bound) { return sm64_next(r) % bound; }
/* rng.rs:62-67: top 53 bits times 2^-53 */
static inline double sm64_unit(sm64 *r) {
    uint64_t bits = sm64_next(r) >> 11;
    return (double)bits * (1.0 / 9007199254740992.0);
}
/* rng.rs:79-101: inverse-CDF geometric */
static inline double sm64_geom(sm64 *r, double p) {
    if (p >= 1.0) return 0.0;
    double u = sm64_unit(r);
    double one_minus_u = 1.0 - u;
    if (one_minus_u == 1.0) return 0.0;
    double lp = log(1.0 - p);
    if (lp == 0.0) return INFINITY;
    return floor(log(one_minus_u) / lp);
}

uint64_t or_splitmix_next(uint64_t *state) {
    sm64 r = {*state};
    uint64_t v = sm64_next(&r);
    *state = r.s;
    return v;
}
double or_splitmix_unit(uint64_t *state) {
    sm64 r = {*state};
    double v = sm64_unit(&r);
    *state = r.s;
    return v;
}

void or_free(void *p) { free(p); }

/* growable edge buffer */
typedef struct { uint32_t *f, *t; uint64_t len, cap; } ebuf;
static int eb_push(ebuf *b, uint32_t u, uint32_t v) {
    if (b->len == b->cap) {
        uint64_t nc = b->cap ? b->cap * 2 : 1024;
        uint32_t *nf = (uint32_t *)realloc(b->f, nc * sizeof(uint32_t));
        if (!nf) return -1;
        b->f = nf;
        uint32_t *nt = (uint32_t *)realloc(b->t, nc * sizeof(uint32_t));
        if (!nt) return -1;
        b->t = nt;
        b->cap = nc;
    }
    b->f[b->len] = u;
    b->t[b->len] = v;
    b->len++;
    return 0;
}
/* Graph::add_edges canonicalisation (graph.rs:771-777) */
static int eb_add(ebuf *b, int directed, uint32_t u, uint32_t v) {
    if (!directed && u > v) return eb_push(b, v, u);
    return eb_push(b, u, v);
}
static int64_t eb_finish(ebuf *b, uint32_t **from, uint32_t **to) {
    if (b->len == 0) { /* hand back valid pointers for an empty list */
        free(b->f); free(b->t);
        b->f = (uint32_t *)malloc(4); b->t = (uint32_t *)malloc(4);
    }
    *from = b->f;
    *to = b->t;
    return (int64_t)b->len;
}

/* ---- G(n, m): erdos_renyi.rs:59-170 (decode_pair, max_edges,
 *      distinct_sample) and :328-353 (erdos_renyi_gnm) ---- */

static void decode_pair(uint64_t idx, uint32_t n, int directed, int loops, uint32_t *pf, uint32_t *pt) {
    uint64_t nn = n;
    if (directed && loops) {
        uint64_t to = idx / nn, from = idx - to * nn;
        *pf = (uint32_t)from; *pt = (uint32_t)to;
    } else if (directed && !loops) {
        uint64_t to = idx / nn, from = idx - to * nn;
        if (from == to) to = nn - 1;
        *pf = (uint32_t)from; *pt = (uint32_t)to;
    } else if (!directed && loops) {
        double idx_f = (double)idx;
        double to_f = (sqrt(8.0 * idx_f + 1.0) - 1.0) / 2.0;
        uint64_t to = (uint64_t)trunc(to_f);
        uint64_t from = idx - to * (to + 1) / 2;
        while (from > to) { to += 1; from = idx - to * (to + 1) / 2; }
        *pf = (uint32_t)from; *pt = (uint32_t)to;
    } else {
        double idx_f = (double)idx;
        double to_f = (sqrt(8.0 * idx_f + 1.0) + 1.0) / 2.0;
        uint64_t to = (uint64_t)trunc(to_f);
        if (to < 1) to = 1;
        uint64_t from = idx - to * (to - 1) / 2;
        while (from >= to) { to += 1; from = idx - to * (to - 1) / 2; }
        *pf = (uint32_t)from; *pt = (uint32_t)to;
    }
}

static uint64_t max_edges(uint32_t n, int directed, int loops) {
    uint64_t nn = n, nm1 = n ? nn - 1 : 0;
    if (directed && loops) return nn * nn;
    if (directed) return nn * nm1;
    if (loops) return nn * (nn + 1) / 2;
    return nn * nm1 / 2;
}

/* open-addressing u64 set for Floyd's sampler */
typedef struct { uint64_t *slot; uint64_t mask; } u64set;
static inline uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}
/* returns 1 if inserted, 0 if present */
static int u64set_insert(u64set *s, uint64_t key) {
    uint64_t h = mix64(key) & s->mask;
    for (;;) {
        if (s->slot[h] == UINT64_MAX) { s->slot[h] = key; return 1; }
        if (s->slot[h] == key) return 0;
        h = (h + 1) & s->mask;
    }
}
static int cmp_u64(const void *a, const void *b) {
    uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return x < y ? -1 : x > y;
}

int64_t or_er_gnm(uint32_t n, uint64_t m, int directed, int loops, uint64_t seed, uint32_t **from, uint32_t **to) {
    ebuf b = {0};
    uint64_t cap = max_edges(n, directed, loops);
    if (m > cap) return -1;
    if (m == 0) return eb_finish(&b, from, to);
    if (m == cap) { /* complete(): erdos_renyi.rs:206-235 */
        for (uint32_t i = 0; i < n; i++) {
            if (directed) {
                for (uint32_t j = 0; j < n; j++) {
                    if (i == j && !loops) continue;
                    if (eb_add(&b, directed, i, j)) return -2;
                }
            } else {
                for (uint32_t j = loops ? i : i + 1; j < n; j++)
                    if (eb_add(&b, directed, i, j)) return -2;
            }
        }
        return eb_finish(&b, from, to);
    }
    sm64 rng = {seed};
    uint64_t tsize = 16;
    while (tsize < 2 * m) tsize <<= 1;
    u64set set = {(uint64_t *)malloc(tsize * sizeof(uint64_t)), tsize - 1};
    uint64_t *picks = (uint64_t *)malloc(m * sizeof(uint64_t));
    if (!set.slot || !picks) return -2;
    memset(set.slot, 0xff, tsize * sizeof(uint64_t));
    uint64_t k = 0;
    for (uint64_t j = cap - m; j < cap; j++) {
        uint64_t t = sm64_index(&rng, j + 1);
        uint64_t pick;
        if (u64set_insert(&set, t)) pick = t;
        else { u64set_insert(&set, j); pick = j; }
        picks[k++] = pick;
    }
    free(set.slot);
    qsort(picks, m, sizeof(uint64_t), cmp_u64);
    for (uint64_t i = 0; i < m; i++) {
        uint32_t u, v;
        decode_pair(picks[i], n, directed, loops, &u, &v);
        if (eb_add(&b, directed, u, v)) return -2;
    }
    free(picks);
    return eb_finish(&b, from, to);
}

/* ---- Barabási–Albert bag variant: barabasi.rs:114-179 ---- */
int64_t or_ba_bag(uint32_t n, uint32_t m, int outpref, int directed, uint64_t seed, uint32_t **from, uint32_t **to) {
    ebuf b = {0};
    outpref = outpref || !directed;
    if (n == 0 || n == 1 || m == 0) return eb_finish(&b, from, to);
    uint64_t steps = (uint64_t)n - 1, total = steps * m;
    uint64_t bagcap = (uint64_t)n + total + (outpref ? total : 0);
    uint32_t *bag = (uint32_t *)malloc(bagcap * sizeof(uint32_t));
    uint32_t *ef = (uint32_t *)malloc(total * sizeof(uint32_t));
    uint32_t *et = (uint32_t *)malloc(total * sizeof(uint32_t));
    if (!bag || !ef || !et) return -2;
    uint64_t bl = 0, el = 0;
    bag[bl++] = 0;
    sm64 rng = {seed};
    for (uint32_t i = 1; i < n; i++) {
        uint64_t bag_len = bl, es = el;
        for (uint32_t k = 0; k < m; k++) {
            uint64_t pick = sm64_index(&rng, bag_len);
            ef[el] = i; et[el] = bag[pick]; el++;
        }
        bag[bl++] = i;
        for (uint32_t k = 0; k < m; k++) {
            bag[bl++] = et[es + k];
            if (outpref) bag[bl++] = i;
        }
    }
    free(bag);
    /* Graph::add_edges canonicalisation */
    if (!directed)
        for (uint64_t e = 0; e < el; e++)
            if (ef[e] > et[e]) { uint32_t t = ef[e]; ef[e] = et[e]; et[e] = t; }
    *from = ef;
    *to = et;
    return (int64_t)el;
}

/* ---- SBM: sbm.rs:84-146 (PairShape), :224-258 (sample_pair_with_max),
 *      :307-372 (sbm_game) ---- */
enum { RECT = 0, RECT_NO_DIAG = 1, TRI_INCL = 2, TRI_EXCL = 3 };

static void shape_decode(int shape, uint64_t idx, uint32_t fromsize, uint32_t *pf, uint32_t *pt) {
    uint64_t fs = fromsize;
    if (shape == RECT) {
        uint64_t vto = idx / fs, vfrom = idx - vto * fs;
        *pf = (uint32_t)vfrom; *pt = (uint32_t)vto;
    } else if (shape == RECT_NO_DIAG) {
        uint64_t vto = idx / fs, vfrom = idx - vto * fs;
        if (vfrom == vto) vto = fs - 1;
        *pf = (uint32_t)vfrom; *pt = (uint32_t)vto;
    } else if (shape == TRI_INCL) {
        double idx_f = (double)idx;
        double vto_f = (sqrt(8.0 * idx_f + 1.0) - 1.0) / 2.0;
        uint64_t vto = (uint64_t)trunc(vto_f);
        uint64_t vfrom = idx - vto * (vto + 1) / 2;
        while (vfrom > vto) { vto += 1; vfrom = idx - vto * (vto + 1) / 2; }
        *pf = (uint32_t)vfrom; *pt = (uint32_t)vto;
    } else {
        double idx_f = (double)idx;
        double vto_f = (sqrt(8.0 * idx_f + 1.0) + 1.0) / 2.0;
        uint64_t vto = (uint64_t)trunc(vto_f);
        if (vto < 1) vto = 1;
        uint64_t vfrom = idx - vto * (vto - 1) / 2;
        while (vfrom >= vto) { vto += 1; vfrom = idx - vto * (vto - 1) / 2; }
        *pf = (uint32_t)vfrom; *pt = (uint32_t)vto;
    }
}

int64_t or_sbm(uint32_t k, const double *pref, const uint32_t *sizes, int directed, int loops, int multiple,
               uint64_t seed, uint32_t **from, uint32_t **to) {
    ebuf b = {0};
    uint32_t *off = (uint32_t *)malloc((k + 1) * sizeof(uint32_t));
    uint64_t acc = 0;
    off[0] = 0;
    for (uint32_t i = 0; i < k; i++) { acc += sizes[i]; off[i + 1] = (uint32_t)acc; }
    if (k == 0 || acc == 0) { free(off); return eb_finish(&b, from, to); }
    sm64 rng = {seed};
    for (uint32_t fb = 0; fb < k; fb++) {
        uint32_t fromsize = sizes[fb];
        if (fromsize == 0) continue;
        uint32_t fromoff = off[fb];
        for (uint32_t tb = directed ? 0 : fb; tb < k; tb++) {
            uint32_t tosize = sizes[tb];
            if (tosize == 0) continue;
            uint32_t tooff = off[tb];
            double prob = pref[(uint64_t)fb * k + tb];
            if (prob <= 0.0) continue;
            int diag = fb == tb, shape;
            if (directed && !loops && diag) shape = RECT_NO_DIAG;
            else if (!directed && loops && diag) shape = TRI_INCL;
            else if (!directed && !loops && diag) shape = TRI_EXCL;
            else shape = RECT;
            uint64_t fs = fromsize, maxe;
            if (shape == RECT) maxe = fs * (uint64_t)tosize;
            else if (shape == RECT_NO_DIAG) maxe = fs * (fs ? fs - 1 : 0);
            else if (shape == TRI_INCL) maxe = fs * (fs + 1) / 2;
            else maxe = fs * (fs ? fs - 1 : 0) / 2;
            /* sample_pair_with_max */
            if (maxe == 0 || prob <= 0.0) continue;
            double prob_step = multiple ? prob / (1.0 + prob) : prob;
            if (prob_step <= 0.0) continue;
            double max_f = (double)maxe;
            double step_extra = multiple ? 0.0 : 1.0;
            double last = sm64_geom(&rng, prob_step);
            while (last < max_f) {
                uint64_t idx = (uint64_t)trunc(last);
                if (idx >= maxe) break;
                uint32_t vf, vt;
                shape_decode(shape, idx, fromsize, &vf, &vt);
                if (eb_add(&b, directed, fromoff + vf, tooff + vt)) return -2;
                last += sm64_geom(&rng, prob_step);
                last += step_extra;
            }
        }
    }
    free(off);
    return eb_finish(&b, from, to);
}

/* ---- project R-MAT (no reference counterpart) ----
 * Edge e draws from its own SplitMix64 stream seeded with
 * seed ^ (e * 0xD1B54A32D192ED03); each of `scale` levels draws one
 * gen_unit() r and picks quadrant a (r < t1), b (r < t2), c (r < t3) or d,
 * where t1 = a, t2 = a + b, t3 = a + b + c in double.  Quadrant b sets the
 * column (target) bit, c the row (source) bit, d both.  The CUDA generator
 * uses the identical arithmetic, so edge lists agree bit-for-bit. */
typedef struct { uint32_t scale; uint64_t m; double t1, t2, t3; uint64_t seed; uint32_t *from, *to; } rmat_ctx;
static void rmat_part(void *c_, int t, int nt) {
    rmat_ctx *c = (rmat_ctx *)c_;
    uint64_t lo = c->m * (uint64_t)t / nt, hi = c->m * (uint64_t)(t + 1) / nt;
    for (uint64_t e = lo; e < hi; e++) {
        sm64 r = {c->seed ^ (e * 0xD1B54A32D192ED03ULL)};
        uint32_t u = 0, v = 0;
        for (uint32_t l = 0; l < c->scale; l++) {
            double x = sm64_unit(&r);
            uint32_t rb, cb;
            if (x < c->t1) { rb = 0; cb = 0; }
            else if (x < c->t2) { rb = 0; cb = 1; }
            else if (x < c->t3) { rb = 1; cb = 0; }
            else { rb = 1; cb = 1; }
            u = (u << 1) | rb;
            v = (v << 1) | cb;
        }
        c->from[e] = u;
        c->to[e] = v;
    }
}
void or_rmat(uint32_t scale, uint64_t m, double a, double b, double c, uint64_t seed, uint32_t *from,
             uint32_t *to, int nthreads) {
    rmat_ctx ctx = {scale, m, a, a + b, a + b + c, seed, from, to};
    par_run(nthreads, rmat_part, &ctx);
}

/* Edge weights for the weighted BA workload: w[e] = (float)(lo + (hi-lo)*gen_unit())
 * drawn in edge-id order from SplitMix64(seed), stored as double. */
void or_uniform_weights(uint64_t m, uint64_t seed, double lo, double hi, double *w) {
    sm64 r = {seed};
    for (uint64_t e = 0; e < m; e++) w[e] = (double)(float)(lo + (hi - lo) * sm64_unit(&r));
}

/* ------------------------------------------------------------------ */
/* 2. Reference restatements                                           */
/* ------------------------------------------------------------------ */

#define REF_DAMPING 0.85
#define REF_EPS 1e-10
#define REF_MAX_ITER 1000

/* in_adj as CSR, rows filled in edge-id order exactly as the reference
 * pushes into Vec<Vec<_>> (pagerank.rs:76-101). Returns arc count. */
static uint64_t build_in_adj(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to, int directed,
                             const double *w, uint64_t **rp_out, uint32_t **src_out, double **val_out) {
    uint64_t *rp = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t));
    for (uint64_t e = 0; e < m; e++) {
        uint32_t u = from[e], v = to[e];
        if (directed) rp[v + 1]++;
        else if (u == v) rp[v + 1] += 2;
        else { rp[u + 1]++; rp[v + 1]++; }
    }
    for (uint32_t i = 0; i < n; i++) rp[i + 1] += rp[i];
    uint64_t arcs = rp[n];
    uint64_t *cur = (uint64_t *)malloc(((size_t)n + 1) * sizeof(uint64_t));
    memcpy(cur, rp, ((size_t)n + 1) * sizeof(uint64_t));
    uint32_t *src = (uint32_t *)malloc((arcs ? arcs : 1) * sizeof(uint32_t));
    double *val = w ? (double *)malloc((arcs ? arcs : 1) * sizeof(double)) : NULL;
#define PUSH(row, s, wv)                      \
    do {                                      \
        uint64_t p_ = cur[row]++;             \
        src[p_] = (s);                        \
        if (val) val[p_] = (wv);              \
    } while (0)
    for (uint64_t e = 0; e < m; e++) {
        uint32_t u = from[e], v = to[e];
        double we = w ? w[e] : 0.0;
        if (directed) PUSH(v, u, we);
        else if (u == v) { PUSH(v, u, we); PUSH(v, u, we); }
        else { PUSH(u, v, we); PUSH(v, u, we); }
    }
#undef PUSH
    free(cur);
    *rp_out = rp;
    *src_out = src;
    if (val_out) *val_out = val;
    return arcs;
}

/* out-degree as neighbors_iter(v).len() (graph.rs:877-900): directed counts
 * out-edges; undirected counts out+in lists, so a self-loop counts twice. */
static uint64_t *out_degrees(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to, int directed) {
    uint64_t *deg = (uint64_t *)calloc(n ? n : 1, sizeof(uint64_t));
    for (uint64_t e = 0; e < m; e++) {
        deg[from[e]]++;
        if (!directed) deg[to[e]]++;
    }
    return deg;
}

/* pagerank.rs:52-143 */
int or_pagerank(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to, int directed, double *out,
                uint32_t *iters_out) {
    if (iters_out) *iters_out = 0;
    if (n == 0) return 0;
    if (n == 1) { out[0] = 1.0; return 0; }
    double n_f = (double)n;
    uint64_t *out_deg = out_degrees(n, m, from, to, directed);
    uint64_t *rp; uint32_t *src;
    build_in_adj(n, m, from, to, directed, NULL, &rp, &src, NULL);
    double *pr = (double *)malloc(n * sizeof(double));
    double *pr_new = (double *)calloc(n, sizeof(double));
    for (uint32_t v = 0; v < n; v++) pr[v] = 1.0 / n_f;
    uint32_t it = 0;
    for (uint32_t k = 0; k < REF_MAX_ITER; k++) {
        it++;
        double dangling_sum = 0.0;
        for (uint32_t v = 0; v < n; v++)
            if (out_deg[v] == 0) dangling_sum += pr[v];
        double teleport = (1.0 - REF_DAMPING) / n_f;
        double dangling_share = REF_DAMPING * dangling_sum / n_f;
        for (uint32_t v = 0; v < n; v++) {
            double incoming = 0.0;
            for (uint64_t p = rp[v]; p < rp[v + 1]; p++) {
                uint32_t u = src[p];
                double denom = (double)out_deg[u];
                if (denom > 0.0) incoming += pr[u] / denom;
            }
            pr_new[v] = teleport + dangling_share + REF_DAMPING * incoming;
        }
        double diff = 0.0;
        for (uint32_t v = 0; v < n; v++) diff += fabs(pr_new[v] - pr[v]);
        double *t = pr; pr = pr_new; pr_new = t;
        if (diff < REF_EPS) break;
    }
    memcpy(out, pr, n * sizeof(double));
    if (iters_out) *iters_out = it;
    free(out_deg); free(rp); free(src); free(pr); free(pr_new);
    return 0;
}

/* pagerank_weighted.rs:52-161 (validation stays with the caller) */
int or_pagerank_weighted(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to, int directed,
                         const double *weights, double *out, uint32_t *iters_out) {
    if (iters_out) *iters_out = 0;
    if (n == 0) return 0;
    if (n == 1) { out[0] = 1.0; return 0; }
    double n_f = (double)n;
    double *s = (double *)calloc(n, sizeof(double));
    for (uint64_t e = 0; e < m; e++) {
        uint32_t u = from[e], v = to[e];
        if (directed) s[u] += weights[e];
        else if (u == v) s[u] += 2.0 * weights[e];
        else { s[u] += weights[e]; s[v] += weights[e]; }
    }
    uint64_t *rp; uint32_t *src; double *val;
    build_in_adj(n, m, from, to, directed, weights, &rp, &src, &val);
    double *pr = (double *)malloc(n * sizeof(double));
    double *pr_new = (double *)calloc(n, sizeof(double));
    for (uint32_t v = 0; v < n; v++) pr[v] = 1.0 / n_f;
    uint32_t it = 0;
    for (uint32_t k = 0; k < REF_MAX_ITER; k++) {
        it++;
        double dangling_sum = 0.0;
        for (uint32_t v = 0; v < n; v++)
            if (s[v] == 0.0) dangling_sum += pr[v];
        double teleport = (1.0 - REF_DAMPING) / n_f;
        double dangling_share = REF_DAMPING * dangling_sum / n_f;
        for (uint32_t v = 0; v < n; v++) {
            double incoming = 0.0;
            for (uint64_t p = rp[v]; p < rp[v + 1]; p++) {
                uint32_t u = src[p];
                double su = s[u];
                if (su > 0.0) incoming += val[p] * pr[u] / su;
            }
            pr_new[v] = teleport + dangling_share + REF_DAMPING * incoming;
        }
        double diff = 0.0;
        for (uint32_t v = 0; v < n; v++) diff += fabs(pr_new[v] - pr[v]);
        double *t = pr; pr = pr_new; pr_new = t;
        if (diff < REF_EPS) break;
    }
    memcpy(out, pr, n * sizeof(double));
    if (iters_out) *iters_out = it;
    free(s); free(rp); free(src); free(val); free(pr); free(pr_new);
    return 0;
}

/* personalized_pagerank.rs:65-182 (validation stays with the caller;
 * `reset` is the caller's raw vector, normalised here as :110-111 does) */
int or_personalized_pagerank(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to, int directed,
                             const double *reset, double damping, double *out, uint32_t *iters_out) {
    if (iters_out) *iters_out = 0;
    if (n == 0) return 0;
    if (n == 1) { out[0] = 1.0; return 0; }
    double reset_sum = 0.0;
    for (uint32_t v = 0; v < n; v++) reset_sum += reset[v];
    double inv_sum = 1.0 / reset_sum;
    double *nr = (double *)malloc(n * sizeof(double));
    for (uint32_t v = 0; v < n; v++) nr[v] = reset[v] * inv_sum;
    uint64_t *out_deg = out_degrees(n, m, from, to, directed);
    uint64_t *rp; uint32_t *src;
    build_in_adj(n, m, from, to, directed, NULL, &rp, &src, NULL);
    double *pr = (double *)malloc(n * sizeof(double));
    double *pr_new = (double *)calloc(n, sizeof(double));
    memcpy(pr, nr, n * sizeof(double));
    uint32_t it = 0;
    for (uint32_t k = 0; k < REF_MAX_ITER; k++) {
        it++;
        double dangling_sum = 0.0;
        for (uint32_t v = 0; v < n; v++)
            if (out_deg[v] == 0) dangling_sum += pr[v];
        for (uint32_t v = 0; v < n; v++) {
            double incoming = 0.0;
            for (uint64_t p = rp[v]; p < rp[v + 1]; p++) {
                uint32_t u = src[p];
                double denom = (double)out_deg[u];
                if (denom > 0.0) incoming += pr[u] / denom;
            }
            pr_new[v] = (1.0 - damping) * nr[v] + damping * (incoming + dangling_sum * nr[v]);
        }
        double diff = 0.0;
        for (uint32_t v = 0; v < n; v++) diff += fabs(pr_new[v] - pr[v]);
        double *t = pr; pr = pr_new; pr_new = t;
        if (diff < REF_EPS) break;
    }
    memcpy(out, pr, n * sizeof(double));
    if (iters_out) *iters_out = it;
    free(nr); free(out_deg); free(rp); free(src); free(pr); free(pr_new);
    return 0;
}

/* Residuals of K personalized vectors against the operator of
 * personalized_pagerank.rs:149-182: for column k with reset r_k uniform over
 * seeds[off[k] .. off[k+1]) (duplicates add weight, as _vs builds it at
 * :241-268) and the vector x_k = X[v*K + k] (float, row-major, as the
 * batched solver returns it), res[k] = ||G_k(x_k) - x_k||_1 with
 *   G_k(x)[v] = (1-d) r_k[v] + d (sum_{u->v} x[u]/outdeg[u] + dsum_k(x) r_k[v]),
 * in FP64.  G_k is an L1 contraction with factor d, so ||x_k - x*_k||_1 <=
 * res[k] / (1 - d): a certificate for every column from one pass.
 * Multithreaded over row chunks. */
typedef struct {
    uint32_t n, K; const uint64_t *rp; const uint32_t *src; const double *inv;
    const float *X; const uint64_t *sp; const uint32_t *scol; const double *sw;
    const double *dsum; double damping; double *part; int nchunk;
} pres_ctx;
static void pres_part(void *c_, int t, int nt) {
    pres_ctx *c = (pres_ctx *)c_;
    const uint32_t K = c->K;
    double *acc = (double *)malloc((size_t)K * sizeof(double));
    double *r = (double *)malloc((size_t)K * sizeof(double));
    double *pr = c->part + (size_t)t * K;
    for (uint32_t k = 0; k < K; k++) pr[k] = 0.0;
    for (int ch = t; ch < c->nchunk; ch += nt) {
        uint64_t lo = (uint64_t)c->n * ch / c->nchunk, hi = (uint64_t)c->n * (ch + 1) / c->nchunk;
        for (uint64_t v = lo; v < hi; v++) {
            for (uint32_t k = 0; k < K; k++) { acc[k] = 0.0; r[k] = 0.0; }
            for (uint64_t p = c->rp[v]; p < c->rp[v + 1]; p++) {
                const uint32_t u = c->src[p];
                const double iv = c->inv[u];
                const float *xu = c->X + (size_t)u * K;
                for (uint32_t k = 0; k < K; k++) acc[k] += (double)xu[k] * iv;
            }
            for (uint64_t e = c->sp[v]; e < c->sp[v + 1]; e++) r[c->scol[e]] += c->sw[e];
            const float *xv = c->X + (size_t)v * K;
            for (uint32_t k = 0; k < K; k++) {
                const double g = (1.0 - c->damping) * r[k] + c->damping * (acc[k] + c->dsum[k] * r[k]);
                pr[k] += fabs(g - (double)xv[k]);
            }
        }
    }
    free(acc); free(r);
}
int or_ppr_residuals(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to, int directed, uint32_t K,
                     const uint64_t *off, const uint32_t *seeds, double damping, const float *X, double *res,
                     int nthreads) {
    if (n == 0 || K == 0) return 0;
    if (nthreads < 1) nthreads = 1;
    if (nthreads > 256) nthreads = 256;
    uint64_t *deg = out_degrees(n, m, from, to, directed);
    double *inv = (double *)malloc((size_t)n * sizeof(double));
    for (uint32_t v = 0; v < n; v++) inv[v] = deg[v] ? 1.0 / (double)deg[v] : 0.0;
    uint64_t *rp; uint32_t *src;
    build_in_adj(n, m, from, to, directed, NULL, &rp, &src, NULL);
    /* seed entries as a vertex-major list of (column, weight) */
    const uint64_t S = off[K];
    uint64_t *sp = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t));
    for (uint64_t i = 0; i < S; i++) sp[seeds[i] + 1]++;
    for (uint32_t v = 0; v < n; v++) sp[v + 1] += sp[v];
    uint64_t *cur = (uint64_t *)malloc(((size_t)n + 1) * sizeof(uint64_t));
    memcpy(cur, sp, ((size_t)n + 1) * sizeof(uint64_t));
    uint32_t *scol = (uint32_t *)malloc((S ? S : 1) * sizeof(uint32_t));
    double *sw = (double *)malloc((S ? S : 1) * sizeof(double));
    for (uint32_t k = 0; k < K; k++) {
        const double w = 1.0 / (double)(off[k + 1] - off[k]);
        for (uint64_t i = off[k]; i < off[k + 1]; i++) {
            const uint64_t p = cur[seeds[i]]++;
            scol[p] = k;
            sw[p] = w;
        }
    }
    double *dsum = (double *)calloc(K, sizeof(double));
    for (uint32_t v = 0; v < n; v++)
        if (deg[v] == 0)
            for (uint32_t k = 0; k < K; k++) dsum[k] += (double)X[(size_t)v * K + k];
    double *part = (double *)calloc((size_t)nthreads * K, sizeof(double));
    pres_ctx c = {n, K, rp, src, inv, X, sp, scol, sw, dsum, damping, part, 1024};
    par_run(nthreads, pres_part, &c);
    for (uint32_t k = 0; k < K; k++) {
        double tot = 0.0;
        for (int t = 0; t < nthreads; t++) tot += part[(size_t)t * K + k];
        res[k] = tot;
    }
    free(deg); free(inv); free(rp); free(src); free(sp); free(cur); free(scol); free(sw); free(dsum); free(part);
    return 0;
}

/* Timed CPU-baseline kernel: `iters` iterations of the pagerank.rs:107-140
 * loop over a prebuilt in-adjacency, starting from the uniform vector. The
 * adjacency build (pagerank.rs:63-101) is a separate call so the two phases
 * are timed apart.  Handle-based so bench.py can build once. */
typedef struct { uint32_t n; uint64_t arcs; uint64_t *rp; uint32_t *src; uint64_t *deg; } or_adj;

void *or_adj_build(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to, int directed) {
    or_adj *a = (or_adj *)malloc(sizeof(or_adj));
    a->n = n;
    a->deg = out_degrees(n, m, from, to, directed);
    a->arcs = build_in_adj(n, m, from, to, directed, NULL, &a->rp, &a->src, NULL);
    return a;
}
void or_adj_free(void *h) {
    or_adj *a = (or_adj *)h;
    if (!a) return;
    free(a->rp); free(a->src); free(a->deg); free(a);
}
uint64_t or_adj_arcs(void *h) { return ((or_adj *)h)->arcs; }

/* Runs exactly `iters` reference iterations (no early stop), returns the last diff. */
double or_adj_iterate(void *h, uint32_t iters, double *pr_io) {
    or_adj *a = (or_adj *)h;
    uint32_t n = a->n;
    double n_f = (double)n, diff = 0.0;
    double *pr = pr_io;
    double *pr_new = (double *)malloc(n * sizeof(double));
    for (uint32_t k = 0; k < iters; k++) {
        double dangling_sum = 0.0;
        for (uint32_t v = 0; v < n; v++)
            if (a->deg[v] == 0) dangling_sum += pr[v];
        double teleport = (1.0 - REF_DAMPING) / n_f;
        double dangling_share = REF_DAMPING * dangling_sum / n_f;
        for (uint32_t v = 0; v < n; v++) {
            double incoming = 0.0;
            for (uint64_t p = a->rp[v]; p < a->rp[v + 1]; p++) {
                uint32_t u = a->src[p];
                double denom = (double)a->deg[u];
                if (denom > 0.0) incoming += pr[u] / denom;
            }
            pr_new[v] = teleport + dangling_share + REF_DAMPING * incoming;
        }
        diff = 0.0;
        for (uint32_t v = 0; v < n; v++) diff += fabs(pr_new[v] - pr[v]);
        memcpy(pr, pr_new, n * sizeof(double));
    }
    free(pr_new);
    return diff;
}

/* ------------------------------------------------------------------ */
/* 3. Tight FP64 oracle                                                */
/* ------------------------------------------------------------------ */

/* Neumaier-compensated accumulator */
typedef struct { double s, c; } kahan;
static inline void kadd(kahan *k, double x) {
    double t = k->s + x;
    if (fabs(k->s) >= fabs(x)) k->c += (k->s - t) + x;
    else k->c += (x - t) + k->s;
    k->s = t;
}
static inline double kval(const kahan *k) { return k->s + k->c; }

typedef struct {
    uint32_t n; const uint64_t *rp; const uint32_t *src; const double *val;
    const double *xt, *x; double *xn; const double *r; double damping, dsum; double *part_d; int nchunk;
} tight_ctx;
static void tight_part(void *c_, int t, int nt) {
    tight_ctx *c = (tight_ctx *)c_;
    for (int ch = t; ch < c->nchunk; ch += nt) {
        uint64_t lo = (uint64_t)c->n * ch / c->nchunk, hi = (uint64_t)c->n * (ch + 1) / c->nchunk;
        kahan kdf = {0, 0};
        for (uint64_t v = lo; v < hi; v++) {
            kahan acc = {0, 0};
            for (uint64_t p = c->rp[v]; p < c->rp[v + 1]; p++)
                kadd(&acc, (c->val ? c->val[p] : 1.0) * c->xt[c->src[p]]);
            kahan tot = {0, 0};
            kadd(&tot, c->damping * kval(&acc));
            kadd(&tot, c->damping * c->dsum * c->r[v]);
            kadd(&tot, (1.0 - c->damping) * c->r[v]);
            c->xn[v] = kval(&tot);
            kadd(&kdf, fabs(c->xn[v] - c->x[v]));
        }
        c->part_d[ch] = kval(&kdf);
    }
}

/* Fixed point of the reference operator
 *   x = d*P^T x + d*(sum_{dangling} x)*r + (1-d)*r
 * (r = uniform 1/n when reset == NULL, else the normalised reset; weights
 * optional) iterated with compensated sums until the successive L1 change is
 * below `tol`.  Starts from `out` if start_from_out != 0, else from r.
 * Returns the iteration count; writes the final successive change to *last_diff. */
int64_t or_pagerank_tight(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to, int directed,
                          const double *weights, const double *reset, double damping, double tol,
                          uint32_t max_iter, int start_from_out, double *out, double *last_diff,
                          int nthreads) {
    if (n == 0) return 0;
    if (n == 1) { out[0] = 1.0; return 0; }
    double *r = (double *)malloc(n * sizeof(double));
    if (reset) {
        kahan ks = {0, 0};
        for (uint32_t v = 0; v < n; v++) kadd(&ks, reset[v]);
        double sum = kval(&ks);
        for (uint32_t v = 0; v < n; v++) r[v] = reset[v] / sum;
    } else {
        for (uint32_t v = 0; v < n; v++) r[v] = 1.0 / (double)n;
    }
    /* out-strength (weights) or out-degree */
    double *s = (double *)calloc(n, sizeof(double));
    for (uint64_t e = 0; e < m; e++) {
        uint32_t u = from[e], v = to[e];
        double we = weights ? weights[e] : 1.0;
        if (directed) s[u] += we;
        else if (u == v) s[u] += 2.0 * we;
        else { s[u] += we; s[v] += we; }
    }
    uint64_t *rp; uint32_t *src; double *val = NULL;
    build_in_adj(n, m, from, to, directed, weights, &rp, &src, weights ? &val : NULL);
    double *x = (double *)malloc(n * sizeof(double));
    double *xt = (double *)malloc(n * sizeof(double));
    double *xn = (double *)malloc(n * sizeof(double));
    if (start_from_out) memcpy(x, out, n * sizeof(double));
    else memcpy(x, r, n * sizeof(double));
    int64_t it = 0;
    double diff = INFINITY;
    int nchunk = 256;
    double *part_d = (double *)malloc(nchunk * 2 * sizeof(double));
    while (it < (int64_t)max_iter) {
        it++;
        kahan kd = {0, 0};
        for (uint32_t v = 0; v < n; v++) {
            if (s[v] == 0.0) { kadd(&kd, x[v]); xt[v] = 0.0; }
            else xt[v] = x[v] / s[v];
        }
        double dsum = kval(&kd);
        tight_ctx tc = {n, rp, src, val, xt, x, xn, r, damping, dsum, part_d, nchunk};
        par_run(nthreads, tight_part, &tc);
        kahan kdiff = {0, 0};
        for (int c = 0; c < nchunk; c++) kadd(&kdiff, part_d[c]);
        diff = kval(&kdiff);
        double *t = x; x = xn; xn = t;
        if (diff < tol) break;
    }
    memcpy(out, x, n * sizeof(double));
    if (last_diff) *last_diff = diff;
    free(r); free(s); free(rp); free(src); free(val); free(x); free(xt); free(xn); free(part_d);
    return it;
}

/* ------------------------------------------------------------------------
 * Eigenvector centrality and HITS (unweighted).  Neighbour lists are sorted
 * ascending, the order the reference's index (rebuild_indexes sorts by
 * (from, to) and (to, from), graph.rs:1708-1768) gives neighbors() /
 * out_neighbors_vec() / in_neighbors_vec(), so the sums run in its order.
 * ---------------------------------------------------------------------- */

static int cmp_u32(const void *a, const void *b) {
    const uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
    return x < y ? -1 : x > y;
}

/* rows[v] = sorted list of key->val pairs grouped by key (counting sort,
 * then each row sorted ascending). */
static void sorted_lists(uint32_t n, uint64_t cnt, const uint32_t *key, const uint32_t *val, uint64_t **rp_out,
                         uint32_t **col_out) {
    uint64_t *rp = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t));
    uint32_t *col = (uint32_t *)malloc((cnt ? cnt : 1) * sizeof(uint32_t));
    for (uint64_t i = 0; i < cnt; i++) rp[key[i] + 1]++;
    for (uint32_t v = 0; v < n; v++) rp[v + 1] += rp[v];
    uint64_t *pos = (uint64_t *)malloc(((size_t)n + 1) * sizeof(uint64_t));
    memcpy(pos, rp, ((size_t)n + 1) * sizeof(uint64_t));
    for (uint64_t i = 0; i < cnt; i++) col[pos[key[i]]++] = val[i];
    for (uint32_t v = 0; v < n; v++) qsort(col + rp[v], rp[v + 1] - rp[v], sizeof(uint32_t), cmp_u32);
    free(pos);
    *rp_out = rp;
    *col_out = col;
}

/* Undirected neighbour lists: each edge in both rows, a loop twice. */
static void undirected_lists(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to, uint64_t **rp,
                             uint32_t **col) {
    uint32_t *k = (uint32_t *)malloc((2 * m + 1) * sizeof(uint32_t));
    uint32_t *v = (uint32_t *)malloc((2 * m + 1) * sizeof(uint32_t));
    for (uint64_t e = 0; e < m; e++) {
        k[2 * e] = from[e];
        v[2 * e] = to[e];
        k[2 * e + 1] = to[e];
        v[2 * e + 1] = from[e];
    }
    sorted_lists(n, 2 * m, k, v, rp, col);
    free(k);
    free(v);
}

static double rescale_max_abs(double *x, uint32_t n) {
    double mx = 0.0;
    for (uint32_t i = 0; i < n; i++) mx = fmax(mx, fabs(x[i]));
    if (mx > 0.0)
        for (uint32_t i = 0; i < n; i++) x[i] /= mx;
    return mx;
}

/* eigenvector_centrality, undirected and unweighted (eigenvector.rs:286-372):
 * x = 1; repeat x' = (A + I) x, x' /= max|x'|, until sum|x' - x| < 1e-14
 * or 5000 iterations; eigenvalue = Rayleigh quotient x.Ax / x.x; negatives
 * clamped to 0.  Returns the iterations run. */
int or_eigenvector_centrality(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to, double *out,
                              double *eigval) {
    if (n == 0) return 0;
    if (m == 0 || n == 1) {
        for (uint32_t i = 0; i < n; i++) out[i] = 1.0;
        if (eigval) *eigval = 0.0;
        return 0;
    }
    uint64_t *rp;
    uint32_t *col;
    undirected_lists(n, m, from, to, &rp, &col);
    double *x = (double *)malloc(n * sizeof(double)), *xn = (double *)malloc(n * sizeof(double));
    for (uint32_t i = 0; i < n; i++) x[i] = 1.0;
    int it = 0;
    for (; it < 5000;) {
        it++;
        for (uint32_t v = 0; v < n; v++) {
            double s = x[v];
            for (uint64_t p = rp[v]; p < rp[v + 1]; p++) s += x[col[p]];
            xn[v] = s;
        }
        rescale_max_abs(xn, n);
        double diff = 0.0;
        for (uint32_t v = 0; v < n; v++) diff += fabs(xn[v] - x[v]);
        double *t = x; x = xn; xn = t;
        if (diff < 1e-14) break;
    }
    double num = 0.0, den = 0.0;
    for (uint32_t v = 0; v < n; v++) {
        double s = 0.0;
        for (uint64_t p = rp[v]; p < rp[v + 1]; p++) s += x[col[p]];
        num += x[v] * s;
        den += x[v] * x[v];
    }
    if (eigval) *eigval = den > 0.0 ? num / den : 0.0;
    for (uint32_t v = 0; v < n; v++) out[v] = x[v] < 0.0 ? 0.0 : x[v];
    free(rp); free(col); free(x); free(xn);
    return it;
}

/* hub_and_authority_scores, unweighted (hits.rs:122-230).  Directed: h = out-degrees
 * max-normalised; repeat tmp = A^T h, h' = A tmp, eigenvalue = max|h'|, h' /= it,
 * until sum|h' - h| < 1e-12 or 5000 iterations; then clamp, authority = A^T h
 * rescaled and clamped.  Undirected: hub = authority = eigenvector
 * centrality, eigenvalue = (Rayleigh quotient of A)^2 (hits.rs:131-141, 586-605). */
int or_hits(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to, int directed, double *hub,
            double *auth, double *eigval) {
    if (n == 0) return 0;
    if (!directed) {
        double lam = 0.0;
        int it = or_eigenvector_centrality(n, m, from, to, hub, NULL);
        memcpy(auth, hub, n * sizeof(double));
        if (m > 0) {
            uint64_t *rp;
            uint32_t *col;
            undirected_lists(n, m, from, to, &rp, &col);
            double num = 0.0, den = 0.0;
            for (uint32_t v = 0; v < n; v++) {
                double s = 0.0;
                for (uint64_t p = rp[v]; p < rp[v + 1]; p++) s += hub[col[p]];
                den += hub[v] * hub[v];
                num += hub[v] * s;
            }
            lam = den > 0.0 ? num / den : 0.0;
            free(rp); free(col);
        }
        if (eigval) *eigval = lam * lam;
        return it;
    }
    if (m == 0) {
        for (uint32_t i = 0; i < n; i++) hub[i] = auth[i] = 1.0;
        if (eigval) *eigval = 0.0;
        return 0;
    }
    uint64_t *orp, *irp;
    uint32_t *ocol, *icol;
    sorted_lists(n, m, from, to, &orp, &ocol);  /* out_adj[u] = targets */
    sorted_lists(n, m, to, from, &irp, &icol);  /* in_adj[v] = sources */
    double *h = (double *)malloc(n * sizeof(double)), *hn = (double *)malloc(n * sizeof(double));
    double *tmp = (double *)malloc(n * sizeof(double));
    for (uint32_t u = 0; u < n; u++) h[u] = (double)(orp[u + 1] - orp[u]);
    rescale_max_abs(h, n);
    double lam = 0.0;
    int it = 0;
    for (; it < 5000;) {
        it++;
        for (uint32_t v = 0; v < n; v++) {
            double s = 0.0;
            for (uint64_t p = irp[v]; p < irp[v + 1]; p++) s += h[icol[p]];
            tmp[v] = s;
        }
        for (uint32_t u = 0; u < n; u++) {
            double s = 0.0;
            for (uint64_t p = orp[u]; p < orp[u + 1]; p++) s += tmp[ocol[p]];
            hn[u] = s;
        }
        double mx = 0.0;
        for (uint32_t u = 0; u < n; u++) mx = fmax(mx, fabs(hn[u]));
        if (mx > 0.0) {
            lam = mx;
            for (uint32_t u = 0; u < n; u++) hn[u] /= mx;
        }
        double diff = 0.0;
        for (uint32_t u = 0; u < n; u++) diff += fabs(hn[u] - h[u]);
        double *t = h; h = hn; hn = t;
        if (diff < 1e-12) break;
    }
    for (uint32_t u = 0; u < n; u++) hub[u] = h[u] < 0.0 ? 0.0 : h[u];
    for (uint32_t v = 0; v < n; v++) {
        double s = 0.0;
        for (uint64_t p = irp[v]; p < irp[v + 1]; p++) s += hub[icol[p]];
        auth[v] = s;
    }
    rescale_max_abs(auth, n);
    for (uint32_t v = 0; v < n; v++) if (auth[v] < 0.0) auth[v] = 0.0;
    if (eigval) *eigval = lam;
    free(orp); free(irp); free(ocol); free(icol); free(h); free(hn); free(tmp);
    return it;
}

/* ---- weighted variants: incident-edge lists in the reference's order ----
 * Undirected incident(v) = the out-range (edges with from == v, sorted by
 * to) followed by the in-range (edges with to == v, sorted by from); a loop
 * is in both (graph.rs:1212-1225).  Directed: out-range / in-range only.
 * Ties (parallel edges) keep edge-id order. */

typedef struct { uint32_t key, other, e; } kev;
static int cmp_kev(const void *a, const void *b) {
    const kev *x = (const kev *)a, *y = (const kev *)b;
    if (x->key != y->key) return x->key < y->key ? -1 : 1;
    if (x->other != y->other) return x->other < y->other ? -1 : 1;
    return x->e < y->e ? -1 : x->e > y->e;
}

/* rows of (other endpoint, edge) pairs grouped by key, sorted by other */
static void edge_rows(uint32_t n, uint64_t m, const uint32_t *key, const uint32_t *other, uint64_t **rp_out,
                      uint32_t **oth_out, uint32_t **eid_out) {
    kev *t = (kev *)malloc((m ? m : 1) * sizeof(kev));
    for (uint64_t e = 0; e < m; e++) t[e] = (kev){key[e], other[e], (uint32_t)e};
    qsort(t, m, sizeof(kev), cmp_kev);
    uint64_t *rp = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t));
    uint32_t *oth = (uint32_t *)malloc((m ? m : 1) * sizeof(uint32_t)), *eid = (uint32_t *)malloc((m ? m : 1) * 4);
    for (uint64_t i = 0; i < m; i++) {
        rp[t[i].key + 1]++;
        oth[i] = t[i].other;
        eid[i] = t[i].e;
    }
    for (uint32_t v = 0; v < n; v++) rp[v + 1] += rp[v];
    free(t);
    *rp_out = rp;
    *oth_out = oth;
    *eid_out = eid;
}

/* The signed component of greatest magnitude, the first in index order on
 * ties (eigenvector.rs:464-476, hits.rs:399-411): the pivot with negative
 * weights. */
static double signed_pivot(const double *x, uint32_t n) {
    double best = 0.0, sg = 0.0;
    for (uint32_t i = 0; i < n; i++)
        if (fabs(x[i]) > best) {
            best = fabs(x[i]);
            sg = x[i];
        }
    return sg;
}

static int any_negative_w(const double *w, uint64_t m) {
    for (uint64_t e = 0; e < m; e++)
        if (w[e] < 0.0) return 1;
    return 0;
}

/* The reference's "symmetric" weighted iteration over incident edges:
 * undirected graphs walk the out-range then the in-range of v (a loop twice);
 * out_only walks the out-edges alone, which is what graph.incident gives on a
 * directed graph.  Seed: the strength s of v's incident edges, |s| for
 * eigenvector centrality (eigenvector.rs:413-443) or s itself for HITS
 * (hits.rs:483-503); with negative weights a zero strength on a non-empty
 * list seeds 1; all zero -> ones; max-abs rescaled.  x' = x + W x, divided by
 * the max |x'| (the signed pivot with negative weights), until the L1 change
 * < 1e-12 or 5000 iterations.  Eigenvector form: eigenvalue = x.Wx / x.x,
 * then rescale and (non-negative weights) clamp.  HITS form: clamp
 * (non-negative weights), then eigenvalue = x.Wx / x.x of the result. */
static int weighted_core(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to, const double *w,
                         int out_only, int hits_form, double *out, double *eigval) {
    const int neg = any_negative_w(w, m);
    uint64_t *orp, *irp = NULL;
    uint32_t *ooth, *oeid, *ioth = NULL, *ieid = NULL;
    edge_rows(n, m, from, to, &orp, &ooth, &oeid);
    if (!out_only) edge_rows(n, m, to, from, &irp, &ioth, &ieid);
    double *x = (double *)malloc(n * sizeof(double)), *xn = (double *)malloc(n * sizeof(double));
    int any = 0;
    for (uint32_t v = 0; v < n; v++) {
        double s = 0.0;
        uint64_t deg = orp[v + 1] - orp[v];
        for (uint64_t p = orp[v]; p < orp[v + 1]; p++) s += w[oeid[p]];
        if (!out_only) {
            for (uint64_t p = irp[v]; p < irp[v + 1]; p++) s += w[ieid[p]];
            deg += irp[v + 1] - irp[v];
        }
        if (s != 0.0) x[v] = hits_form ? s : fabs(s);
        else x[v] = (neg && deg > 0) ? 1.0 : 0.0;
        any |= x[v] != 0.0;
    }
    if (!any)
        for (uint32_t v = 0; v < n; v++) x[v] = 1.0;
    rescale_max_abs(x, n);
#define WX(v, vec) ({                                                               \
        double s_ = 0.0;                                                            \
        for (uint64_t p = orp[v]; p < orp[v + 1]; p++) s_ += w[oeid[p]] * vec[ooth[p]];  \
        if (!out_only)                                                              \
            for (uint64_t p = irp[v]; p < irp[v + 1]; p++) s_ += w[ieid[p]] * vec[ioth[p]]; \
        s_; })
    int it = 0;
    while (it < 5000) {
        it++;
        for (uint32_t v = 0; v < n; v++) xn[v] = x[v] + WX(v, x);
        if (neg) {
            const double pv = signed_pivot(xn, n);
            if (pv != 0.0)
                for (uint32_t v = 0; v < n; v++) xn[v] /= pv;
        } else {
            rescale_max_abs(xn, n);
        }
        double diff = 0.0;
        for (uint32_t v = 0; v < n; v++) diff += fabs(xn[v] - x[v]);
        double *t = x; x = xn; xn = t;
        if (diff < 1e-12) break;
    }
    if (!hits_form) {
        double num = 0.0, den = 0.0;
        for (uint32_t v = 0; v < n; v++) {
            num += x[v] * WX(v, x);
            den += x[v] * x[v];
        }
        if (eigval) *eigval = den > 0.0 ? num / den : 0.0;
        rescale_max_abs(x, n);
    }
    if (!neg)
        for (uint32_t v = 0; v < n; v++) if (x[v] < 0.0) x[v] = 0.0;
    if (hits_form) {
        double num = 0.0, den = 0.0;
        for (uint32_t v = 0; v < n; v++) {
            num += x[v] * WX(v, x);
            den += x[v] * x[v];
        }
        if (eigval) *eigval = den > 0.0 ? num / den : 0.0;
    }
#undef WX
    memcpy(out, x, n * sizeof(double));
    free(orp); free(ooth); free(oeid); free(irp); free(ioth); free(ieid); free(x); free(xn);
    return it;
}

/* eigenvector_centrality_weighted (eigenvector.rs:375-538): n == 0 -> empty;
 * m == 0, all-zero weights or n == 1 -> ones, eigenvalue 0; otherwise the
 * weighted core in its eigenvector form.  Returns iterations. */
int or_eigenvector_weighted(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to, const double *w,
                            double *out, double *eigval) {
    if (eigval) *eigval = 0.0;
    if (n == 0) return 0;
    int allzero = 1;
    for (uint64_t e = 0; e < m; e++) allzero &= w[e] == 0.0;
    if (m == 0 || allzero || n == 1) {
        for (uint32_t i = 0; i < n; i++) out[i] = 1.0;
        return 0;
    }
    return weighted_core(n, m, from, to, w, 0, 0, out, eigval);
}

/* hub_and_authority_scores_weighted (hits.rs:288-470).  m == 0 or all-zero
 * weights -> ones.  Undirected: the weighted core in its HITS form, hub =
 * authority, eigenvalue = (x.Wx / x.x)^2.  Directed: h = out-strength (with
 * negative weights a zero strength on a non-empty out-list seeds 1), max-abs
 * rescaled; tmp = W^T h, h' = W tmp, divided by max |h'| (the signed pivot
 * with negative weights), which is the eigenvalue estimate; L1 stop 1e-12;
 * clamp (non-negative weights); authority = W^T h, max-abs rescaled, clamped
 * likewise. */
int or_hits_weighted(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to, const double *w, int directed,
                     double *hub, double *auth, double *eigval) {
    if (eigval) *eigval = 0.0;
    if (n == 0) return 0;
    int allzero = 1;
    for (uint64_t e = 0; e < m; e++) allzero &= w[e] == 0.0;
    if (m == 0 || allzero) {
        for (uint32_t i = 0; i < n; i++) hub[i] = auth[i] = 1.0;
        return 0;
    }
    if (!directed) {
        double lam = 0.0;
        int it = weighted_core(n, m, from, to, w, 0, 1, hub, &lam);
        memcpy(auth, hub, n * sizeof(double));
        if (eigval) *eigval = lam * lam;
        return it;
    }
    const int neg = any_negative_w(w, m);
    uint64_t *orp, *irp;
    uint32_t *ooth, *oeid, *ioth, *ieid;
    edge_rows(n, m, from, to, &orp, &ooth, &oeid);  /* out_inc[u]: targets */
    edge_rows(n, m, to, from, &irp, &ioth, &ieid);  /* in_inc[v]: sources */
    double *h = (double *)malloc(n * sizeof(double)), *hn = (double *)malloc(n * sizeof(double));
    double *tmp = (double *)malloc(n * sizeof(double));
    for (uint32_t u = 0; u < n; u++) {
        double s = 0.0;
        for (uint64_t p = orp[u]; p < orp[u + 1]; p++) s += w[oeid[p]];
        h[u] = s != 0.0 ? s : ((neg && orp[u + 1] > orp[u]) ? 1.0 : 0.0);
    }
    rescale_max_abs(h, n);
    double lam = 0.0;
    int it = 0;
    for (; it < 5000;) {
        it++;
        for (uint32_t v = 0; v < n; v++) {
            double s = 0.0;
            for (uint64_t p = irp[v]; p < irp[v + 1]; p++) s += w[ieid[p]] * h[ioth[p]];
            tmp[v] = s;
        }
        for (uint32_t u = 0; u < n; u++) {
            double s = 0.0;
            for (uint64_t p = orp[u]; p < orp[u + 1]; p++) s += w[oeid[p]] * tmp[ooth[p]];
            hn[u] = s;
        }
        double scale;
        if (neg) {
            scale = signed_pivot(hn, n);
        } else {
            scale = 0.0;
            for (uint32_t u = 0; u < n; u++) scale = fmax(scale, fabs(hn[u]));
        }
        if (scale != 0.0) {
            lam = scale;
            for (uint32_t u = 0; u < n; u++) hn[u] /= scale;
        }
        double diff = 0.0;
        for (uint32_t u = 0; u < n; u++) diff += fabs(hn[u] - h[u]);
        double *t = h; h = hn; hn = t;
        if (diff < 1e-12) break;
    }
    for (uint32_t u = 0; u < n; u++) hub[u] = (!neg && h[u] < 0.0) ? 0.0 : h[u];
    for (uint32_t v = 0; v < n; v++) {
        double s = 0.0;
        for (uint64_t p = irp[v]; p < irp[v + 1]; p++) s += w[ieid[p]] * hub[ioth[p]];
        auth[v] = s;
    }
    rescale_max_abs(auth, n);
    if (!neg)
        for (uint32_t v = 0; v < n; v++) if (auth[v] < 0.0) auth[v] = 0.0;
    if (eigval) *eigval = lam;
    free(orp); free(irp); free(ooth); free(oeid); free(ioth); free(ieid); free(h); free(hn); free(tmp);
    return it;
}

/* Infomap's flow model, node flows (community/infomap.rs:233-355):
 * out-adjacency lists in edge-id order (an undirected edge u-v appends (v, w)
 * to u's list and then (u, w) to v's), out-strength summed in edge order,
 * teleport weights vw / sum(vw) (uniform 1/n without them), in-adjacency
 * filled in ascending source order with w / out_strength[u], then from
 * pr = 1/n: buf = tau t + (1 - tau) link + dangling_sum t, buf /= sum(buf),
 * until the L1 change < 1e-10 or 1000 iterations (tau = 0.15).  ew / vw may
 * be NULL.  Returns the iteration count. */
int or_infomap_flow(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to, int directed,
                    const double *ew, const double *vw, double *out) {
    const double tau = 0.15, eps = 1e-10;
    if (n == 0) return 0;
    if (n == 1) {
        out[0] = 1.0;
        return 0;
    }
    const uint64_t arcs = directed ? m : 2 * m;
    uint64_t *orp = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t));
    uint32_t *ov = (uint32_t *)malloc((arcs ? arcs : 1) * sizeof(uint32_t));
    double *ow = (double *)malloc((arcs ? arcs : 1) * sizeof(double));
    double *str = (double *)calloc(n, sizeof(double));
    for (uint64_t e = 0; e < m; e++) {
        orp[from[e] + 1]++;
        if (!directed) orp[to[e] + 1]++;
    }
    for (uint32_t v = 0; v < n; v++) orp[v + 1] += orp[v];
    uint64_t *cur = (uint64_t *)malloc(((size_t)n + 1) * sizeof(uint64_t));
    memcpy(cur, orp, ((size_t)n + 1) * sizeof(uint64_t));
    for (uint64_t e = 0; e < m; e++) {
        const uint32_t u = from[e], v = to[e];
        const double w = ew ? ew[e] : 1.0;
        ov[cur[u]] = v;
        ow[cur[u]++] = w;
        str[u] += w;
        if (!directed) {
            ov[cur[v]] = u;
            ow[cur[v]++] = w;
            str[v] += w;
        }
    }
    double *t = (double *)malloc(n * sizeof(double));
    double vs = 0.0;
    if (vw)
        for (uint32_t v = 0; v < n; v++) vs += vw[v];
    for (uint32_t v = 0; v < n; v++) t[v] = (vw && vs > 0.0) ? vw[v] / vs : 1.0 / (double)n;
    /* in-adjacency: ascending u, each u's out-list in order */
    uint64_t *irp = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t));
    for (uint32_t u = 0; u < n; u++)
        if (str[u] > 0.0)
            for (uint64_t p = orp[u]; p < orp[u + 1]; p++) irp[ov[p] + 1]++;
    for (uint32_t v = 0; v < n; v++) irp[v + 1] += irp[v];
    const uint64_t ia = irp[n];
    uint32_t *iu = (uint32_t *)malloc((ia ? ia : 1) * sizeof(uint32_t));
    double *iw = (double *)malloc((ia ? ia : 1) * sizeof(double));
    memcpy(cur, irp, ((size_t)n + 1) * sizeof(uint64_t));
    for (uint32_t u = 0; u < n; u++)
        if (str[u] > 0.0)
            for (uint64_t p = orp[u]; p < orp[u + 1]; p++) {
                const uint32_t v = ov[p];
                iu[cur[v]] = u;
                iw[cur[v]++] = ow[p] / str[u];
            }
    double *pr = (double *)malloc(n * sizeof(double)), *buf = (double *)malloc(n * sizeof(double));
    for (uint32_t v = 0; v < n; v++) pr[v] = 1.0 / (double)n;
    int it = 0;
    while (it < 1000) {
        it++;
        double ds = 0.0;
        for (uint32_t v = 0; v < n; v++)
            if (str[v] <= 0.0) ds += pr[v];
        for (uint32_t v = 0; v < n; v++) {
            double link = 0.0;
            for (uint64_t p = irp[v]; p < irp[v + 1]; p++) link += pr[iu[p]] * iw[p];
            buf[v] = tau * t[v] + (1.0 - tau) * link + ds * t[v];
        }
        double s = 0.0;
        for (uint32_t v = 0; v < n; v++) s += buf[v];
        if (s > 0.0)
            for (uint32_t v = 0; v < n; v++) buf[v] /= s;
        double diff = 0.0;
        for (uint32_t v = 0; v < n; v++) diff += fabs(pr[v] - buf[v]);
        double *tmp = pr;
        pr = buf;
        buf = tmp;
        if (diff < eps) break;
    }
    memcpy(out, pr, n * sizeof(double));
    free(orp); free(ov); free(ow); free(str); free(cur); free(t); free(irp); free(iu); free(iw); free(pr); free(buf);
    return it;
}

/* Kahn's algorithm: 1 when the directed graph has no cycle (a loop is one). */
static int is_dag(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to) {
    uint64_t *orp = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t));
    uint32_t *oc = (uint32_t *)malloc((m ? m : 1) * sizeof(uint32_t));
    uint32_t *indeg = (uint32_t *)calloc(n ? n : 1, sizeof(uint32_t));
    uint32_t *queue = (uint32_t *)malloc((n ? n : 1) * sizeof(uint32_t));
    for (uint64_t e = 0; e < m; e++) {
        orp[from[e] + 1]++;
        indeg[to[e]]++;
    }
    for (uint32_t v = 0; v < n; v++) orp[v + 1] += orp[v];
    uint64_t *cur = (uint64_t *)malloc(((size_t)n + 1) * sizeof(uint64_t));
    memcpy(cur, orp, ((size_t)n + 1) * sizeof(uint64_t));
    for (uint64_t e = 0; e < m; e++) oc[cur[from[e]]++] = to[e];
    uint32_t head = 0, tail = 0;
    for (uint32_t v = 0; v < n; v++)
        if (indeg[v] == 0) queue[tail++] = v;
    while (head < tail) {
        const uint32_t u = queue[head++];
        for (uint64_t p = orp[u]; p < orp[u + 1]; p++)
            if (--indeg[oc[p]] == 0) queue[tail++] = oc[p];
    }
    free(orp); free(oc); free(indeg); free(queue); free(cur);
    return tail == n;
}

/* eigenvector_centrality_full (eigenvector.rs:238-285), weights of either
 * sign (w may be NULL = unit): mode 0 = Out, 1 = In, 2 = All.
 * Undirected graphs take All.  All on a directed graph runs the "undirected"
 * routines over what graph.neighbors / graph.incident return there, the
 * out-edges only (graph.rs:808-819, 1212-1217): unweighted x' = x + sum over
 * ascending out-neighbours (eps 1e-14); weighted x' = x + sum over out-edges
 * in (target, edge id) order with an out-strength seed (eps 1e-12).
 * Out / In (directed_path, eigenvector.rs:539-720): m == 0 or all-zero
 * weights -> ones; a DAG -> 1 on vertices with zero out-strength (Out) / zero
 * in-strength (In), 0 elsewhere, eigenvalue 0; else walk the in-edges (Out)
 * / out-edges (In) of v in edge order, seed |strength| of that walk
 * (all-zero -> ones) max-normalised, shift = max(max walk strength, 1) + 1,
 * x' = shift x + M x max-normalised until the L1 change < 1e-12 (5000
 * iterations); eigenvalue = x.Mx / x.x, and <= 1e-12 gives zeros.  With a
 * negative weight: no DAG short-circuit, a zero strength on a non-empty walk
 * seeds 1, the signed pivot normalises, and neither the zero rule nor the
 * clamp applies. */
int or_eigenvector_full(uint32_t n, uint64_t m, const uint32_t *from, const uint32_t *to, int directed, int mode,
                        const double *w, double *out, double *eigval) {
    if (eigval) *eigval = 0.0;
    if (!directed) {
        if (w) return or_eigenvector_weighted(n, m, from, to, w, out, eigval);
        return or_eigenvector_centrality(n, m, from, to, out, eigval);
    }
    if (n == 0) return 0;
    if (mode == 2) {
        if (m == 0 || n == 1) {
            for (uint32_t i = 0; i < n; i++) out[i] = 1.0;
            return 0;
        }
        int allzero = 1;
        if (w)
            for (uint64_t e = 0; e < m; e++) allzero &= w[e] == 0.0;
        if (w && allzero) {
            for (uint32_t i = 0; i < n; i++) out[i] = 1.0;
            return 0;
        }
        if (w) return weighted_core(n, m, from, to, w, 1, 0, out, eigval);
        /* unweighted: ascending out-neighbours, x' = x + sum, eps 1e-14 */
        uint64_t *rp;
        uint32_t *oth, *eid;
        edge_rows(n, m, from, to, &rp, &oth, &eid); /* out-edges by (source, target, id) */
        double *x = (double *)malloc(n * sizeof(double)), *xn = (double *)malloc(n * sizeof(double));
        for (uint32_t v = 0; v < n; v++) x[v] = 1.0;
        int it = 0;
        while (it < 5000) {
            it++;
            for (uint32_t v = 0; v < n; v++) {
                double s = x[v];
                for (uint64_t p = rp[v]; p < rp[v + 1]; p++) s += x[oth[p]];
                xn[v] = s;
            }
            rescale_max_abs(xn, n);
            double diff = 0.0;
            for (uint32_t v = 0; v < n; v++) diff += fabs(xn[v] - x[v]);
            double *t = x; x = xn; xn = t;
            if (diff < 1e-14) break;
        }
        double num = 0.0, den = 0.0;
        for (uint32_t v = 0; v < n; v++) {
            double s = 0.0;
            for (uint64_t p = rp[v]; p < rp[v + 1]; p++) s += x[oth[p]];
            num += x[v] * s;
            den += x[v] * x[v];
        }
        if (eigval) *eigval = den > 0.0 ? num / den : 0.0;
        for (uint32_t v = 0; v < n; v++) out[v] = x[v] < 0.0 ? 0.0 : x[v];
        free(rp); free(oth); free(eid); free(x); free(xn);
        return it;
    }
    /* Out / In */
    int allzero = 1;
    if (w)
        for (uint64_t e = 0; e < m; e++) allzero &= w[e] == 0.0;
    if (m == 0 || (w && allzero)) {
        for (uint32_t i = 0; i < n; i++) out[i] = 1.0;
        return 0;
    }
    const int neg = w ? any_negative_w(w, m) : 0;
    if (!neg && is_dag(n, m, from, to)) {
        double *st = (double *)calloc(n, sizeof(double));
        for (uint64_t e = 0; e < m; e++) st[mode == 0 ? from[e] : to[e]] += w ? w[e] : 1.0;
        for (uint32_t v = 0; v < n; v++) out[v] = st[v] == 0.0 ? 1.0 : 0.0;
        free(st);
        return 0;
    }
    /* walk[v]: (edge, neighbour) in edge order; Out: in-edges u->v, In: out-edges v->u */
    const uint32_t *key = mode == 0 ? to : from, *nbr = mode == 0 ? from : to;
    uint64_t *rp = (uint64_t *)calloc((size_t)n + 1, sizeof(uint64_t));
    uint32_t *wn = (uint32_t *)malloc(m * sizeof(uint32_t)), *we = (uint32_t *)malloc(m * sizeof(uint32_t));
    for (uint64_t e = 0; e < m; e++) rp[key[e] + 1]++;
    for (uint32_t v = 0; v < n; v++) rp[v + 1] += rp[v];
    uint64_t *cur = (uint64_t *)malloc(((size_t)n + 1) * sizeof(uint64_t));
    memcpy(cur, rp, ((size_t)n + 1) * sizeof(uint64_t));
    for (uint64_t e = 0; e < m; e++) {
        wn[cur[key[e]]] = nbr[e];
        we[cur[key[e]]++] = (uint32_t)e;
    }
    double *x = (double *)malloc(n * sizeof(double)), *xn = (double *)malloc(n * sizeof(double));
    double row_norm = 0.0;
    int any = 0;
    for (uint32_t v = 0; v < n; v++) {
        double s = 0.0, sa = 0.0;
        for (uint64_t p = rp[v]; p < rp[v + 1]; p++) {
            const double wv = w ? w[we[p]] : 1.0;
            s += wv;
            sa += fabs(wv);
        }
        if (s != 0.0) x[v] = fabs(s);
        else x[v] = (neg && rp[v + 1] > rp[v]) ? 1.0 : 0.0;
        any |= x[v] != 0.0;
        if (sa > row_norm) row_norm = sa;
    }
    if (!any)
        for (uint32_t v = 0; v < n; v++) x[v] = 1.0;
    rescale_max_abs(x, n);
    const double shift = (row_norm > 1.0 ? row_norm : 1.0) + 1.0;
    int it = 0;
    while (it < 5000) {
        it++;
        for (uint32_t v = 0; v < n; v++) {
            double s = shift * x[v];
            for (uint64_t p = rp[v]; p < rp[v + 1]; p++) s += (w ? w[we[p]] : 1.0) * x[wn[p]];
            xn[v] = s;
        }
        if (neg) {
            const double pv = signed_pivot(xn, n);
            if (pv != 0.0)
                for (uint32_t v = 0; v < n; v++) xn[v] /= pv;
        } else {
            rescale_max_abs(xn, n);
        }
        double diff = 0.0;
        for (uint32_t v = 0; v < n; v++) diff += fabs(xn[v] - x[v]);
        double *t = x; x = xn; xn = t;
        if (diff < 1e-12) break;
    }
    double num = 0.0, den = 0.0;
    for (uint32_t v = 0; v < n; v++) {
        double s = 0.0;
        for (uint64_t p = rp[v]; p < rp[v + 1]; p++) s += (w ? w[we[p]] : 1.0) * x[wn[p]];
        num += x[v] * s;
        den += x[v] * x[v];
    }
    double lam = den > 0.0 ? num / den : 0.0;
    if (!neg && lam <= 1e-12) {
        lam = 0.0;
        for (uint32_t v = 0; v < n; v++) out[v] = 0.0;
    } else {
        rescale_max_abs(x, n);
        for (uint32_t v = 0; v < n; v++) out[v] = (!neg && x[v] < 0.0) ? 0.0 : x[v];
    }
    if (eigval) *eigval = lam;
    free(rp); free(wn); free(we); free(cur); free(x); free(xn);
    return it;
}
