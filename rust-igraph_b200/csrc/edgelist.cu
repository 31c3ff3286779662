// edgelist.cu — rust-igraph's plain edge-list reader (read_edgelist,
// src/algorithms/io/edgelist.rs:25-72) on the GPU.
//
// Format: one edge per line, "u v" (u32 ids separated by whitespace); after
// trimming, blank lines and lines starting with '#' are skipped; anything
// else is an error reported with its 1-based line number, and the first
// failing line in file order wins.  The graph is undirected with
// n = max id + 1 (Graph::with_vertices + add_edges).
//
// Pipeline (the text is read from HBM a small number of times):
//   1. newline count per 512-byte warp chunk (16-byte loads, coalesced);
//   2. exclusive scan of the counts, then each newline writes the start of
//      the line after it (u64 offsets: texts may exceed 4 GiB);
//   3. one thread per line trims, tokenises and parses with Rust's rules
//      (ASCII whitespace, u32::from_str: optional '+', the first bad
//      character decides between "invalid digit" and "too large") and
//      writes a code plus (u, v);
//   4. lines that hold any byte >= 0x80 are rare; they are resolved on the
//      host with the full rules (UTF-8 validation, Unicode White_Space), as
//      is the message of the first failing line, which names its token;
//   5. the edge lines are compacted in order (scan) into from/to, and the
//      largest id gives n.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/prg_b200.h"
#include "edgelist.cuh"
#include "graph.cuh"
#include "prims.cuh"

namespace prg {
namespace el {

__host__ __device__ inline bool ascii_ws(uint8_t c) { return c == ' ' || (c >= 9 && c <= 13); }

// u32::from_str: an optional '+' (a lone sign is invalid), then digits only;
// per character the digit check comes before the overflow check.
__host__ __device__ inline int parse_u32(const uint8_t *s, uint64_t len, uint32_t *out) {
    uint64_t i = 0;
    if (len == 0) return kErrEmpty;
    if (s[0] == '+' || s[0] == '-') {
        if (len == 1) return kErrInvalid;
        if (s[0] == '+') i = 1;
    }
    uint64_t acc = 0;
    for (; i < len; i++) {
        const uint8_t c = s[i];
        if (c < '0' || c > '9') return kErrInvalid;
        acc = acc * 10u + (uint64_t)(c - '0');
        if (acc > 0xFFFFFFFFull) return kErrOverflow;
    }
    *out = (uint32_t)acc;
    return kEdge;
}

// One line of ASCII bytes (newline excluded).  Token errors carry the token
// index in bit 4 (0: first id, 1: second id).
__host__ __device__ inline int parse_line_ascii(const uint8_t *p, uint64_t len, uint32_t *u, uint32_t *v) {
    uint64_t b = 0, e = len;
    while (b < e && ascii_ws(p[b])) b++;
    while (e > b && ascii_ws(p[e - 1])) e--;
    if (b == e || p[b] == '#') return kSkip;
    const uint64_t t1 = b;
    while (b < e && !ascii_ws(p[b])) b++;
    int r = parse_u32(p + t1, b - t1, u);
    if (r != kEdge) return r;
    while (b < e && ascii_ws(p[b])) b++;
    if (b == e) return kErrMissing;
    const uint64_t t2 = b;
    while (b < e && !ascii_ws(p[b])) b++;
    r = parse_u32(p + t2, b - t2, v);
    if (r != kEdge) return r | kSecondToken;
    while (b < e && ascii_ws(p[b])) b++;
    if (b != e) return kErrExtra;
    return kEdge;
}

constexpr int kChunkBytes = 512;  // one warp: 32 lanes x 16 bytes

__device__ inline uint32_t count_nl16(uint4 q) {
    uint32_t c = 0;
    const uint32_t w[4] = {q.x, q.y, q.z, q.w};
#pragma unroll
    for (int k = 0; k < 4; k++) {
        // exact per-byte compare (0xFF per byte equal to '\n'); the borrow
        // trick of zero-byte tests misfires on a 0x0B byte after a newline
        c += __popc(__vcmpeq4(w[k], 0x0A0A0A0Au)) >> 3;
    }
    return c;
}

// The 16 bytes of lane `lane` in chunk `chunk` (bytes past len read as 0).
__device__ inline uint4 load16(const uint8_t *text, uint64_t len, uint64_t chunk, int lane, bool aligned) {
    const uint64_t off = chunk * kChunkBytes + (uint64_t)lane * 16u;
    if (aligned && off + 16 <= len) return __ldg(reinterpret_cast<const uint4 *>(text + off));
    uint8_t b[16];
#pragma unroll
    for (int i = 0; i < 16; i++) b[i] = off + i < len ? text[off + i] : 0;
    uint4 q;
    std::memcpy(&q, b, 16);
    return q;
}

__global__ void nl_count_kernel(const uint8_t *text, uint64_t len, uint64_t nchunks, bool aligned, uint32_t *counts) {
    const int lane = threadIdx.x & 31;
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t c = warp; c < nchunks; c += nw) {
        uint32_t k = count_nl16(load16(text, len, c, lane, aligned));
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) k += __shfl_xor_sync(0xffffffffu, k, o);
        if (lane == 0) counts[c] = k;
    }
}

// starts[i + 1] = position after the i-th newline
__global__ void nl_write_kernel(const uint8_t *text, uint64_t len, uint64_t nchunks, bool aligned,
                                const uint32_t *offs, uint64_t *starts) {
    const int lane = threadIdx.x & 31;
    const uint64_t warp = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t c = warp; c < nchunks; c += nw) {
        const uint4 q = load16(text, len, c, lane, aligned);
        const uint32_t k = count_nl16(q);
        const uint32_t incl = warp_incl_scan(k);
        uint64_t idx = (uint64_t)offs[c] + (incl - k);
        uint8_t b[16];
        std::memcpy(b, &q, 16);
        const uint64_t base = c * kChunkBytes + (uint64_t)lane * 16u;
#pragma unroll
        for (int i = 0; i < 16; i++)
            if (b[i] == '\n' && base + i < len) starts[1 + idx++] = base + i + 1;
    }
}

__global__ void parse_lines_kernel(const uint8_t *text, uint64_t len, const uint64_t *starts, uint64_t nl,
                                   uint64_t nlines, uint8_t *codes, uint32_t *U, uint32_t *V, uint64_t *host_idx,
                                   unsigned long long *host_cnt, unsigned long long *first_err) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nlines;
         k += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = starts[k];
        const uint64_t e = k < nl ? starts[k + 1] - 1 : len;  // exclude the newline
        const uint8_t *p = text + b;
        bool ascii = true;
        for (uint64_t i = 0; i < e - b; i++)
            if (p[i] >= 0x80) {
                ascii = false;
                break;
            }
        uint32_t u = 0, v = 0;
        int code;
        if (!ascii) {
            code = kHost;
            host_idx[atomicAdd(host_cnt, 1ull)] = k;
        } else {
            code = parse_line_ascii(p, e - b, &u, &v);
            if (code >= kErrMissing) atomicMin(first_err, (unsigned long long)k);
        }
        codes[k] = (uint8_t)code;
        U[k] = u;
        V[k] = v;
    }
}

__global__ void line_bounds_kernel(const uint64_t *starts, uint64_t nl, uint64_t len, const uint64_t *idx,
                                   uint64_t cnt, uint64_t *b, uint64_t *e) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k = idx[i];
        b[i] = starts[k];
        e[i] = k < nl ? starts[k + 1] - 1 : len;
    }
}

struct HostLine {
    uint64_t k;
    uint32_t code, u, v;
};

__global__ void apply_host_lines_kernel(const HostLine *hl, uint64_t cnt, uint8_t *codes, uint32_t *U, uint32_t *V) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += (uint64_t)gridDim.x * blockDim.x) {
        codes[hl[i].k] = (uint8_t)hl[i].code;
        U[hl[i].k] = hl[i].u;
        V[hl[i].k] = hl[i].v;
    }
}

__global__ void edge_flags_kernel(const uint8_t *codes, uint64_t nlines, uint32_t *flags) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nlines;
         k += (uint64_t)gridDim.x * blockDim.x)
        flags[k] = codes[k] == kEdge ? 1u : 0u;
}

__global__ void scatter_edges_kernel(const uint8_t *codes, const uint32_t *U, const uint32_t *V,
                                     const uint32_t *offs, uint64_t nlines, uint32_t *from, uint32_t *to,
                                     uint32_t *max_id) {
    uint32_t mx = 0;
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nlines;
         k += (uint64_t)gridDim.x * blockDim.x) {
        if (codes[k] == kEdge) {
            const uint32_t o = offs[k];
            from[o] = U[k];
            to[o] = V[k];
            mx = max(mx, max(U[k], V[k]));
        }
    }
    for (int o = 16; o > 0; o >>= 1) mx = max(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if ((threadIdx.x & 31) == 0) atomicMax(max_id, mx);
}

// ---------------------------------------------------------------- host rules

// Rust's `lines()` yields valid UTF-8 only; `trim` / `split_whitespace`
// use the Unicode White_Space property (char::is_whitespace).
static bool unicode_ws(uint32_t c) {
    return (c >= 0x09 && c <= 0x0D) || c == 0x20 || c == 0x85 || c == 0xA0 || c == 0x1680 ||
           (c >= 0x2000 && c <= 0x200A) || c == 0x2028 || c == 0x2029 || c == 0x202F || c == 0x205F ||
           c == 0x3000;
}

// Decodes UTF-8 with the validity rules of str::from_utf8 (no overlong
// forms, no surrogates, nothing above U+10FFFF).  Returns false on error.
static bool decode_utf8(const uint8_t *p, size_t len, std::vector<uint32_t> &cps, std::vector<size_t> &pos) {
    size_t i = 0;
    while (i < len) {
        const uint8_t c = p[i];
        uint32_t cp;
        size_t n;
        if (c < 0x80) {
            cp = c;
            n = 1;
        } else if (c >= 0xC2 && c <= 0xDF) {
            cp = c & 0x1F;
            n = 2;
        } else if (c >= 0xE0 && c <= 0xEF) {
            cp = c & 0x0F;
            n = 3;
        } else if (c >= 0xF0 && c <= 0xF4) {
            cp = c & 0x07;
            n = 4;
        } else {
            return false;
        }
        if (i + n > len) return false;
        for (size_t k = 1; k < n; k++) {
            const uint8_t t = p[i + k];
            if ((t & 0xC0) != 0x80) return false;
            cp = (cp << 6) | (t & 0x3F);
        }
        if ((n == 3 && (cp < 0x800 || (cp >= 0xD800 && cp <= 0xDFFF))) || (n == 4 && (cp < 0x10000 || cp > 0x10FFFF)))
            return false;
        cps.push_back(cp);
        pos.push_back(i);
        i += n;
    }
    pos.push_back(len);
    return true;
}

// Full rules for one line (bytes without the newline).  Returns the code;
// for token errors *tok receives the offending token's bytes.
int parse_line_host(const uint8_t *p, size_t len, uint32_t *u, uint32_t *v, std::string *tok) {
    std::vector<uint32_t> cps;
    std::vector<size_t> pos;
    if (!decode_utf8(p, len, cps, pos)) return kErrUtf8;
    size_t b = 0, e = cps.size();
    while (b < e && unicode_ws(cps[b])) b++;
    while (e > b && unicode_ws(cps[e - 1])) e--;
    if (b == e || cps[b] == '#') return kSkip;
    std::vector<std::pair<size_t, size_t>> toks;  // byte ranges
    size_t i = b;
    while (i < e) {
        while (i < e && unicode_ws(cps[i])) i++;
        if (i >= e) break;
        const size_t s = i;
        while (i < e && !unicode_ws(cps[i])) i++;
        toks.push_back({pos[s], pos[i]});
    }
    auto parse_tok = [&](size_t t, uint32_t *out) {
        const int r = parse_u32(p + toks[t].first, toks[t].second - toks[t].first, out);
        if (r != kEdge && tok) tok->assign((const char *)p + toks[t].first, toks[t].second - toks[t].first);
        return r;
    };
    int r = parse_tok(0, u);
    if (r != kEdge) return r;
    if (toks.size() < 2) return kErrMissing;
    r = parse_tok(1, v);
    if (r != kEdge) return r | kSecondToken;
    if (toks.size() > 2) return kErrExtra;
    return kEdge;
}

std::string error_message(int code, const std::string &tok) {
    switch (code & ~kSecondToken) {
        case kErrMissing: return "missing vertex id";
        case kErrExtra: return "expected exactly two vertex ids";
        case kErrInvalid: return "invalid vertex id `" + tok + "`: invalid digit found in string";
        case kErrOverflow: return "invalid vertex id `" + tok + "`: number too large to fit in target type";
        case kErrEmpty: return "invalid vertex id `" + tok + "`: cannot parse integer from empty string";
        default: return "stream did not contain valid UTF-8";
    }
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

static unsigned grid_for(uint64_t items, uint64_t per_block) {
    uint64_t g = (items + per_block - 1) / per_block;
    return (unsigned)std::min<uint64_t>(std::max<uint64_t>(g, 1), 148ull * 64ull);
}

ParseResult parse(const uint8_t *d_text, const uint8_t *h_text, uint64_t len, cudaStream_t s) {
    ParseResult r;
    if (len == 0) return r;
    const uint64_t nchunks = (len + kChunkBytes - 1) / kChunkBytes;
    const bool aligned = ((uintptr_t)d_text & 15u) == 0;
    uint32_t *counts = alloc<uint32_t>(nchunks + 1, s);
    uint32_t *offs = alloc<uint32_t>(nchunks + 1, s);
    nl_count_kernel<<<grid_for(nchunks * 32, 256), 256, 0, s>>>(d_text, len, nchunks, aligned, counts);
    PRG_CUDA(cudaGetLastError());
    exclusive_scan_u32(counts, offs, nchunks, s);
    uint32_t nl32 = 0;
    PRG_CUDA(cudaMemcpyAsync(&nl32, offs + nchunks, 4, cudaMemcpyDeviceToHost, s));
    uint8_t last = 0;
    if (h_text) last = h_text[len - 1];
    else PRG_CUDA(cudaMemcpyAsync(&last, d_text + len - 1, 1, cudaMemcpyDeviceToHost, s));
    PRG_CUDA(cudaStreamSynchronize(s));
    const uint64_t nl = nl32;
    const uint64_t nlines = nl + (last != '\n' ? 1u : 0u);
    r.lines = nlines;
    if (nlines >= 0xFFFFFFFFull) {
        release(counts, s);
        release(offs, s);
        r.status = PRG_ERR_INTERNAL;
        r.message = "edge list has too many lines";
        return r;
    }
    uint64_t *starts = alloc<uint64_t>(nl + 2, s);
    PRG_CUDA(cudaMemsetAsync(starts, 0, 8, s));
    nl_write_kernel<<<grid_for(nchunks * 32, 256), 256, 0, s>>>(d_text, len, nchunks, aligned, offs, starts);
    PRG_CUDA(cudaGetLastError());
    release(counts, s);
    release(offs, s);

    uint8_t *codes = alloc<uint8_t>(nlines, s);
    uint32_t *U = alloc<uint32_t>(nlines, s), *V = alloc<uint32_t>(nlines, s);
    uint64_t *host_idx = alloc<uint64_t>(nlines, s);
    unsigned long long *cnt = alloc<unsigned long long>(2, s);  // [0] host lines, [1] first error
    const unsigned long long init[2] = {0ull, ~0ull};
    PRG_CUDA(cudaMemcpyAsync(cnt, init, sizeof(init), cudaMemcpyHostToDevice, s));
    parse_lines_kernel<<<grid_for(nlines, 256), 256, 0, s>>>(d_text, len, starts, nl, nlines, codes, U, V, host_idx,
                                                             cnt, cnt + 1);
    PRG_CUDA(cudaGetLastError());
    unsigned long long hc[2];
    PRG_CUDA(cudaMemcpyAsync(hc, cnt, sizeof(hc), cudaMemcpyDeviceToHost, s));
    PRG_CUDA(cudaStreamSynchronize(s));

    auto line_bytes = [&](uint64_t k, std::vector<uint8_t> &buf) {
        uint64_t se[2];
        PRG_CUDA(cudaMemcpyAsync(se, starts + k, k < nl ? 16 : 8, cudaMemcpyDeviceToHost, s));
        PRG_CUDA(cudaStreamSynchronize(s));
        const uint64_t b = se[0], e = k < nl ? se[1] - 1 : len;
        buf.resize(e - b);
        if (h_text) std::memcpy(buf.data(), h_text + b, e - b);
        else if (e > b) {
            PRG_CUDA(cudaMemcpyAsync(buf.data(), d_text + b, e - b, cudaMemcpyDeviceToHost, s));
            PRG_CUDA(cudaStreamSynchronize(s));
        }
    };

    // lines with non-ASCII bytes: full rules on the host, in file order up to
    // the first failing line; results go back in one scatter
    uint64_t first_err = hc[1];
    if (hc[0] > 0) {
        const uint64_t cnt = hc[0];
        std::vector<uint64_t> idx(cnt), hb(cnt), he(cnt);
        uint64_t *db = alloc<uint64_t>(cnt, s), *de = alloc<uint64_t>(cnt, s);
        line_bounds_kernel<<<grid_for(cnt, 256), 256, 0, s>>>(starts, nl, len, host_idx, cnt, db, de);
        PRG_CUDA(cudaGetLastError());
        PRG_CUDA(cudaMemcpyAsync(idx.data(), host_idx, cnt * 8, cudaMemcpyDeviceToHost, s));
        PRG_CUDA(cudaMemcpyAsync(hb.data(), db, cnt * 8, cudaMemcpyDeviceToHost, s));
        PRG_CUDA(cudaMemcpyAsync(he.data(), de, cnt * 8, cudaMemcpyDeviceToHost, s));
        PRG_CUDA(cudaStreamSynchronize(s));
        release(db, s);
        release(de, s);
        std::vector<uint64_t> order(cnt);
        for (uint64_t i = 0; i < cnt; i++) order[i] = i;
        std::sort(order.begin(), order.end(), [&](uint64_t a, uint64_t b) { return idx[a] < idx[b]; });
        std::vector<HostLine> out;
        std::vector<uint8_t> buf;
        for (uint64_t i : order) {
            const uint64_t k = idx[i];
            if (k > first_err) break;  // an earlier failing line decides already
            const uint8_t *p;
            if (h_text) {
                p = h_text + hb[i];
            } else {
                buf.resize(he[i] - hb[i]);
                if (!buf.empty())
                    PRG_CUDA(cudaMemcpy(buf.data(), d_text + hb[i], buf.size(), cudaMemcpyDeviceToHost));
                p = buf.data();
            }
            HostLine h{k, 0u, 0u, 0u};
            h.code = (uint32_t)parse_line_host(p, he[i] - hb[i], &h.u, &h.v, nullptr);
            out.push_back(h);
            if (h.code >= (uint32_t)kErrMissing) first_err = std::min<uint64_t>(first_err, k);
        }
        if (!out.empty()) {
            HostLine *dh = alloc<HostLine>(out.size(), s);
            PRG_CUDA(cudaMemcpyAsync(dh, out.data(), out.size() * sizeof(HostLine), cudaMemcpyHostToDevice, s));
            apply_host_lines_kernel<<<grid_for(out.size(), 256), 256, 0, s>>>(dh, out.size(), codes, U, V);
            PRG_CUDA(cudaGetLastError());
            PRG_CUDA(cudaStreamSynchronize(s));
            release(dh, s);
        }
    }
    release(host_idx, s);
    release(cnt, s);

    if (first_err != ~0ull) {
        std::vector<uint8_t> buf;
        line_bytes(first_err, buf);
        uint32_t u, v;
        std::string tok;
        const int code = parse_line_host(buf.data(), buf.size(), &u, &v, &tok);
        r.status = code == kErrUtf8 ? PRG_ERR_IO : PRG_ERR_PARSE;
        r.err_line = first_err + 1;
        r.message = error_message(code, tok);
        release(starts, s);
        release(codes, s);
        release(U, s);
        release(V, s);
        PRG_CUDA(cudaStreamSynchronize(s));
        return r;
    }
    release(starts, s);

    // compaction in line order
    uint32_t *flags = alloc<uint32_t>(nlines + 1, s), *eoff = alloc<uint32_t>(nlines + 1, s);
    edge_flags_kernel<<<grid_for(nlines, 256), 256, 0, s>>>(codes, nlines, flags);
    PRG_CUDA(cudaGetLastError());
    exclusive_scan_u32(flags, eoff, nlines, s);
    uint32_t m32 = 0;
    PRG_CUDA(cudaMemcpyAsync(&m32, eoff + nlines, 4, cudaMemcpyDeviceToHost, s));
    PRG_CUDA(cudaStreamSynchronize(s));
    r.m = m32;
    r.d_from = alloc<uint32_t>(r.m, s);
    r.d_to = alloc<uint32_t>(r.m, s);
    uint32_t *mx = alloc<uint32_t>(1, s);
    PRG_CUDA(cudaMemsetAsync(mx, 0, 4, s));
    scatter_edges_kernel<<<grid_for(nlines, 256), 256, 0, s>>>(codes, U, V, eoff, nlines, r.d_from, r.d_to, mx);
    PRG_CUDA(cudaGetLastError());
    uint32_t hmx = 0;
    PRG_CUDA(cudaMemcpyAsync(&hmx, mx, 4, cudaMemcpyDeviceToHost, s));
    PRG_CUDA(cudaStreamSynchronize(s));
    release(mx, s);
    release(flags, s);
    release(eoff, s);
    release(codes, s);
    release(U, s);
    release(V, s);
    if (r.m > 0) {
        if (hmx == 0xFFFFFFFFu) {
            r.status = PRG_ERR_INTERNAL;
            r.message = "vertex id u32::MAX cannot be sized into n";  // edgelist.rs:50-55
            return r;
        }
        r.n = hmx + 1u;
    }
    return r;
}

void free_result(ParseResult &r, cudaStream_t s) {
    release(r.d_from, s);
    release(r.d_to, s);
}

}  // namespace el
}  // namespace prg
