// edgelist.cuh — GPU reader for rust-igraph's plain edge-list format.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

namespace prg {
namespace el {

// Per-line codes (bit 4 marks an error in the second id).
enum : int {
    kSkip = 0,
    kEdge = 1,
    kHost = 2,          // non-ASCII bytes: resolved on the host
    kErrMissing = 3,    // "missing vertex id"
    kErrInvalid = 4,    // ParseIntError InvalidDigit
    kErrOverflow = 5,   // ParseIntError PosOverflow
    kErrEmpty = 6,      // ParseIntError Empty (not reachable through split_whitespace)
    kErrExtra = 7,      // "expected exactly two vertex ids"
    kErrUtf8 = 8,       // the line is not valid UTF-8 (an I/O error in the reference)
    kSecondToken = 16,
};

struct ParseResult {
    int status = 0;          // prg_status
    uint64_t err_line = 0;   // 1-based line of the first failing line (status != 0)
    std::string message;
    uint64_t lines = 0;
    uint64_t m = 0;          // edges, in file order
    uint32_t n = 0;          // max id + 1 (0 without edges)
    uint32_t *d_from = nullptr, *d_to = nullptr;  // device, m entries (owned by the result)
};

// d_text: the text in device memory; h_text: the same bytes in host memory,
// or null (line bytes the host needs are then copied back).
ParseResult parse(const uint8_t *d_text, const uint8_t *h_text, uint64_t len, cudaStream_t s);
void free_result(ParseResult &r, cudaStream_t s);

}  // namespace el
}  // namespace prg
