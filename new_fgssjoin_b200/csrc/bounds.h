// bounds.h -- per-length bound tables of one threshold, computed on the host.
//
// The reference evaluates its Jaccard bounds per thread per list entry in
// float32 (include/fgssjoin/similarity.cuh:9-82).  The float32 results differ
// from the exact rational bounds for some lengths (at t = 0.6 and t = 0.8 the
// prefixes and size bounds of several hundred lengths are one shorter), so a
// bit-identical pair set needs the same float32 values.  They depend only on
// the length (or on the sum of two lengths), so they are tabulated once per
// threshold here and the kernels read integers.
//
// Tables, for record length n in [0, kMaxLen] and length sum S in [0, 2 kMaxLen]:
//   probe[n]     jac_max_prefix(n)          similarity.cuh:43-47   (0 for n = 0)
//   index[n]     jac_mid_prefix(n)          similarity.cuh:54-58   (0 for n = 0)
//   minsz[n]     floor(jac_min_size(n))     filtering.cu:91,111
//   maxsz[n]     floor(jac_max_size(n))     filtering.cu:92,112
//   lmin[n]      smallest m with m >= minsz[n] and maxsz[m] >= n: for sets of
//                non-increasing size, the sources of a query of size n that
//                pass the size filter (filtering.cu:114-117) are exactly those
//                of size >= lmin[n]
//   cand_min[S]  smallest integer k with !(float(k) < jac_min_overlap): the
//                positional test of filtering.cu:132
//   inter_min[S] floor(jac_min_overlap)     checking.cu:110,167
//   need[S]      smallest overlap o >= max(1, inter_min[S]) with
//                float(o) / float(S - o) >= t (block.cu:190-192)
#pragma once

#include <stdint.h>

#include <vector>

namespace fgss {

constexpr uint32_t kMaxLen = 65535;  // set sizes are 16-bit (scores are unsigned short in checking.cu:117)

struct BoundTables {
    float t = 0.f;
    int mode = 0;
    std::vector<uint16_t> probe, index;
    std::vector<uint32_t> minsz, maxsz, lmin;
    std::vector<uint32_t> cand_min, inter_min, need;
};

// mode 0: reference float32 expressions; mode 1: exact rational bounds of the
// shortest decimal that rounds to t.
void compute_bounds(float t, int mode, BoundTables& b);

// The shortest decimal string that parses back to t (e.g. 0.7f -> "0.7").
void shortest_decimal(float t, int64_t* num, int64_t* den);

}  // namespace fgss
