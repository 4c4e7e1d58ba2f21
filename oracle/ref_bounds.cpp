// ref_bounds.cpp -- test infrastructure (CPU only): tabulates the reference's
// own float32 bound functions, include/fgssjoin/similarity.cuh of
// RafaelQuirino/new_fgssjoin compiled unchanged on the host (its __host__ /
// __device__ qualifiers defined away), the way its kernels use them:
//   filtering.cu:89-92     jac_max_prefix, floor(jac_min_size), floor(jac_max_size)
//   data.cu:241-257        jac_mid_prefix (index prefix)
//   filtering.cu:130-132   positional test (score + 1 + min_rem) < jac_min_overlap
//   checking.cu:110        minoverlap = floor(jac_min_overlap)
//   block.cu:188-193       score > 0 && jac_similarity(len_q, len_s, score) >= t
// Built by oracle/ref_build.sh into oracle/_ref/ref_bounds; tests compare its
// tables with the library's fgss_bounds_table / fgss_overlap_table.
//
//   ref_bounds <threshold> <max_len>   -> stdout, little-endian uint32 arrays:
//     probe[n], index[n], min_size[n], max_size[n]        n = 0 .. max_len
//     cand_min[S], inter_min[S], need[S]                  S = 0 .. 2 max_len
// cand_min[S]: smallest integer k with !(k < jac_min_overlap(S, 0)) compared as
// the filter compares it (an unsigned int against a float); need[S]: smallest
// overlap o >= 1 that survives checking.cu's floor(min overlap) test and the
// final float test.
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#include <vector>

#define __host__
#define __device__
#include "similarity.cuh"

int main(int argc, char** argv) {
    if (argc != 3) {
        fprintf(stderr, "usage: %s <threshold> <max_len>\n", argv[0]);
        return 2;
    }
    const float t = (float)atof(argv[1]);  // as fgssjoin_cli.cu:31 parses it
    const unsigned L = (unsigned)atoi(argv[2]);
    std::vector<uint32_t> out;
    out.reserve(4 * (L + 1) + 3 * (2 * L + 1));
    for (unsigned n = 0; n <= L; n++) out.push_back(jac_max_prefix(n, t));
    for (unsigned n = 0; n <= L; n++) out.push_back(jac_mid_prefix(n, t));
    for (unsigned n = 0; n <= L; n++) out.push_back((unsigned int)floor(jac_min_size(n, t)));
    for (unsigned n = 0; n <= L; n++) {
        const float mx = floor(jac_max_size(n, t));
        out.push_back(mx > 4294967040.0f ? 0xffffffffu : (unsigned int)mx);
    }
    std::vector<uint32_t> cand(2 * L + 1), inter(2 * L + 1), need(2 * L + 1);
    for (unsigned S = 0; S <= 2 * L; S++) {
        const float mo = jac_min_overlap(S, 0, t);
        // below floor(mo) - 1 every k is rejected: start there, then the
        // filter's own comparison (an unsigned int against a float)
        unsigned int k = mo > 2.0f ? (unsigned int)mo - 2u : 0u;
        while (k < mo) k++;
        cand[S] = k;
        const int minoverlap = floor(jac_min_overlap(S, 0, t));
        inter[S] = (uint32_t)minoverlap;
        unsigned o = minoverlap > 1 ? (unsigned)minoverlap : 1u;  // smaller o fail checking.cu:167
        for (;; o++) {
            if (o > S) break;  // no overlap qualifies (never reached for S >= 2)
            const unsigned short score = (unsigned short)o;
            if ((int)score < minoverlap) continue;
            if (jac_similarity(S, 0u, score) >= t) break;
        }
        need[S] = o;
    }
    out.insert(out.end(), cand.begin(), cand.end());
    out.insert(out.end(), inter.begin(), inter.end());
    out.insert(out.end(), need.begin(), need.end());
    fwrite(out.data(), 4, out.size(), stdout);
    return 0;
}
