// ref_join.cu -- test infrastructure (GPU): the reference's own join kernels,
// compiled unchanged from its sources by oracle/ref_build.sh, driven by this
// harness instead of the reference's process_blocks.
//
//   ref_join <file.bin> <threshold> <out>
//
// Path: ppjoin_format (src/fgssjoin/data.cu:31-126) -> prepare_data
// (data.cu:133-199) -> inverted_index (src/fgssjoin/index.cu:169-211) ->
// filtering_block (src/fgssjoin/filtering.cu:8-69) -> checking_block
// (src/fgssjoin/checking.cu:8-86) with ONE tile: block_size = N, both offsets
// 0, as process_blocks runs it when N records fit its memory-sized tile
// (src/fgssjoin/block.cu:61-213).  Two departures from process_blocks, both
// on the host:
//   * block_size is N, not get_block_size's free-memory formula
//     (block.cu:14-54), which creates a second driver context with cuCtxCreate
//     after the runtime has allocated in the primary one;
//   * each result's score is read as partial_scores[bucket] (the checking
//     kernel writes the verified score there, checking.cu:158-174), because
//     the two independent compactions chk_compact_1/2 (checking.cu:556-595)
//     do not keep buckets and scores paired; the paired count of the
//     reference's own host loop (block.cu:184-197 over its two arrays) is
//     reported beside it.
// Refused (exit 2, nothing run on the GPU): N > 46,340 (block_size^2 must fit
// the int of filter_k, compaction.cu:8) and empty records (jac_mid_prefix(0)
// = 1 would mark a token past the last record, data.cu:241-257).
// Output <out>: little-endian uint64 n_pairs, candidates, intersections,
// results_paired_as_the_reference_prints, then double ms (prepare_data to
// the end of the result loop, the reference's "Total Running Time" region
// without stdout), then n_pairs x (uint32 q, uint32 s, uint32 overlap) in
// memory order, sorted by (q, s).
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <sys/time.h>

#include <algorithm>
#include <vector>

#include "checking.cuh"
#include "data.cuh"
#include "filtering.cuh"
#include "index.cuh"
#include "similarity.cuh"

static double now_ms() {
    struct timeval tv;
    gettimeofday(&tv, nullptr);
    return tv.tv_sec * 1e3 + tv.tv_usec / 1e3;
}

int main(int argc, char** argv) {
    if (argc != 4) {
        fprintf(stderr, "usage: %s <file.bin> <threshold> <out>\n", argv[0]);
        return 2;
    }
    const float t = (float)atof(argv[2]);  // fgssjoin_cli.cu:31
    sets_t* sets = ppjoin_format(argv[1], 0);
    const uint64_t N = sets->num_sets;
    if (N == 0 || N > 46340) {
        fprintf(stderr, "refused: %llu records (the one-tile harness takes 1..46340)\n", (unsigned long long)N);
        return 2;
    }
    for (uint64_t i = 0; i < N; i++)
        if (sets->len[i] == 0) {
            fprintf(stderr, "refused: an empty record\n");
            return 2;
        }
    const double t0 = now_ms();
    prepare_data(sets, t, 0);
    Index index = inverted_index(sets, t, 0);
    const unsigned int B = (unsigned int)N;
    const unsigned int candsize = B * B;
    int* d_compidx;
    short* d_partial;
    unsigned int* d_comp_buckets;
    gpu(cudaMalloc(&d_compidx, sizeof(int)));
    gpu(cudaMalloc(&d_partial, (size_t)candsize * sizeof(short)));
    gpu(cudaMalloc(&d_comp_buckets, (size_t)candsize * sizeof(unsigned int)));
    uint64_t n_cand = 0, n_inter = 0, n_paired = 0;
    std::vector<uint32_t> out;
    // the skip test of block.cu:121-130 for the one tile
    const int q_size = (int)sets->len[N - 1];
    const int s_maxsize = floor(jac_max_size(sets->len[0], t));
    if (!(q_size > s_maxsize)) {
        unsigned int *d_candidates, csize;
        filtering_block(sets, index, d_partial, d_comp_buckets, d_compidx, candsize, t, 0, 0, B, B, &d_candidates,
                        &csize, 0);
        unsigned int *similar_pairs, size;
        unsigned short* scores;
        checking_block(d_partial, d_candidates, sets, t, csize, 0, 0, B, &similar_pairs, &scores, &size, d_compidx,
                       0);
        n_cand = csize;
        n_inter = size;
        std::vector<short> partial(candsize);
        gpu(cudaMemcpy(partial.data(), d_partial, (size_t)candsize * sizeof(short), cudaMemcpyDeviceToHost));
        for (unsigned k = 0; k < size; k++) {
            const unsigned int bucket = similar_pairs[k];
            const unsigned int q = bucket / B, s = bucket % B;
            // as the reference's host loop pairs them (block.cu:184-197)
            if (scores[k] > 0 && jac_similarity(sets->len[q], sets->len[s], scores[k]) >= t) n_paired++;
            const unsigned short score = (unsigned short)partial[bucket];
            if (score > 0 && jac_similarity(sets->len[q], sets->len[s], score) >= t) {
                out.push_back(q);
                out.push_back(s);
                out.push_back(score);
            }
        }
    }
    const double ms = now_ms() - t0;
    // sort (q, s) triples
    const size_t np = out.size() / 3;
    std::vector<size_t> order(np);
    for (size_t i = 0; i < np; i++) order[i] = i;
    std::sort(order.begin(), order.end(), [&](size_t x, size_t y) {
        return out[3 * x] != out[3 * y] ? out[3 * x] < out[3 * y] : out[3 * x + 1] < out[3 * y + 1];
    });
    FILE* f = fopen(argv[3], "wb");
    if (!f) return 1;
    const uint64_t head[4] = {(uint64_t)np, n_cand, n_inter, n_paired};
    fwrite(head, 8, 4, f);
    fwrite(&ms, 8, 1, f);
    for (size_t i : order) fwrite(&out[3 * i], 4, 3, f);
    fclose(f);
    fprintf(stderr, "# Candidates: %llu\n# Intersections: %llu\n# Results: %llu\nms: %.3f\n",
            (unsigned long long)n_cand, (unsigned long long)n_inter, (unsigned long long)np, ms);
    return 0;
}
