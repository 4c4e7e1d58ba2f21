// ref_load.cu -- test infrastructure (CPU only): runs the reference's own
// .bin loader, ppjoin_format (src/fgssjoin/data.cu:31-126 of
// RafaelQuirino/new_fgssjoin, compiled unchanged from its sources by
// oracle/ref_build.sh), and writes what it built in memory order:
//   ref_load <file.bin>  -> stdout, little-endian uint32:
//     n_sets, n_tokens, n_terms, id[n_sets], pos[n_sets], len[n_sets], tokens[n_tokens]
// Only host code runs: the loader reads the file with fread and builds host
// arrays; no CUDA call is made.
#include <stdint.h>
#include <stdio.h>

#include "data.cuh"

int main(int argc, char** argv) {
    if (argc != 2) {
        fprintf(stderr, "usage: %s <file.bin>\n", argv[0]);
        return 2;
    }
    sets_t* s = ppjoin_format(argv[1], 0);
    const uint32_t head[3] = {(uint32_t)s->num_sets, (uint32_t)s->num_tokens, (uint32_t)s->num_terms};
    fwrite(head, 4, 3, stdout);
    fwrite(s->id, 4, s->num_sets, stdout);
    fwrite(s->pos, 4, s->num_sets, stdout);
    fwrite(s->len, 4, s->num_sets, stdout);
    fwrite(s->tokens, 4, s->num_tokens, stdout);
    return 0;
}
