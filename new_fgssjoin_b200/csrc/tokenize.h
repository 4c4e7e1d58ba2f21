// tokenize.h -- GPU tokenizer (tokenize.cu).
#pragma once

#include "ctx.h"

namespace fgss {

struct TokParams {
    int q;
    int mode;      // 0 q-grams, 1 canonical k-mers
    int pad;
    int pad_char;
    int suffix;
    int lower;
};

// Text -> sets in MEMORY order (host arrays malloc'd into *out).
void tokenize_device(Ctx& c, const char* text, uint64_t n_bytes, const TokParams& p, fgss_sets* out);

}  // namespace fgss
