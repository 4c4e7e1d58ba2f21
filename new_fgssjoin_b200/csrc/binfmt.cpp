// binfmt.cpp -- the ppjoin .bin record file and its .loc side file.
//
// .bin: little-endian int32 records [id][size][token x size], ascending size
// in a well-formed file (src/fgssjoin/data.cu:53-89 reads it; the records are
// reversed into memory order at data.cu:97-113).  .loc: one int32 per token,
// in .bin order, giving the token's q-gram position in its line (the shipped
// fixture test/data/string/small.txt.3gram.bin.loc; the join never reads it).
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

#include "../../include/fgss.h"

extern "C" {

fgss_status fgss_load_bin(const char* path, fgss_sets* out) {
    if (!path || !out) return FGSS_ERR_INVALID;
    memset(out, 0, sizeof *out);
    FILE* f = fopen(path, "rb");
    if (!f) return FGSS_ERR_IO;
    std::vector<uint32_t> ids, lens, toks;
    uint32_t terms = 0;
    for (;;) {
        int32_t hdr[2];
        size_t r = fread(hdr, 4, 1, f);
        if (r != 1) break;  // end of file at a record boundary (data.cu:56-60)
        if (fread(hdr + 1, 4, 1, f) != 1 || hdr[1] < 0) {
            fclose(f);
            return FGSS_ERR_FORMAT;  // the reference prints "Reading error." and exits (data.cu:66-68)
        }
        size_t old = toks.size();
        toks.resize(old + (size_t)hdr[1]);
        if (hdr[1] && fread(toks.data() + old, 4, (size_t)hdr[1], f) != (size_t)hdr[1]) {
            fclose(f);
            return FGSS_ERR_FORMAT;
        }
        for (size_t i = old; i < toks.size(); i++)
            if (toks[i] + 1 > terms) terms = toks[i] + 1;  // num_terms = max token + 1 (data.cu:77-78)
        ids.push_back((uint32_t)hdr[0]);
        lens.push_back((uint32_t)hdr[1]);
    }
    fclose(f);
    const size_t n = ids.size(), T = toks.size();
    out->id = (uint32_t*)malloc((n + 1) * 4);
    out->len = (uint32_t*)malloc((n + 1) * 4);
    out->pos = (uint32_t*)malloc((n + 1) * 4);
    out->tokens = (uint32_t*)malloc((T + 1) * 4);
    if (!out->id || !out->len || !out->pos || !out->tokens) {
        fgss_sets_free(out);
        return FGSS_ERR_NOMEM;
    }
    // memory order = file order reversed
    std::vector<size_t> foff(n + 1, 0);
    for (size_t i = 0; i < n; i++) foff[i + 1] = foff[i] + lens[i];
    size_t o = 0;
    uint32_t mx = 0;
    for (size_t i = 0; i < n; i++) {
        size_t fi = n - 1 - i;
        out->id[i] = ids[fi];
        out->len[i] = lens[fi];
        out->pos[i] = (uint32_t)o;
        memcpy(out->tokens + o, toks.data() + foff[fi], (size_t)lens[fi] * 4);
        o += lens[fi];
        if (lens[fi] > mx) mx = lens[fi];
    }
    out->n_sets = n;
    out->n_tokens = T;
    out->n_terms = terms;
    out->max_len = mx;
    return FGSS_OK;
}

fgss_status fgss_write_bin(const char* path, const char* loc_path, const fgss_sets* s) {
    if (!path || !s) return FGSS_ERR_INVALID;
    FILE* f = fopen(path, "wb");
    if (!f) return FGSS_ERR_IO;
    FILE* g = nullptr;
    if (loc_path && s->loc) {
        g = fopen(loc_path, "wb");
        if (!g) {
            fclose(f);
            return FGSS_ERR_IO;
        }
    }
    bool ok = true;
    for (uint64_t k = 0; k < s->n_sets && ok; k++) {
        uint64_t i = s->n_sets - 1 - k;  // file order = memory order reversed
        int32_t hdr[2] = {(int32_t)s->id[i], (int32_t)s->len[i]};
        ok = fwrite(hdr, 4, 2, f) == 2;
        if (ok && s->len[i]) ok = fwrite(s->tokens + s->pos[i], 4, s->len[i], f) == s->len[i];
        if (ok && g && s->len[i]) ok = fwrite(s->loc + s->pos[i], 4, s->len[i], g) == s->len[i];
    }
    if (fclose(f) != 0) ok = false;
    if (g && fclose(g) != 0) ok = false;
    return ok ? FGSS_OK : FGSS_ERR_IO;
}

}  // extern "C"
