/*
 * fgss_oracle.c -- CPU oracle for the set-similarity self-join hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker that the CUDA product
 * path is compared against; the product (libfgss.so) never links, loads or
 * calls it.  Only the tests, the smoke check and the bench's CPU-baseline leg
 * use it.
 *
 * It restates, in plain C, the behaviour of the reference project
 * (RafaelQuirino/new_fgssjoin) for the path it accelerates:
 *
 *   - bounds        include/fgssjoin/similarity.cuh:9-82 (float32 expressions)
 *   - tokenizer     src/preprocess/string/qgram.cpp:20-49 (q-grams with an
 *                   occurrence suffix), data.cpp:36-40 (ASCII lower-case),
 *                   io.cpp:8-26 (non-empty lines), preprocess_cli.cpp:266-340
 *                   (ids by ascending document frequency); the tie-break by
 *                   first occurrence, the per-record id sort and the ascending
 *                   size order of records follow the shipped fixture
 *                   test/data/string/small.txt.3gram.bin(.loc).
 *   - record order  src/fgssjoin/data.cu:97-113 (file order reversed in memory)
 *   - join          src/fgssjoin/block.cu:61-213 (block tiling and skip test),
 *                   src/fgssjoin/filtering.cu:76-141 (prefix, size and
 *                   positional filter), src/fgssjoin/checking.cu:93-175
 *                   (verification with resume and early exit),
 *                   src/fgssjoin/block.cu:184-197 (final float test).
 *
 * The two compactions of checking.cu:556-595 may pair a bucket with another
 * candidate's score; the oracle keeps every (pair, score) together, which is
 * the behaviour the reference intends.
 *
 * Parity pins: the tokenizer reproduces small.txt.3gram.bin and .bin.loc byte
 * for byte, and the join reproduces the golden pairs of that fixture; the join
 * itself has no reference-side golden output beyond that fixture.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_OK 0
#define ORC_ERR_ARG 1
#define ORC_ERR_NOMEM 3

/* ------------------------------------------------------------------------ */
/* Bounds: similarity.cuh:9-58, evaluated in float32 exactly as written.     */
/* ------------------------------------------------------------------------ */

static float jac_min_size_f(unsigned n, float t) { return (float)n * t; }
static float jac_max_size_f(unsigned n, float t) { return (float)n / t; }
static float jac_min_overlap_f(unsigned a, unsigned b, float t)
{
    return (float)(t / (1 + t)) * ((float)(a + b));
}
/* unsigned - float + int is evaluated in float, then truncated on return */
static unsigned jac_max_prefix_f(unsigned n, float t) { return (unsigned)(n - ceilf(jac_min_size_f(n, t)) + 1); }
static unsigned jac_mid_prefix_f(unsigned n, float t) { return (unsigned)(n - ceilf(jac_min_overlap_f(n, n, t)) + 1); }
/* The reference gives an empty record a prefix of 1 and so reads its
   neighbour's first token (similarity.cuh:43-58 with n = 0); here an empty
   record has empty prefixes and takes part in no pair. */
static unsigned probe_prefix(unsigned n, float t) { return n ? jac_max_prefix_f(n, t) : 0; }
static unsigned index_prefix(unsigned n, float t) { return n ? jac_mid_prefix_f(n, t) : 0; }

float orc_min_overlap(float t, uint32_t a, uint32_t b) { return jac_min_overlap_f(a, b, t); }
uint32_t orc_max_prefix(float t, uint32_t n) { return jac_max_prefix_f(n, t); }
uint32_t orc_mid_prefix(float t, uint32_t n) { return jac_mid_prefix_f(n, t); }
uint32_t orc_min_size(float t, uint32_t n) { return (uint32_t)floorf(jac_min_size_f(n, t)); }
uint32_t orc_max_size(float t, uint32_t n) { return (uint32_t)floorf(jac_max_size_f(n, t)); }
/* block.cu:191 + similarity.cuh:78-82: float(inter) / float(a + b - inter) */
float orc_similarity(uint32_t a, uint32_t b, uint32_t inter)
{
    unsigned uni = a + b - inter;
    return (float)inter / (float)uni;
}

/* ------------------------------------------------------------------------ */
/* Tokenizer                                                                 */
/* ------------------------------------------------------------------------ */

typedef struct {
    uint64_t gram;   /* packed bytes (q <= 8) or a 64-bit FNV-1a hash (q > 8) / 2-bit k-mer */
    uint32_t occ;    /* occurrence number of the gram inside its record (suffix mode) */
    uint32_t line;   /* 0-based index among the non-empty lines */
    uint32_t pos;    /* gram position in the line */
    uint32_t id;     /* assigned term id */
} orc_tok;

static char lower_ascii(char c) { return (c <= 'Z' && c >= 'A') ? (char)(c - ('Z' - 'z')) : c; }

static uint64_t gram_key(const unsigned char* p, int q)
{
    if (q <= 8) {
        uint64_t k = 0;
        for (int i = 0; i < q; i++) k = (k << 8) | p[i];
        return k;
    }
    uint64_t h = 1469598103934665603ULL;
    for (int i = 0; i < q; i++) { h ^= p[i]; h *= 1099511628211ULL; }
    return h;
}

static int cmp_line_gram_pos(const void* a, const void* b)
{
    const orc_tok* x = (const orc_tok*)a; const orc_tok* y = (const orc_tok*)b;
    if (x->line != y->line) return x->line < y->line ? -1 : 1;
    if (x->gram != y->gram) return x->gram < y->gram ? -1 : 1;
    if (x->pos != y->pos) return x->pos < y->pos ? -1 : 1;
    return 0;
}
static int cmp_key_line(const void* a, const void* b)
{
    const orc_tok* x = (const orc_tok*)a; const orc_tok* y = (const orc_tok*)b;
    if (x->gram != y->gram) return x->gram < y->gram ? -1 : 1;
    if (x->occ != y->occ) return x->occ < y->occ ? -1 : 1;
    if (x->line != y->line) return x->line < y->line ? -1 : 1;
    if (x->pos != y->pos) return x->pos < y->pos ? -1 : 1;
    return 0;
}
static int cmp_line_id(const void* a, const void* b)
{
    const orc_tok* x = (const orc_tok*)a; const orc_tok* y = (const orc_tok*)b;
    if (x->line != y->line) return x->line < y->line ? -1 : 1;
    if (x->id != y->id) return x->id < y->id ? -1 : 1;
    return 0;
}

typedef struct { uint64_t df; uint64_t first; uint32_t run; } orc_term;
static int cmp_term(const void* a, const void* b)
{
    const orc_term* x = (const orc_term*)a; const orc_term* y = (const orc_term*)b;
    if (x->df != y->df) return x->df < y->df ? -1 : 1;
    if (x->first != y->first) return x->first < y->first ? -1 : 1;
    return 0;
}

typedef struct { uint32_t line; uint32_t size; } orc_rec;
static int cmp_rec(const void* a, const void* b)
{
    const orc_rec* x = (const orc_rec*)a; const orc_rec* y = (const orc_rec*)b;
    if (x->size != y->size) return x->size < y->size ? -1 : 1;
    if (x->line != y->line) return x->line < y->line ? -1 : 1;
    return 0;
}

static int kmer_code(const unsigned char* p, int k, uint64_t* out)
{
    uint64_t f = 0, r = 0;
    for (int i = 0; i < k; i++) {
        int c;
        switch (lower_ascii((char)p[i])) {
            case 'a': c = 0; break; case 'c': c = 1; break;
            case 'g': c = 2; break; case 't': c = 3; break;
            default: return 0;
        }
        f = (f << 2) | (uint64_t)c;
        r |= (uint64_t)(3 - c) << (2 * i);
    }
    *out = f < r ? f : r;
    return 1;
}

/*
 * Text -> records in FILE order (ascending size, ties by line), the layout of
 * a ppjoin .bin.  Output arrays are malloc'd; free with orc_free.
 *   mode: 0 = q-grams, 1 = canonical k-mers (q is k, ACGT only)
 *   pad:  q-grams are padded with q-1 copies of pad_char on both sides
 *   suffix: 1 = every occurrence is its own token (gram + occurrence number,
 *           qgram.cpp:27-44); 0 = distinct grams (first occurrence kept)
 */
int orc_tokenize(const char* text, uint64_t nbytes, int q, int mode, int pad, int pad_char,
                 int suffix, int lower,
                 uint32_t* n_sets_out, uint64_t* n_tokens_out, uint32_t* n_terms_out,
                 uint32_t** ids, uint32_t** lens, uint32_t** tokens, uint32_t** locs)
{
    if (q < 1 || q > 1024) return ORC_ERR_ARG;
    /* split into non-empty lines (io.cpp:8-26) */
    uint64_t nl = 0, cap = 1024;
    uint64_t* ls = (uint64_t*)malloc(cap * sizeof(uint64_t));
    uint64_t* le = (uint64_t*)malloc(cap * sizeof(uint64_t));
    uint64_t start = 0;
    for (uint64_t i = 0; i <= nbytes; i++) {
        if (i == nbytes || text[i] == '\n') {
            if (i > start) {
                if (nl == cap) { cap *= 2; ls = (uint64_t*)realloc(ls, cap * 8); le = (uint64_t*)realloc(le, cap * 8); }
                ls[nl] = start; le[nl] = i; nl++;
            }
            start = i + 1;
        }
    }
    /* grams per line */
    uint64_t total = 0;
    for (uint64_t l = 0; l < nl; l++) {
        int64_t len = (int64_t)(le[l] - ls[l]);
        int64_t g = (mode == 0 && pad) ? len + q - 1 : len - q + 1;
        if (g > 0) total += (uint64_t)g;
    }
    orc_tok* tk = (orc_tok*)malloc((total ? total : 1) * sizeof(orc_tok));
    unsigned char* buf = (unsigned char*)malloc(1 << 20);
    size_t bufcap = 1 << 20;
    uint64_t nt = 0;
    for (uint64_t l = 0; l < nl; l++) {
        uint64_t len = le[l] - ls[l];
        size_t need = len + 2 * (size_t)q + 8;
        if (need > bufcap) { bufcap = need * 2; buf = (unsigned char*)realloc(buf, bufcap); }
        size_t o = 0;
        int npad = (mode == 0 && pad) ? q - 1 : 0;
        for (int i = 0; i < npad; i++) buf[o++] = (unsigned char)pad_char;
        for (uint64_t i = 0; i < len; i++) {
            char c = text[ls[l] + i];
            buf[o++] = (unsigned char)(lower ? lower_ascii(c) : c);
        }
        for (int i = 0; i < npad; i++) buf[o++] = (unsigned char)pad_char;
        int64_t g = (int64_t)o - q + 1;
        for (int64_t p = 0; p < g; p++) {
            uint64_t key;
            if (mode == 1) { if (!kmer_code(buf + p, q, &key)) continue; }
            else key = gram_key(buf + p, q);
            tk[nt].gram = key; tk[nt].occ = 0; tk[nt].line = (uint32_t)l; tk[nt].pos = (uint32_t)p; tk[nt].id = 0;
            nt++;
        }
    }
    free(buf);
    /* occurrence numbering / dedup within each line */
    qsort(tk, nt, sizeof(orc_tok), cmp_line_gram_pos);
    uint64_t w = 0;
    for (uint64_t i = 0; i < nt; i++) {
        int same = (i > 0 && tk[i].line == tk[i - 1].line && tk[i].gram == tk[i - 1].gram);
        if (suffix && mode == 0) {
            tk[i].occ = same ? tk[i - 1].occ + 1 : 0;
            tk[w++] = tk[i];
        } else if (!same) {
            tk[w++] = tk[i];
        }
    }
    nt = w;
    /* document frequency and first occurrence per term */
    qsort(tk, nt, sizeof(orc_tok), cmp_key_line);
    uint64_t nterms = 0;
    for (uint64_t i = 0; i < nt; i++)
        if (i == 0 || tk[i].gram != tk[i - 1].gram || tk[i].occ != tk[i - 1].occ) nterms++;
    orc_term* terms = (orc_term*)malloc((nterms ? nterms : 1) * sizeof(orc_term));
    uint32_t* run_of = (uint32_t*)malloc((nt ? nt : 1) * sizeof(uint32_t));
    int64_t r = -1;
    for (uint64_t i = 0; i < nt; i++) {
        if (i == 0 || tk[i].gram != tk[i - 1].gram || tk[i].occ != tk[i - 1].occ) {
            r++;
            terms[r].df = 0;
            terms[r].first = ((uint64_t)tk[i].line << 32) | tk[i].pos; /* lines ascending inside a run */
            terms[r].run = (uint32_t)r;
        }
        terms[r].df++;
        run_of[i] = (uint32_t)r;
    }
    qsort(terms, nterms, sizeof(orc_term), cmp_term);
    uint32_t* id_of_run = (uint32_t*)malloc((nterms ? nterms : 1) * sizeof(uint32_t));
    for (uint64_t i = 0; i < nterms; i++) id_of_run[terms[i].run] = (uint32_t)i;
    for (uint64_t i = 0; i < nt; i++) tk[i].id = id_of_run[run_of[i]];
    free(terms); free(run_of); free(id_of_run);
    /* ids ascending within each record */
    qsort(tk, nt, sizeof(orc_tok), cmp_line_id);
    uint32_t* lsz = (uint32_t*)calloc(nl ? nl : 1, sizeof(uint32_t));
    uint64_t* loff = (uint64_t*)calloc(nl + 1, sizeof(uint64_t));
    for (uint64_t i = 0; i < nt; i++) lsz[tk[i].line]++;
    for (uint64_t l = 0; l < nl; l++) loff[l + 1] = loff[l] + lsz[l];
    /* records with tokens, ascending size, ties by line */
    orc_rec* rec = (orc_rec*)malloc((nl ? nl : 1) * sizeof(orc_rec));
    uint32_t nr = 0;
    for (uint64_t l = 0; l < nl; l++) if (lsz[l] > 0) { rec[nr].line = (uint32_t)l; rec[nr].size = lsz[l]; nr++; }
    qsort(rec, nr, sizeof(orc_rec), cmp_rec);
    *ids = (uint32_t*)malloc((nr ? nr : 1) * sizeof(uint32_t));
    *lens = (uint32_t*)malloc((nr ? nr : 1) * sizeof(uint32_t));
    *tokens = (uint32_t*)malloc((nt ? nt : 1) * sizeof(uint32_t));
    *locs = (uint32_t*)malloc((nt ? nt : 1) * sizeof(uint32_t));
    uint64_t o = 0;
    for (uint32_t i = 0; i < nr; i++) {
        uint32_t l = rec[i].line;
        (*ids)[i] = l + 1;                 /* 1-based line number */
        (*lens)[i] = rec[i].size;
        for (uint64_t k = loff[l]; k < loff[l + 1]; k++) { (*tokens)[o] = tk[k].id; (*locs)[o] = tk[k].pos; o++; }
    }
    *n_sets_out = nr; *n_tokens_out = nt; *n_terms_out = (uint32_t)nterms;
    free(rec); free(lsz); free(loff); free(tk); free(ls); free(le);
    return ORC_OK;
}

void orc_free(void* p) { free(p); }

/* ------------------------------------------------------------------------ */
/* Join: the reference's per-block algorithm, run on the CPU.                */
/* ------------------------------------------------------------------------ */

typedef struct {
    uint64_t candidates;     /* "# Candidates"    block.cu:180,209 */
    uint64_t intersections;  /* "# Intersections" block.cu:181,210 */
    uint64_t results;        /* "# Results"       block.cu:194,211 */
    uint64_t index_entries;  /* "# Inverted Index Entries" fgssjoin_cli.cu:92 */
    uint64_t probe_entries;  /* list entries scanned by the reference filter (unwindowed) */
} orc_stats;

typedef struct { uint32_t q, s, overlap; float sim; } orc_pair;

static int cmp_pair(const void* a, const void* b)
{
    const orc_pair* x = (const orc_pair*)a; const orc_pair* y = (const orc_pair*)b;
    if (x->q != y->q) return x->q < y->q ? -1 : 1;
    if (x->s != y->s) return x->s < y->s ? -1 : 1;
    return 0;
}

typedef struct { orc_pair* p; uint64_t n, cap; } pairvec;
static void pv_push(pairvec* v, orc_pair x)
{
    if (v->n == v->cap) { v->cap = v->cap ? v->cap * 2 : 256; v->p = (orc_pair*)realloc(v->p, v->cap * sizeof(orc_pair)); }
    v->p[v->n++] = x;
}

/*
 * Self-join over records in MEMORY order (data.cu:97-113: the .bin order
 * reversed, so descending size for a well-formed file).
 *   pos/len/tokens: the reference's sets_t arrays; tokens ascending per record.
 *   block_size: the reference's tile edge (block.cu:14-54); 0 means one tile
 *               covering every record.
 *   q_lo, q_hi: only queries (first records of pairs) in [q_lo, q_hi); 0, 0 = all
 *               (a shard of the join, for the multi-GPU tests).
 *   side:       NULL, or one byte per record; pairs of records with the same
 *               side byte are skipped before any filter (the R-S join as the
 *               self-join of R and S together restricted to pairs across).
 *   q_step, q_phase: with q_step > 1 only queries q with (q - q_lo) % q_step
 *               == q_phase (a strided sample of the queries, keeping their
 *               size distribution: the bounded CPU baseline of large joins).
 *   want_cands: if nonzero, *cands receives every candidate as
 *               (q, s, partial score) triples -- the cells with score > 0
 *               after filtering (filtering.cu:52-57 / compaction.cu:8-17).
 * Returns the number of result pairs (sorted by (q, s)) or a negative error.
 */
int64_t orc_join(const uint32_t* pos, const uint32_t* len, const uint32_t* tokens,
                 uint32_t n, uint32_t n_terms, float t, uint32_t block_size, int nthreads,
                 orc_pair** out, orc_stats* st, int want_cands, uint32_t** cands, uint64_t* n_cands,
                 uint32_t q_lo, uint32_t q_hi, const uint8_t* side, uint32_t q_step, uint32_t q_phase)
{
    if (!(t > 0.0f && t < 1.0f)) return -ORC_ERR_ARG;
    memset(st, 0, sizeof(*st));
    *out = NULL;
    if (cands) *cands = NULL;
    if (n_cands) *n_cands = 0;
    if (n == 0) return 0;
    if (block_size == 0 || block_size > n) block_size = n;
    /* Inverted index of mid-prefix tokens (data.cu:241-278, index.cu:276-342).
       Lists are kept in ascending set order; the reference's atomic scatter
       leaves them unordered, which the filter does not depend on because a set
       appears at most once per list. */
    uint64_t* cnt = (uint64_t*)calloc((size_t)n_terms + 1, sizeof(uint64_t));
    for (uint32_t i = 0; i < n; i++) {
        uint32_t ip = index_prefix(len[i], t);
        for (uint32_t j = 0; j < ip; j++) cnt[tokens[pos[i] + j] + 1]++;
    }
    for (uint32_t w = 0; w < n_terms; w++) cnt[w + 1] += cnt[w];
    uint64_t E = cnt[n_terms];
    uint32_t* ent_s = (uint32_t*)malloc((E ? E : 1) * sizeof(uint32_t));
    uint32_t* ent_p = (uint32_t*)malloc((E ? E : 1) * sizeof(uint32_t));
    uint64_t* fill = (uint64_t*)malloc(((size_t)n_terms + 1) * sizeof(uint64_t));
    memcpy(fill, cnt, ((size_t)n_terms + 1) * sizeof(uint64_t));
    for (uint32_t i = 0; i < n; i++) {
        uint32_t ip = index_prefix(len[i], t);
        for (uint32_t j = 0; j < ip; j++) {
            uint32_t w = tokens[pos[i] + j];
            ent_s[fill[w]] = i; ent_p[fill[w]] = j; fill[w]++;
        }
    }
    free(fill);
    st->index_entries = E;

    uint32_t nblocks = (n + block_size - 1) / block_size;
    pairvec res = {0, 0, 0};
    pairvec cv = {0, 0, 0};
    uint64_t g_cand = 0, g_inter = 0, g_probe = 0;
    int nt = nthreads > 0 ? nthreads : 1;
    (void)nt;

#pragma omp parallel num_threads(nt) reduction(+ : g_cand, g_inter, g_probe)
    {
        short* score = (short*)calloc(block_size, sizeof(short));
        uint32_t* touched = (uint32_t*)malloc(block_size * sizeof(uint32_t));
        pairvec lres = {0, 0, 0};
        pairvec lcv = {0, 0, 0};
        const int64_t qa = (q_hi > q_lo) ? (int64_t)q_lo : 0;
        const int64_t qb = (q_hi > q_lo) ? (int64_t)(q_hi < n ? q_hi : n) : (int64_t)n;
#pragma omp for schedule(dynamic, 16)
        for (int64_t qq = qa; qq < qb; qq++) {
            if (q_step > 1 && (uint32_t)((qq - qa) % q_step) != q_phase) continue;  /* a strided sample */
            uint32_t query = (uint32_t)qq;
            uint32_t jb = query / block_size;          /* query block */
            uint32_t q_offset = jb * block_size;
            uint32_t q_bsize = (jb == nblocks - 1) ? n - q_offset : block_size;
            for (uint32_t ib = jb; ib < nblocks; ib++) {  /* index blocks i >= j (block.cu:101-112) */
                uint32_t i_offset = ib * block_size;
                /* skip test (block.cu:121-130) */
                int q_size = (int)len[(q_offset + q_bsize) - 1];
                int s_maxsize = (int)floorf(jac_max_size_f(len[i_offset], t));
                if (q_size > s_maxsize) continue;
                /* filtering_kernel_block, one query thread (filtering.cu:84-140) */
                uint32_t ntouched = 0;
                uint32_t query_pos = pos[query], query_len = len[query];
                uint32_t qpre = probe_prefix(query_len, t);
                uint32_t q_min = (uint32_t)floorf(jac_min_size_f(query_len, t));
                uint32_t q_max = (uint32_t)floorf(jac_max_size_f(query_len, t));
                for (uint32_t j = 0; j < qpre; j++) {
                    uint32_t token = tokens[query_pos + j];
                    for (uint64_t k = cnt[token]; k < cnt[token + 1]; k++) {
                        uint32_t source = ent_s[k], source_tpos = ent_p[k];
                        g_probe++;
                        if (!(query < source && source >= i_offset && source < i_offset + block_size)) continue;
                        if (side && side[source] == side[query]) continue;
                        uint32_t source_len = len[source];
                        uint32_t s_min = (uint32_t)floorf(jac_min_size_f(source_len, t));
                        uint32_t s_max = (uint32_t)floorf(jac_max_size_f(source_len, t));
                        if (source_len < q_min || source_len > q_max || query_len < s_min || query_len > s_max) continue;
                        uint32_t b = source - i_offset;
                        short sc = score[b];
                        if (sc >= 0) {
                            if (sc == 0) touched[ntouched++] = b;
                            unsigned query_rem = query_len - j;
                            unsigned source_rem = source_len - source_tpos;
                            unsigned min_rem = query_rem < source_rem ? query_rem : source_rem;
                            float mo = jac_min_overlap_f(query_len, source_len, t);
                            if ((float)(unsigned)(sc + 1 + min_rem) < mo) score[b] = -1;
                            else score[b] = (short)(sc + 1);
                        }
                    }
                }
                /* candidates: score > 0 (compaction.cu:8-17); verification (checking.cu:93-175) */
                for (uint32_t u = 0; u < ntouched; u++) {
                    uint32_t b = touched[u];
                    short partial = score[b];
                    score[b] = 0;
                    if (partial <= 0) continue;
                    uint32_t source = b + i_offset;
                    g_cand++;
                    if (want_cands) { orc_pair cp = {query, source, (uint32_t)partial, 0.0f}; pv_push(&lcv, cp); }
                    uint32_t source_len = len[source];
                    int minoverlap = (int)floorf(jac_min_overlap_f(query_len, source_len, t));
                    unsigned p1 = 0, p2 = 0;
                    unsigned short sc = (unsigned short)partial;
                    unsigned query_prefix = jac_max_prefix_f(query_len, t);
                    unsigned source_prefix = jac_mid_prefix_f(source_len, t);
                    unsigned tkn1 = tokens[pos[query] + (query_prefix - 1)];
                    unsigned tkn2 = tokens[pos[source] + (source_prefix - 1)];
                    if (tkn1 <= tkn2) p1 = query_prefix; else p2 = source_prefix;
                    int dropped = 0;
                    while (p1 < query_len && p2 < source_len) {
                        unsigned a = tokens[pos[query] + p1];
                        unsigned c = tokens[pos[source] + p2];
                        if ((p1 == query_len - 1 && a < c) || (p2 == source_len - 1 && c < a)) break;
                        if (a == c) { sc++; p1++; p2++; }
                        else {
                            unsigned rem = a < c ? query_len - p1 : source_len - p2;
                            if ((rem + sc) < (unsigned)minoverlap) { dropped = 1; break; }
                            if (a < c) p1++; else p2++;
                        }
                    }
                    if (dropped || (int)sc < minoverlap || sc == 0) continue;
                    g_inter++;
                    float sim = orc_similarity(query_len, source_len, sc);
                    if (sim >= t) { orc_pair rp = {query, source, sc, sim}; pv_push(&lres, rp); }
                }
            }
        }
#pragma omp critical
        {
            for (uint64_t i = 0; i < lres.n; i++) pv_push(&res, lres.p[i]);
            for (uint64_t i = 0; i < lcv.n; i++) pv_push(&cv, lcv.p[i]);
        }
        free(lres.p); free(lcv.p); free(score); free(touched);
    }
    free(cnt); free(ent_s); free(ent_p);
    qsort(res.p, res.n, sizeof(orc_pair), cmp_pair);
    st->candidates = g_cand; st->intersections = g_inter; st->results = res.n; st->probe_entries = g_probe;
    if (want_cands && cands) {
        qsort(cv.p, cv.n, sizeof(orc_pair), cmp_pair);
        *cands = (uint32_t*)malloc((cv.n ? cv.n : 1) * 3 * sizeof(uint32_t));
        for (uint64_t i = 0; i < cv.n; i++) { (*cands)[3 * i] = cv.p[i].q; (*cands)[3 * i + 1] = cv.p[i].s; (*cands)[3 * i + 2] = cv.p[i].overlap; }
        *n_cands = cv.n;
    }
    free(cv.p);
    *out = res.p;
    return (int64_t)res.n;
}

/*
 * Brute-force checker: every pair q < s (memory order), exact overlap by a
 * full merge, accepted with the reference's final tests only
 * (overlap >= floor(min_overlap) and the float Jaccard test, block.cu:190-193,
 * checking.cu:110,167).  It skips every filter, so it is a superset of the
 * reference's result whenever a float32 prefix or size bound is tighter than
 * the exact one.
 */
int64_t orc_brute(const uint32_t* pos, const uint32_t* len, const uint32_t* tokens,
                  uint32_t n, float t, orc_pair** out)
{
    pairvec res = {0, 0, 0};
    for (uint32_t q = 0; q < n; q++) {
        for (uint32_t s = q + 1; s < n; s++) {
            uint32_t a = len[q], b = len[s], i = 0, j = 0, o = 0;
            const uint32_t* x = tokens + pos[q]; const uint32_t* y = tokens + pos[s];
            while (i < a && j < b) { if (x[i] == y[j]) { o++; i++; j++; } else if (x[i] < y[j]) i++; else j++; }
            if (o == 0) continue;
            int minoverlap = (int)floorf(jac_min_overlap_f(a, b, t));
            if ((int)o < minoverlap) continue;
            float sim = orc_similarity(a, b, o);
            if (sim >= t) { orc_pair p = {q, s, o, sim}; pv_push(&res, p); }
        }
    }
    *out = res.p;
    return (int64_t)res.n;
}

int orc_num_threads(void)
{
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
