// preprocess -- the reference's string preprocessing command, on the GPU.
//
//   preprocess selfjoin <only_file> <q_gram>                 [options]
//   preprocess dualjoin <1st_file> <2nd_file> <q_gram>       [options]
//
// Same arguments, messages and exit behaviour as the reference's
// src/preprocess_cli.cpp:22-127 (usage on stdout; a missing argument, a missing
// file or a q outside 1..1024 prints its message and exits 0), and the same
// tokenization by default: ASCII lower-case lines, unpadded q-grams with an
// occurrence suffix (src/preprocess/string/qgram.cpp:20-49), term ids by
// ascending document frequency with ties by first occurrence
// (preprocess_cli.cpp:266-340).  It prints "Number of tokens: N" and
// "Number of terms: M" on stdout as the reference does.  The reference stops
// there (preprocess_cli.cpp:346-347 "TODO"); this tool also writes what its
// join reads: <file>.<q>gram.bin and <file>.<q>gram.bin.loc in the layout of
// the reference's own fixture (test/data/string/small.txt.3gram.bin): records
// by ascending size, ids ascending inside each record, the .loc side file
// holding each token's q-gram position in its line.  dualjoin tokenizes both
// files over one vocabulary (the reference reads only its first file) and
// writes one .bin/.loc pair per file.
// Options: --pad (pad lines with q-1 pad bytes), --distinct (one token per
// distinct gram), --kmer (canonical k-mers, k = q), --no-lower, --device <n>.
// The term count is the number of distinct terms; the reference's count can
// be one short (its Df loop folds a last hash that occurs once,
// preprocess_cli.cpp:293-306).
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include <string>
#include <vector>

#include "../../include/fgss.h"

static const char* kUsage =
    "\033[1mfgssjoin\033[0m's string preprocess engine.\n"
    "Usage:\n"
    "    preprocess selfjoin <only_file> <q_gram>\n"
    "    preprocess dualjoin <1st_file> <2nd_file> <q_gram>\n"
    "Arguments:\n"
    "    <only_file>    Single file with string data, one for each line (for selfjoin)\n"
    "    <1st_file>     First file with string data (for dualjoin)\n"
    "    <2nd_file>     Second file with string data (for dualjoin)\n"
    "    <q_gram>       Qgram size (positive integer)\n"
    "Options (after the arguments): --pad --distinct --kmer --no-lower --device <n>\n";

static bool read_file(const char* path, std::vector<char>& buf) {
    FILE* f = fopen(path, "rb");
    if (!f) return false;
    fseek(f, 0, SEEK_END);
    long sz = ftell(f);
    fseek(f, 0, SEEK_SET);
    buf.assign((size_t)(sz > 0 ? sz : 0), 0);
    const bool ok = sz <= 0 || fread(buf.data(), 1, (size_t)sz, f) == (size_t)sz;
    fclose(f);
    return ok;
}

static int fail(fgss_ctx* ctx, fgss_status st, const char* what) {
    fprintf(stderr, "%s: %s (%s)\n", what, fgss_strerror(st), fgss_last_error(ctx));
    return 1;
}

static bool file_arg(const char* fname) {
    if (access(fname, F_OK) != -1) return true;
    fprintf(stderr, "File \"%s\" does not exist.\n", fname);
    return false;
}

static int write_sets(fgss_ctx* ctx, const std::string& path, int q, const fgss_sets& s) {
    const std::string bin = path + "." + std::to_string(q) + "gram.bin", loc = bin + ".loc";
    const fgss_status st = fgss_write_bin(bin.c_str(), loc.c_str(), &s);
    if (st != FGSS_OK) return fail(ctx, st, "fgss_write_bin");
    fprintf(stderr, "wrote %s (%llu records) and %s\n", bin.c_str(), (unsigned long long)s.n_sets, loc.c_str());
    return 0;
}

int main(int argc, char** argv) {
    if (argc < 2) {
        fprintf(stdout, "%s", kUsage);
        return 0;
    }
    const bool self = strcmp(argv[1], "selfjoin") == 0, dual = strcmp(argv[1], "dualjoin") == 0;
    if (!self && !dual) {
        fprintf(stderr, "%s", kUsage);
        return 0;
    }
    const int npos = self ? 4 : 5;  // argv[0], command, file(s), q
    if (argc < npos) {
        fprintf(stderr, "Missing arguments.\n\n%s", kUsage);
        return 0;
    }
    const char* f1 = argv[2];
    const char* f2 = dual ? argv[3] : nullptr;
    if (!file_arg(f1) || (f2 && !file_arg(f2))) return 0;
    const int q = atoi(argv[npos - 1]);
    if (q < 1 || q > 1024) {
        fprintf(stderr, "Bad \"qgram\" value. Must be between 1 and %d.\n", 1024);
        return 0;
    }
    fgss_tok_opts to;
    fgss_tok_opts_default(&to);
    to.q = q;
    to.mode = FGSS_TOK_QGRAM;
    to.pad = 0;
    to.suffix = 1;
    to.lower = 1;
    int device = 0;
    for (int i = npos; i < argc; i++) {
        if (strcmp(argv[i], "--pad") == 0) to.pad = 1;
        else if (strcmp(argv[i], "--distinct") == 0) to.suffix = 0;
        else if (strcmp(argv[i], "--kmer") == 0) to.mode = FGSS_TOK_KMER;
        else if (strcmp(argv[i], "--no-lower") == 0) to.lower = 0;
        else if (strcmp(argv[i], "--device") == 0 && i + 1 < argc) device = atoi(argv[++i]);
        else {
            fprintf(stderr, "%s", kUsage);
            return 0;
        }
    }
    if (to.mode == FGSS_TOK_KMER && q > 32) {
        fprintf(stderr, "Bad \"qgram\" value for k-mers. Must be between 1 and 32.\n");
        return 0;
    }
    fprintf(stdout, "Command: %s\n", argv[1]);
    fprintf(stdout, "Q-gram size: %d\n", q);
    fgss_options o;
    fgss_options_default(&o);
    o.device = device;
    fgss_ctx* ctx = nullptr;
    fgss_status st = fgss_create(&ctx, &o);
    if (st != FGSS_OK) return fail(nullptr, st, "fgss_create");
    std::vector<char> t1, t2;
    int rc = 0;
    if (!read_file(f1, t1) || (f2 && !read_file(f2, t2))) rc = fail(ctx, FGSS_ERR_IO, "read");
    if (!rc && self) {
        fgss_sets s;
        st = fgss_tokenize(ctx, t1.data(), t1.size(), &to, &s);
        if (st != FGSS_OK) {
            rc = fail(ctx, st, "fgss_tokenize");
        } else {
            fprintf(stdout, "Number of tokens: %llu\n", (unsigned long long)s.n_tokens);
            fprintf(stdout, "Number of terms: %u\n", s.n_terms);
            fflush(stdout);
            rc = write_sets(ctx, f1, q, s);
            fgss_sets_free(&s);
        }
    } else if (!rc) {
        fgss_sets r, s;
        st = fgss_tokenize_dual(ctx, t1.data(), t1.size(), t2.data(), t2.size(), &to, &r, &s);
        if (st != FGSS_OK) {
            rc = fail(ctx, st, "fgss_tokenize_dual");
        } else {
            fprintf(stdout, "Number of tokens: %llu\n", (unsigned long long)(r.n_tokens + s.n_tokens));
            fprintf(stdout, "Number of terms: %u\n", r.n_terms);
            fflush(stdout);
            rc = write_sets(ctx, f1, q, r);
            if (!rc) rc = write_sets(ctx, f2, q, s);
            fgss_sets_free(&r);
            fgss_sets_free(&s);
        }
    }
    fgss_destroy(ctx);
    return rc;
}
