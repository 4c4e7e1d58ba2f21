// fgssjoin -- command line front end of libfgss.
//
// Two argument forms:
//   fgssjoin <ppjoin.bin> <threshold> [verbose|debug]      the reference binary's form
//                                                          (src/fgssjoin_cli.cu:20-49)
//   fgssjoin -f <text> -q <q> -t <threshold> [options]     the form its README documents
//                                                          (README.md:12-15,46): text in,
//                                                          tokenized on the GPU
// Options of the second form: --pad (pad q-grams), --distinct (one token per
// distinct gram instead of gram + occurrence), --kmer (canonical k-mers, k = q),
// --method batched|plain (default batched), --bounds reference|exact, --write-bin <path> (also
// write the tokenized .bin and .bin.loc), --device <n>, -s <text>: an R-S
// join of the -f file (R) with this one (S) over one vocabulary, printing
// "id_in_R id_in_S similarity" (no reference counterpart), and
// --out <path> [--shards K] [--binary]: the pairs streamed to a file while
// the GPU joins the next of K query ranges (fgss_selfjoin_to_file).
// stdout: "id id similarity" per pair (block.cu:193); stderr: the reference's
// counters and timers (fgssjoin_cli.cu:55-65,92,108; block.cu:209-212).
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/time.h>
#include <unistd.h>

#include <string>
#include <vector>

#include "../../include/fgss.h"

static double now_us() {
    struct timeval tv;
    gettimeofday(&tv, nullptr);
    return tv.tv_sec * 1e6 + tv.tv_usec;
}

static int die(fgss_ctx* ctx, fgss_status st, const char* what) {
    fprintf(stderr, "%s: %s (%s)\n", what, fgss_strerror(st), ctx ? fgss_last_error(ctx) : fgss_last_error(nullptr));
    return 1;
}

static bool read_file(const std::string& path, std::vector<char>& buf) {
    FILE* f = fopen(path.c_str(), "rb");
    if (!f) return false;
    fseek(f, 0, SEEK_END);
    long sz = ftell(f);
    fseek(f, 0, SEEK_SET);
    buf.assign((size_t)(sz > 0 ? sz : 0), 0);
    const bool ok = sz <= 0 || fread(buf.data(), 1, (size_t)sz, f) == (size_t)sz;
    fclose(f);
    return ok;
}

static void usage(const char* argv0) {
    fprintf(stdout,
            "Usage:\n"
            "  %s <ppjoin bin file> <threshold> [verbose|debug]\n"
            "  %s -f <text file> [-s <second text file>] -q <q> -t <threshold> [--pad] [--distinct] [--kmer]\n"
            "     [--method plain|batched] [--bounds reference|exact] [--write-bin <path>] [--device <n>]\n"
            "     [--out <path> [--shards <k>] [--binary]]\n",
            argv0, argv0);
}

int main(int argc, char** argv) {
    if (argc < 3) {
        usage(argv[0]);
        return 1;
    }
    std::string bin_path, text_path, second_path, write_bin, out_path;
    int shards = 4, out_binary = 0;
    float threshold = 0.f;
    int q = 3, pad = 0, suffix = 1, kmer = 0, method = FGSS_METHOD_BATCHED, bounds = FGSS_BOUNDS_REFERENCE;
    int device = 0;
    char verbose = 0, debug = 0;
    if (argv[1][0] == '-') {
        for (int i = 1; i < argc; i++) {
            std::string a = argv[i];
            auto next = [&](const char* what) -> const char* {
                if (i + 1 >= argc) {
                    fprintf(stderr, "missing value for %s\n", what);
                    exit(1);
                }
                return argv[++i];
            };
            if (a == "-f") text_path = next("-f");
            else if (a == "-s") second_path = next("-s");
            else if (a == "--out") out_path = next("--out");
            else if (a == "--shards") shards = atoi(next("--shards"));
            else if (a == "--binary") out_binary = 1;
            else if (a == "-q") q = atoi(next("-q"));
            else if (a == "-t") threshold = (float)atof(next("-t"));
            else if (a == "--pad") pad = 1;
            else if (a == "--distinct") suffix = 0;
            else if (a == "--kmer") kmer = 1;
            else if (a == "--method") method = strcmp(next("--method"), "batched") == 0 ? FGSS_METHOD_BATCHED : FGSS_METHOD_PLAIN;
            else if (a == "--bounds") bounds = strcmp(next("--bounds"), "exact") == 0 ? FGSS_BOUNDS_EXACT : FGSS_BOUNDS_REFERENCE;
            else if (a == "--write-bin") write_bin = next("--write-bin");
            else if (a == "--device") device = atoi(next("--device"));
            else if (a == "verbose" || a == "--verbose") verbose = 1;
            else {
                usage(argv[0]);
                return 1;
            }
        }
        if (text_path.empty()) {
            usage(argv[0]);
            return 1;
        }
    } else {
        bin_path = argv[1];
        threshold = (float)atof(argv[2]);  // fgssjoin_cli.cu:31
        for (int i = 3; i < argc && i < 5; i++) {
            if (strcmp(argv[i], "verbose") == 0) verbose = 1;
            if (strcmp(argv[i], "debug") == 0) debug = 1;
        }
    }
    const std::string& in_path = bin_path.empty() ? text_path : bin_path;
    for (const std::string* pth : std::vector<const std::string*>{&in_path, &second_path}) {
        if (!pth->empty() && access(pth->c_str(), F_OK) == -1) {
            fprintf(stderr, "File \"%s\" does not exist.\n", pth->c_str());
            return 1;
        }
    }
    if (threshold <= 0.0f || threshold >= 1.0) {
        fprintf(stderr, "Threshold must be a float in the range (0.0..1.0).\n");
        return 1;
    }
    fprintf(stderr, "Document: %s\n", in_path.c_str());
    fprintf(stderr, "Algorithm: %s\n", "fgssjoin");
    fprintf(stderr, "Threshold: Jaccard %g\n", threshold);

    fgss_options o;
    fgss_options_default(&o);
    o.device = device;
    o.verbose = verbose;
    fgss_ctx* ctx = nullptr;
    fgss_status st = fgss_create(&ctx, &o);
    if (st != FGSS_OK) return die(nullptr, st, "fgss_create");

    fgss_tok_opts to;
    fgss_tok_opts_default(&to);
    to.q = q;
    to.mode = kmer ? FGSS_TOK_KMER : FGSS_TOK_QGRAM;
    to.pad = pad;
    to.suffix = suffix;
    if (!second_path.empty()) {
        // R-S join of the -f text (R) with the -s text (S)
        std::vector<char> tr, ts;
        if (!read_file(text_path, tr) || !read_file(second_path, ts)) return die(ctx, FGSS_ERR_IO, "read");
        fgss_sets r, s2;
        st = fgss_tokenize_dual(ctx, tr.data(), tr.size(), ts.data(), ts.size(), &to, &r, &s2);
        if (st != FGSS_OK) return die(ctx, st, "fgss_tokenize_dual");
        fprintf(stderr, "# Records: %llu + %llu\n# Terms: %u\n", (unsigned long long)r.n_sets,
                (unsigned long long)s2.n_sets, r.n_terms);
        fprintf(stderr, "=== BEGIN JOIN (TIMER STARTED) ===\n");
        double t0 = now_us();
        fgss_sets_view vr = fgss_sets_view_of(&r), vs = fgss_sets_view_of(&s2);
        fgss_join_opts jo;
        fgss_join_opts_default(&jo);
        jo.threshold = threshold;
        jo.method = method;
        jo.bounds = bounds;
        fgss_pairs pairs;
        fgss_stats stats;
        st = fgss_rsjoin(ctx, &vr, &vs, &jo, &pairs, &stats);
        if (st != FGSS_OK) return die(ctx, st, "fgss_rsjoin");
        fgss_pairs_print(&pairs, stdout);
        fprintf(stderr, "# Candidates: %llu\n", (unsigned long long)stats.candidates);
        fprintf(stderr, "# Intersections: %llu\n", (unsigned long long)stats.intersections);
        fprintf(stderr, "# Results: %llu\n", (unsigned long long)stats.results);
        fprintf(stderr, "===  END JOIN (TIMER STOPPED)  ===\n");
        fprintf(stderr, "Total Running Time: %g s\n", (now_us() - t0) / 1e6);
        fgss_pairs_free(&pairs);
        fgss_sets_free(&r);
        fgss_sets_free(&s2);
        fgss_destroy(ctx);
        return 0;
    }
    fprintf(stderr, "... LOADING DATASET ...\n");
    fgss_sets sets;
    memset(&sets, 0, sizeof sets);
    if (!bin_path.empty()) {
        st = fgss_load_bin(bin_path.c_str(), &sets);
        if (st != FGSS_OK) return die(ctx, st, "fgss_load_bin");
    } else {
        std::vector<char> buf;
        if (!read_file(text_path, buf)) return die(ctx, FGSS_ERR_IO, "read");
        st = fgss_tokenize(ctx, buf.data(), buf.size(), &to, &sets);
        if (st != FGSS_OK) return die(ctx, st, "fgss_tokenize");
        if (!write_bin.empty()) {
            std::string loc = write_bin + ".loc";
            st = fgss_write_bin(write_bin.c_str(), loc.c_str(), &sets);
            if (st != FGSS_OK) return die(ctx, st, "fgss_write_bin");
        }
    }
    double avg = sets.n_sets ? (double)sets.n_tokens / (double)sets.n_sets : 0.0;
    fprintf(stderr, "# Records: %llu\n", (unsigned long long)sets.n_sets);
    fprintf(stderr, "# Terms: %u\n", sets.n_terms);
    fprintf(stderr, "# Tokens: %llu\n", (unsigned long long)sets.n_tokens);
    fprintf(stderr, "# Average size: %g\n", avg);
    if (debug) {
        for (uint64_t i = 0; i < sets.n_sets; i++) {
            fprintf(stdout, "id: [%u]\nsize: [%u]\n", sets.id[i], sets.len[i]);
            for (uint32_t j = 0; j < sets.len[i]; j++) fprintf(stdout, "(%u) ", sets.tokens[sets.pos[i] + j]);
            fprintf(stdout, "\n\n");
        }
    }
    fprintf(stderr, "=== BEGIN JOIN (TIMER STARTED) ===\n");
    double t0 = now_us();
    fgss_sets_view v = fgss_sets_view_of(&sets);
    fgss_join_opts jo;
    fgss_join_opts_default(&jo);
    jo.threshold = threshold;
    jo.method = method;
    jo.bounds = bounds;
    fgss_pairs pairs;
    fgss_stats stats;
    memset(&pairs, 0, sizeof pairs);
    if (!out_path.empty()) {
        // streamed to the file shard by shard while the GPU joins the next shard
        st = fgss_selfjoin_to_file(ctx, &v, &jo, out_path.c_str(), out_binary ? FGSS_OUT_BINARY : FGSS_OUT_TEXT,
                                   shards > 0 ? shards : 1, &stats);
        if (st != FGSS_OK) return die(ctx, st, "fgss_selfjoin_to_file");
    } else {
        st = fgss_selfjoin(ctx, &v, &jo, &pairs, &stats);
        if (st != FGSS_OK) return die(ctx, st, "fgss_selfjoin");
    }
    fprintf(stderr, "# Inverted Index Entries: %llu\n", (unsigned long long)stats.index_entries);
    double r0 = now_us();
    fgss_pairs_print(&pairs, stdout);
    double r1 = now_us();
    fprintf(stderr, "# Candidates: %llu\n", (unsigned long long)stats.candidates);
    fprintf(stderr, "# Intersections: %llu\n", (unsigned long long)stats.intersections);
    fprintf(stderr, "# Results: %llu\n", (unsigned long long)stats.results);
    fprintf(stderr, "  - Time rendering: %g ms\n", (r1 - r0) / 1000.0);
    double t1 = now_us();
    fprintf(stderr, "===  END JOIN (TIMER STOPPED)  ===\n");
    fprintf(stderr, "Total Running Time: %g s\n", (t1 - t0) / 1e6);
    if (verbose)
        fprintf(stderr, "# Device ms: index %.3f, filter+verify %.3f, output %.3f\n", stats.ms_index, stats.ms_filter,
                stats.ms_output);
    fgss_pairs_free(&pairs);
    fgss_sets_free(&sets);
    fgss_destroy(ctx);
    return 0;
}
