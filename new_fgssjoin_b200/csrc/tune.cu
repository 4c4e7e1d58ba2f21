// tune.cu -- the autotuner's cache: the best launch shape of the batched
// method's fused kernel per workload class, kept in the context and in a small
// JSON file ({"key": [threads, hash_log2, regs_rt, ctas_per_sm, ms, heavy_min_probe], ...}).
#include <math.h>
#include <stdio.h>
#include <string.h>

#include <string>

#include "join.h"

namespace fgss {

std::string tune_key(uint64_t n, uint64_t n_tokens, float t) {
    int ln = n ? (int)floor(log2((double)n)) : 0;
    int la = n ? (int)floor(log2((double)n_tokens / (double)n + 1.0)) : 0;
    char buf[64];
    snprintf(buf, sizeof buf, "fused.t%03d.n%02d.a%02d", (int)lround(t * 100.0), ln, la);
    return buf;
}

TuneEntry tune_lookup(Ctx& c, const std::string& key) {
    auto it = c.tune.find(key);
    if (it != c.tune.end()) return it->second;
    TuneEntry d;
    d.threads = 64;
    d.hash_log2 = 9;
    d.regs_rt = 1024;
    d.ctas_per_sm = 0;
    return d;
}

void tune_load(Ctx& c) {
    if (c.tune_path.empty()) return;
    FILE* f = fopen(c.tune_path.c_str(), "r");
    if (!f) return;
    char line[512];
    while (fgets(line, sizeof line, f)) {
        char key[128];
        int th, hl, rt, cps, hmp = 0;
        float ms;
        const int got = sscanf(line, " \"%127[^\"]\" : [ %d , %d , %d , %d , %f , %d ]", key, &th, &hl, &rt, &cps, &ms,
                               &hmp);
        if (got == 6 || got == 7) {
            bool known = false;
            for (int i = 0; i < kNumFusedShapes; i++)
                known |= kFusedShapes[i][0] == th && kFusedShapes[i][1] == hl && kFusedShapes[i][2] == rt;
            if (!known || cps < 0 || cps > 64 || hmp < 0 || hmp > 1) continue;  // a stale or foreign entry is ignored
            TuneEntry e;
            e.threads = th;
            e.hash_log2 = hl;
            e.regs_rt = rt;
            e.ctas_per_sm = cps;
            e.ms = ms;
            e.heavy_min_probe = hmp;
            c.tune[key] = e;
        }
    }
    fclose(f);
}

void tune_save(Ctx& c) {
    if (c.tune_path.empty()) return;
    std::string tmp = c.tune_path + ".tmp";
    FILE* f = fopen(tmp.c_str(), "w");
    if (!f) return;
    fprintf(f, "{\n");
    bool first = true;
    for (auto& kv : c.tune) {
        if (kv.first.compare(0, 6, "fused.") != 0) continue;
        fprintf(f, "%s \"%s\": [%d, %d, %d, %d, %.4f, %d]", first ? "" : ",\n", kv.first.c_str(), kv.second.threads,
                kv.second.hash_log2, kv.second.regs_rt, kv.second.ctas_per_sm, kv.second.ms, kv.second.heavy_min_probe);
        first = false;
    }
    fprintf(f, "\n}\n");
    fclose(f);
    rename(tmp.c_str(), c.tune_path.c_str());
}

}  // namespace fgss
