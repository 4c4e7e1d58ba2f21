// bounds.cpp -- see bounds.h.  Compiled as host C++ with strict IEEE float
// (no fast-math, no FMA contraction) so each expression rounds exactly as
// the reference's float32 code does.
#include "bounds.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>

namespace fgss {

namespace {

// similarity.cuh:9-36, written out with the same operand types and order.
inline float min_size_f(uint32_t n, float t) { return (float)n * t; }
inline float max_size_f(uint32_t n, float t) { return (float)n / t; }
inline float min_overlap_f(uint32_t a, uint32_t b, float t) {
    volatile float r = t / (1 + t);  // one rounding, as (float)(t/(1+t))
    return r * (float)(a + b);
}
// similarity.cuh:43-58: unsigned - float + 1 evaluates in float
inline uint32_t max_prefix_f(uint32_t n, float t) {
    volatile float c = ceilf(min_size_f(n, t));
    volatile float r = (float)n - c;
    return (uint32_t)(r + 1.0f);
}
inline uint32_t mid_prefix_f(uint32_t n, float t) {
    volatile float c = ceilf(min_overlap_f(n, n, t));
    volatile float r = (float)n - c;
    return (uint32_t)(r + 1.0f);
}

int64_t ceil_div(int64_t a, int64_t b) { return a >= 0 ? (a + b - 1) / b : -((-a) / b); }

}  // namespace

void shortest_decimal(float t, int64_t* num, int64_t* den) {
    char buf[64];
    for (int digits = 1; digits <= 9; digits++) {
        snprintf(buf, sizeof buf, "%.*f", digits, (double)t);
        if (strtof(buf, nullptr) == t) {
            int64_t d = 1;
            for (int i = 0; i < digits; i++) d *= 10;
            int64_t n = llround((double)strtod(buf, nullptr) * (double)d);
            // reduce
            int64_t a = n, b = d;
            while (b) { int64_t r = a % b; a = b; b = r; }
            *num = n / a;
            *den = d / a;
            return;
        }
    }
    *num = llround((double)t * 1e9);
    *den = 1000000000;
}

void compute_bounds(float t, int mode, BoundTables& b) {
    const uint32_t L = kMaxLen;
    b.t = t;
    b.mode = mode;
    b.probe.assign(L + 1, 0);
    b.index.assign(L + 1, 0);
    b.minsz.assign(L + 1, 0);
    b.maxsz.assign(L + 1, 0);
    b.lmin.assign(L + 1, 0);
    b.cand_min.assign(2 * L + 1, 0);
    b.inter_min.assign(2 * L + 1, 0);
    b.need.assign(2 * L + 1, 0);
    if (mode == 0) {
        for (uint32_t n = 0; n <= L; n++) {
            b.probe[n] = n ? (uint16_t)max_prefix_f(n, t) : 0;
            b.index[n] = n ? (uint16_t)mid_prefix_f(n, t) : 0;
            b.minsz[n] = (uint32_t)floorf(min_size_f(n, t));
            float mx = floorf(max_size_f(n, t));
            b.maxsz[n] = mx > 4294967040.0f ? 0xffffffffu : (uint32_t)mx;
        }
        for (uint32_t S = 0; S <= 2 * L; S++) {
            // cand_min/inter_min from jac_min_overlap(a, b) with a + b = S
            float mo = min_overlap_f(S, 0, t);
            float c = ceilf(mo);
            b.cand_min[S] = (uint32_t)c;  // float(k) < mo  <=>  k < ceil(mo) for integer k < 2^24
            b.inter_min[S] = (uint32_t)floorf(mo);
            uint32_t o = b.inter_min[S] > 1 ? b.inter_min[S] : 1;
            while (o <= S / 2 + 1 && o < S) {
                float sim = (float)o / (float)(S - o);
                if (sim >= t) break;
                o++;
            }
            b.need[S] = o;
        }
    } else {
        int64_t p, q;  // t = p / q exactly
        shortest_decimal(t, &p, &q);
        for (uint32_t n = 0; n <= L; n++) {
            int64_t mins = ceil_div((int64_t)n * p, q);            // |s| >= t |x|
            int64_t ov = ceil_div((int64_t)2 * n * p, q + p);      // overlap of two n-sets
            b.probe[n] = n ? (uint16_t)(n - mins + 1) : 0;
            b.index[n] = n ? (uint16_t)(n - ov + 1) : 0;
            b.minsz[n] = (uint32_t)mins;
            int64_t mx = ((int64_t)n * q) / p;                      // |s| <= |x| / t
            b.maxsz[n] = mx > 0xffffffffLL ? 0xffffffffu : (uint32_t)mx;
        }
        for (uint32_t S = 0; S <= 2 * L; S++) {
            int64_t need = ceil_div((int64_t)S * p, q + p);        // o >= t S / (1 + t)
            b.cand_min[S] = (uint32_t)need;
            b.inter_min[S] = (uint32_t)need;
            b.need[S] = (uint32_t)(need > 1 ? need : 1);
        }
    }
    // lmin[n]: smallest m in [minsz[n], n] with maxsz[m] >= n (maxsz is non-decreasing)
    uint32_t m = 0;
    for (uint32_t n = 0; n <= L; n++) {
        while (m <= L && b.maxsz[m] < n) m++;
        uint32_t lo = b.minsz[n] > m ? b.minsz[n] : m;
        b.lmin[n] = lo;
    }
}

}  // namespace fgss
