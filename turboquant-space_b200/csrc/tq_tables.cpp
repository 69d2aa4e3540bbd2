// tq_tables.cpp -- host-side construction of a space's tables.
//
// The Lloyd-Max table and the sign vectors must be bit-identical to the
// reference's, so the arithmetic below follows its algorithms step for step
// (computeLloydMax space_turbo_quant.h:76-131; RndGen64/generateSigns
// turbo_quant.h:27-39, 74-86).  This file is compiled without fast-math and
// without FP contraction (see the Makefile).
#include "tq_tables.h"

#include <algorithm>
#include <cmath>
#include <cstring>

namespace tq {

namespace {

uint64_t splitmix64_next(uint64_t &state) {
    uint64_t z = (state += 0x9e3779b97f4a7c15ULL);
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

constexpr double kPi = 3.14159265358979323846;
constexpr double kSqrt1_2 = 0.70710678118654752440;

double gauss_pdf(double x) { return std::exp(-0.5 * x * x) / std::sqrt(2.0 * kPi); }
double gauss_cdf(double x) { return 0.5 * std::erfc(-x * kSqrt1_2); }

// Mean of N(0,1) restricted to [a, b).
double cell_mean(double a, double b) {
    const double mass = gauss_cdf(b) - gauss_cdf(a);
    if (mass < 1e-15) return 0.5 * (a + b);
    return (gauss_pdf(a) - gauss_pdf(b)) / mass;
}

uint32_t ordered_key(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}

float from_key(uint32_t k) {
    const uint32_t u = (k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k;
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}

}  // namespace

std::vector<float> sign_vector(size_t d, uint64_t seed) {
    std::vector<float> s(d);
    uint64_t state = seed;
    for (size_t i = 0; i < d; ++i) s[i] = (splitmix64_next(state) & 1u) ? 1.0f : -1.0f;
    return s;
}

void lloyd_max(int mse_bits, std::vector<float> &centroids, std::vector<float> &boundaries) {
    const int levels = 1 << mse_bits;
    const int half = levels / 2;
    std::vector<double> c(half), mid(half > 1 ? half - 1 : 0), next(half);
    for (int i = 0; i < half; ++i) c[i] = (i + 0.5) * 3.5 / half;
    for (int iter = 0; iter < 1000; ++iter) {
        for (int i = 0; i + 1 < half; ++i) mid[i] = 0.5 * (c[i] + c[i + 1]);
        double worst = 0.0;
        for (int i = 0; i < half; ++i) {
            const double lo = (i == 0) ? 0.0 : mid[i - 1];
            const double hi = (i == half - 1) ? 1e10 : mid[i];
            next[i] = cell_mean(lo, hi);
            worst = std::max(worst, std::abs(next[i] - c[i]));
        }
        c = next;
        if (worst < 1e-12) break;
    }
    centroids.assign(levels, 0.0f);
    boundaries.assign(levels - 1, 0.0f);
    for (int i = 0; i < half; ++i) {
        centroids[half + i] = static_cast<float>(c[i]);
        centroids[half - 1 - i] = -static_cast<float>(c[i]);
    }
    boundaries[half - 1] = 0.0f;
    for (int i = 0; i + 1 < half; ++i) {
        const double b = 0.5 * (c[i] + c[i + 1]);
        boundaries[half + i] = static_cast<float>(b);
        boundaries[half - 2 - i] = -static_cast<float>(b);
    }
}

int quant_bucket(float z, float s, float c, int buckets) {
    float y = std::fmaf(z, s, c);
    y = std::fminf(std::fmaxf(y, 0.0f), static_cast<float>(buckets - 1));
    return static_cast<int>(y);
}

bool build_quant_lut(const std::vector<float> &boundaries, int buckets, int max_k, QuantLut &lut) {
    const int nb = static_cast<int>(boundaries.size());
    if (nb < 1) return false;
    for (int i = 1; i < nb; ++i)
        if (!(boundaries[i - 1] < boundaries[i])) return false;
    const float lo = boundaries.front(), hi = boundaries.back();
    // one boundary (bits = 2): any positive width gives lo = 0 and k = 1
    const float width = (hi > lo) ? (hi - lo) / static_cast<float>(buckets) : 1.0f;
    const float r0 = lo - width, r1 = hi + width;
    lut.s = static_cast<float>(buckets) / (r1 - r0);
    lut.c = -r0 * lut.s;
    lut.buckets = buckets;
    // vmin[j]: the smallest float (by value order, -inf included) whose bucket
    // is >= j; bucket(v) is monotone non-decreasing in v, so bucket j holds
    // exactly the floats in [vmin[j], vmin[j+1]).
    std::vector<uint32_t> vmin_key(buckets + 1);
    const uint32_t kneg = ordered_key(-INFINITY), kpos = ordered_key(INFINITY);
    vmin_key[0] = kneg;
    for (int j = 1; j < buckets; ++j) {
        uint32_t a = kneg, b = kpos;  // bucket(from_key(b)) >= j always holds
        while (a < b) {
            const uint32_t m = a + (b - a) / 2;
            if (quant_bucket(from_key(m), lut.s, lut.c, buckets) >= j) b = m;
            else a = m + 1;
        }
        vmin_key[j] = a;
    }
    vmin_key[buckets] = kpos + 1;  // one past +inf
    lut.lo.assign(buckets, 0);
    lut.span.assign(buckets, 0);
    int kmax = 0;
    for (int j = 0; j < buckets; ++j) {
        // lo: boundaries strictly below every value of the bucket
        int lo_j = 0;
        const float vmin = from_key(vmin_key[j]);
        for (int b = 0; b < nb; ++b) lo_j += (boundaries[b] < vmin) ? 1 : 0;
        // hi: boundaries strictly below the next bucket's smallest value
        int hi_j = nb;
        if (vmin_key[j + 1] <= kpos) {
            const float vnext = from_key(vmin_key[j + 1]);
            hi_j = 0;
            for (int b = 0; b < nb; ++b) hi_j += (boundaries[b] < vnext) ? 1 : 0;
        }
        if (lo_j > 255) return false;
        lut.lo[j] = static_cast<uint8_t>(lo_j);
        lut.span[j] = static_cast<uint8_t>(std::min(hi_j - lo_j, 255));
        kmax = std::max(kmax, hi_j - lo_j);
    }
    if (kmax > max_k) return false;
    lut.k = kmax < 1 ? 1 : kmax;
    return true;
}

}  // namespace tq
