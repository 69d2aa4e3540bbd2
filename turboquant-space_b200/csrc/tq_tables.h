// tq_tables.h -- host-side construction of a space's tables (tq_tables.cpp).
#pragma once

#include <cstddef>
#include <cstdint>
#include <vector>

namespace tq {

// generateSigns (turbo_quant.h:74-86): splitmix64 draw i, bit 0 set -> +1.
std::vector<float> sign_vector(size_t d, uint64_t seed);

// computeLloydMax (space_turbo_quant.h:76-131) for 2^mse_bits levels:
// FP64 iteration, FP32 output, ascending boundaries.
void lloyd_max(int mse_bits, std::vector<float> &centroids, std::vector<float> &boundaries);

// Bucket table of the quantizer for many boundaries: bucket(z) =
// clamp(fma(z, s, c), 0, buckets-1) truncated; lo[j] = boundaries below every
// z of bucket j; at most k more boundaries lie inside a bucket.
struct QuantLut {
    float s = 0.0f, c = 0.0f;
    int buckets = 0, k = 0;
    std::vector<uint8_t> lo;
    std::vector<uint8_t> span;  // boundaries inside bucket j (0 .. k)
};
int quant_bucket(float z, float s, float c, int buckets);
bool build_quant_lut(const std::vector<float> &boundaries, int buckets, int max_k, QuantLut &lut);

}  // namespace tq
