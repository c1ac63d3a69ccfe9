// ha_hist.cuh -- log-linear latency histograms: 16 buckets per power of two
// of clock cycles, exact below 16 cycles.  The device side files a sample,
// the host side turns bucket counts into percentiles.
#pragma once

#include <stdint.h>

#include "halloc_c.h"

namespace ha {

constexpr uint32_t kHistBuckets = HA_SERVE_HIST;

__device__ __forceinline__ uint32_t lat_bucket(unsigned long long c) {
  if (c < 16) return (uint32_t)c;
  const uint32_t e = 63 - __clzll(c);
  const uint32_t b = (e - 3) * 16 + (uint32_t)((c >> (e - 4)) & 15);
  return b < kHistBuckets ? b : kHistBuckets - 1;
}

// lower bound of a bucket, in cycles
inline double bucket_value(uint32_t b) {
  if (b < 16) return b;
  const uint32_t e = b / 16 + 3, m = b % 16;
  return (double)((16ull + m) << (e - 4));
}

// the q-quantile of the samples in h (midpoint of its bucket), 0 when empty
inline double percentile(const unsigned long long *h, double q) {
  unsigned long long total = 0;
  for (uint32_t i = 0; i < kHistBuckets; i++) total += h[i];
  if (!total) return 0;
  const double want = q * (double)total;
  unsigned long long run = 0;
  for (uint32_t i = 0; i < kHistBuckets; i++) {
    run += h[i];
    if ((double)run >= want) return 0.5 * (bucket_value(i) + bucket_value(i + 1));
  }
  return bucket_value(kHistBuckets - 1);
}

}  // namespace ha
