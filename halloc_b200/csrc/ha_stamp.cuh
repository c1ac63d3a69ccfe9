// ha_stamp.cuh -- latency stamps of instrumented builds (-DHA_STAMPS).
#pragma once

#include <stdint.h>

namespace ha {

// ---------------------------------------------------------------------------
// latency stamps (instrumented builds only: -DHA_STAMPS)
// ---------------------------------------------------------------------------
// A build with HA_STAMPS records, for the lanes of the first warp of block 0,
// the SM clock after each dependent round trip of hamalloc / hafree, into
// the launch's dynamic shared memory: word `lane` counts the lane's stamps,
// then 2 words per stamp (point id, clock low word) at 32 + 2 * (lane *
// kStampSlots + i).  Only a launch that provides kStampBytes of dynamic
// shared memory gets stamps (%dynamic_smem_size is checked first), so other
// kernels of the instrumented build are untouched.  The clock is read only
// once `dep` -- a value the round trip returned -- is available: the read
// is predicated on it.  Normal builds compile HA_STAMP to nothing.
enum StampPoint : uint32_t {
  kStMallocIn = 1,   // hamalloc entered
  kStMallocTicket,   // ticket and head word back
  kStMallocProbe,    // bit reservation back
  kStMallocCount,    // slab count back (block committed)
  kStMallocOut,      // hamalloc returns
  kStSlowIn,         // slow path entered
  kStSlowOut,        // slow path returns
  kStFreeIn,         // hafree entered
  kStFreeNibble,     // size nibble and slab descriptor back
  kStFreeCount,      // count-down back
  kStFreeOut,        // hafree returns
  kStUser,           // a point of the calling kernel
};
constexpr uint32_t kStampSlots = 160;  // 41 KB of stamps: under the 48 KB default
constexpr uint32_t kStampBytes = 4 * (32 + 2 * 32 * kStampSlots);
#ifdef HA_STAMPS
extern __shared__ uint32_t ha_stamp_smem[];
__device__ __forceinline__ void stamp(uint32_t point, uint32_t dep) {
  uint32_t dyn, clk;
  asm volatile("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn));
  if (dyn < kStampBytes || blockIdx.x != 0 || threadIdx.x >= 32) return;
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.u32 p, %1, 0x5bd1e995;\n\t"
      "@p mov.u32 %0, %%clock;\n\t@!p mov.u32 %0, 0;\n\t}"
      : "=r"(clk) : "r"(dep) : "memory");
  const uint32_t lane = threadIdx.x, i = ha_stamp_smem[lane];
  if (i < kStampSlots) {
    ha_stamp_smem[32 + 2 * (lane * kStampSlots + i)] = point;
    ha_stamp_smem[33 + 2 * (lane * kStampSlots + i)] = clk;
    ha_stamp_smem[lane] = i + 1;
  }
}
#define HA_STAMP(point, dep) ::ha::stamp(point, (uint32_t)(dep))
#else
#define HA_STAMP(point, dep) ((void)0)
#endif

// ---------------------------------------------------------------------------
// probe counters (instrumented builds only: -DHA_PROBE_STATS)
// ---------------------------------------------------------------------------
// Per-lane event counts of hamalloc's probing, summed over every launch until
// read (ha_probe_stats_c).  Each event is one fire-and-forget reduction into
// one of 32 copies chosen by SM, 128 B apart, so the counting adds no
// latency to the allocator's chain and no hot word.  Normal builds compile
// HA_PSTAT to nothing.
enum ProbeStat : uint32_t {
  kPsAlloc = 0,    // lanes entering the small-block allocation
  kPsFirstMiss,    // lanes whose first probe found its chunks taken
  kPsSlow,         // lanes continuing in the slow path
  kPsRound,        // look-ahead rounds (4 bit words and the count loaded)
  kPsReserve,      // reservation atomics issued by the look-ahead
  kPsHead,         // head replacements asked for (one per warp and head slot)
  kPsJudge,        // probe-storm windows judged
  kPsStorm,        // of those, judged a storm
  kPsOpenLocked,   // surge_open calls that took set 0's head lock
  kPsCount
};
constexpr uint32_t kPsCopies = 32, kPsStride = 16;
#ifndef HA_PROBE_STATS
#define HA_PROBE_STATS 0
#endif
#if HA_PROBE_STATS
extern __device__ unsigned long long g_pstats[kPsCopies * kPsStride];
__device__ __forceinline__ void pstat(uint32_t i, uint32_t v) {
  uint32_t smid;
  asm("mov.u32 %0, %%smid;" : "=r"(smid));
  atomicAdd(&g_pstats[(smid % kPsCopies) * kPsStride + i], (unsigned long long)v);
}
#define HA_PSTAT(i, v) ::ha::pstat(i, v)
#else
#define HA_PSTAT(i, v) ((void)0)
#endif

}  // namespace ha
