// ha_types.h -- constants and data layout of the halloc-b200 allocator state.
//
// Policy constants keep halloc 0.11's values (src/halloc.cu:38-45,
// src/slab.h:31-63, src/size-info.h:28-47) because the slab/hash policy, and
// with it every address a single thread receives, depends on them.  Layout
// constants (strides, limits) are this implementation's own.
#pragma once

#include <stdint.h>

#include "halloc_c.h"

namespace ha {

// ---- policy (reference values) -------------------------------------------
constexpr uint32_t kNSizes = 16;        // 2 sizes per unit x 8 units, 16..3072 B
constexpr uint32_t kNChunkIds = 4;      // chunk sizes 16, 24, 256, 384 B
constexpr uint32_t kMinBlock = 16;
constexpr uint32_t kMaxBlock = 3072;
constexpr uint32_t kFirstTicket = 0x0B0B0B0Bu;
constexpr uint32_t kHashFreq = 11;      // hash slots are 11 blocks apart
constexpr uint32_t kTriesPerRound = 32; // probe round length
constexpr uint32_t kCountCheck = 2;     // read the slab count every 2nd collision
constexpr uint32_t kStepScale = 64;     // probe step multiplier
constexpr uint32_t kNone = 0xffffffffu;

// packed slab counter word: used chunks in bits 12-31, head flag in bit 8,
// chunk id in bits 5-7 (7 = none), bits 0-4 left at 31
constexpr uint32_t kCntShift = 12;
constexpr uint32_t kHeadFlag = 1u << 8;
constexpr uint32_t kChunkShift = 5;
constexpr uint32_t kChunkField = 7u;
constexpr uint32_t kCtrInit = (kChunkField << kChunkShift) | 31u;

// ---- layout (this implementation) ----------------------------------------
constexpr uint32_t kMaxSlabs = 32768;          // 128 GiB of 4-MiB slabs
constexpr uint32_t kSetWords = kMaxSlabs / 32;
constexpr uint32_t kSumWords = kSetWords / 32;
constexpr uint32_t kSetFree = 0;
constexpr uint32_t kSetSparse = 1;             // + chunk id
constexpr uint32_t kSetRoomy = kSetSparse + kNChunkIds;  // + size id
constexpr uint32_t kSetBusy = kSetRoomy + kNSizes;       // + size id
constexpr uint32_t kNSets = kSetBusy + kNSizes;
constexpr uint32_t kTicketStride = 32;  // one 128-B line per size's ticket / lock
constexpr uint32_t kCtrStride = 8;      // one 32-B sector per slab counter
constexpr uint32_t kMaxRounds = 1u << 16;  // outer-loop bound of one hamalloc
constexpr uint32_t kMaxHeads = 8;          // head slabs per size (1 = the reference policy)
constexpr uint32_t kDefaultWaitUs = 1000000;  // 1 s

// head words: slab id in bits 0-27 (all ones = no head), and in the word of
// head set 0 the surge level in bits 28-29: 2^level head sets are open for
// the size (level 0 = the reference's single head)
constexpr uint32_t kSlabField = 0x0fffffffu;
constexpr uint32_t kLevelShift = 28;
constexpr uint32_t kMaxLevel = 3;          // 2^3 = kMaxHeads sets
constexpr uint32_t kRedirect = 0xfffffffeu;  // replace_head: use head set 0
// surge trigger: warps that queued for one size's head lock during the life
// of one head of set 0 (a grid of 1,024 warps can never reach it)
constexpr uint32_t kSurgeUp = 2048;
constexpr uint32_t kSurgeDown = 256;
// second trigger (off unless built with HA_SURGE_TICKETS_UP > 0): at least
// kSurgeQueueMin warps queued per open set while the head served fewer than
// kSurgeTicketsUp allocations per queued warp (P: 1,024 warps at most against
// a 218,890-block head); closing needs kSurgeTicketsDown per queued warp or a
// short queue
#ifndef HA_SURGE_TICKETS_UP
#define HA_SURGE_TICKETS_UP 96  // 0 turns the second trigger off
#endif
constexpr uint32_t kSurgeQueueMin = 128;
// pool headroom: a level opens only while 1/kSurgeFreeOpen of the committed
// slabs is free, and one closes per head change while under 1/kSurgeFreeClose
#ifndef HA_SURGE_FREE_OPEN
#define HA_SURGE_FREE_OPEN 4
#endif
#ifndef HA_SURGE_FREE_CLOSE
#define HA_SURGE_FREE_CLOSE 8
#endif
// third trigger, probing storms: lanes whose probe call needed
// kLongProbeRounds or more look-ahead rounds in a slab under half its busy
// threshold -- a head far from full whose first positions keep meeting taken
// chunks.  kProbeStormUp of them while the size's set-0 counter gave out
// fewer than kProbeStormTickets tickets each open a level at once (the head
// may never fill, so no head change would come to decide it).
#ifndef HA_PROBE_STORM
#define HA_PROBE_STORM 1  // 0 builds without the third trigger
#endif
constexpr uint32_t kLongProbeRounds = 2;
constexpr uint32_t kProbeStormUp = 2048;
constexpr uint32_t kProbeStormTickets = 16;
constexpr uint32_t kSurgeFreeOpen = HA_SURGE_FREE_OPEN;
constexpr uint32_t kSurgeFreeClose = HA_SURGE_FREE_CLOSE;
constexpr uint32_t kSurgeTicketsUp = HA_SURGE_TICKETS_UP;
constexpr uint32_t kSurgeTicketsDown = 4 * HA_SURGE_TICKETS_UP;

// size class, 32 bytes, the field order of halloc src/size-info.h:8-26
struct alignas(32) Class {
  uint32_t nchunks;    // chunks of this size's chunk size in one slab
  uint32_t chunk_enc;  // (3 or 1) << 16 | log2 of the power-of-two part
  uint32_t chunk_id;
  uint32_t ncib;       // chunks in one block: 1, 2, 4 or 8
  uint32_t sparse;     // thresholds, in chunks
  uint32_t hash_step;
  uint32_t roomy;
  uint32_t busy;
};

// slab descriptor
struct alignas(16) Desc {
  uint32_t size_id;    // kNone when free
  uint32_t chunk_id;   // kNone when free
  uint32_t is_head;
  uint32_t chunk_enc;  // 0 when free
};

// read-only after ha_init (constant memory)
struct Config {
  char *pool;           // slab i at pool + (i << sb_sh)
  uint64_t pool_bytes;  // nsbs << sb_sh
  uint32_t *bits;       // one bit per 16 B of pool, slab after slab
  uint32_t *nibs;       // one 4-bit block length per 16 B of pool
  uint32_t nsbs;
  uint32_t sb_sh;
  uint32_t bit_words_sh;  // log2(words of bits per slab) = sb_sh - 9
  uint32_t nib_words_sh;  // log2(words of nibbles per slab) = sb_sh - 7
  uint32_t set_words;     // ceil(nsbs / 32)
  uint32_t sum_words;     // ceil(set_words / 32)
  uint32_t nheads;        // head slabs per size, a power of two <= kMaxHeads
  uint32_t growth;        // 1: slabs are backed on demand (ha_grow_c)
  uint32_t surge;         // 1: head sets 1.. open under contention (nheads == 1 only)
  uint32_t spec_mask;     // bit s: size s adds its slab count with the reservation
};

// Early count: size classes whose blocks are one chunk (16, 24, 256, 384 B)
// add their slab count in the same round trip as the bit reservation, and a
// lane whose reservation failed keeps that chunk of count as a credit in the
// slow path.  Each thread holds at most one such chunk, so a class qualifies
// when its slab's chunk count plus every thread the device can hold fits in
// the count field (checked at init).  -DHA_SPEC_COMMIT=0 builds without it.
#ifndef HA_SPEC_COMMIT
#define HA_SPEC_COMMIT 1
#endif

// mutable allocator state (global memory, one instance per device)
// per-head arrays are indexed [ihead * kNSizes + size]; head 0 is the one
// the reference has
struct State {
  uint32_t ticket[kMaxHeads * kNSizes * kTicketStride];
  uint32_t head_lock[kMaxHeads * kNSizes * kTicketStride];
  alignas(128) uint32_t head[kMaxHeads * kNSizes];
  uint32_t cached[kMaxHeads * kNSizes];
  alignas(128) uint32_t status;
  uint32_t wait_limit_us;
  uint32_t n_head_changes;
  uint32_t n_null;
  uint32_t committed;     // slabs backed by device memory
  uint32_t n_surge_changes;  // surge level changes since init
  uint32_t n_free;        // slabs in the free set
  // bumped by every insertion into a slab set; no_slab[hs] = epoch + 1 when
  // the last head search for (head, size) hs found nothing at that epoch
  alignas(128) uint32_t set_epoch;
  uint32_t no_slab[kMaxHeads * kNSizes];
  // per size, one 128-B line: [0] warps that queued for the head lock since
  // the last change of its set-0 head, capped near kSurgeUp; [1] set 0's
  // ticket at that change; [2] long-probe lanes in the current probe-storm
  // window; [3] set 0's ticket when that window began
  alignas(128) uint32_t storm[kNSizes * kTicketStride];
  alignas(128) uint32_t ctr[kMaxSlabs * kCtrStride];
  Desc desc[kMaxSlabs];
  uint32_t sb_lock[kMaxSlabs];
  uint32_t sets[kNSets][kSetWords];
  uint32_t sums[kNSets][kSumWords];
};

}  // namespace ha
