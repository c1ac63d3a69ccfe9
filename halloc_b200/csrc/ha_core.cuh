// ha_core.cuh -- device core of the halloc-b200 small-block allocator.
//
// Policy: halloc 0.11's slab/hash policy, step for step (size classes,
// per-size tickets, hashed first probe, probe sequence, packed slab
// counters, roomy/sparse/free/busy slab sets, head and cached-head slabs).
// A single thread calling hamalloc/hafree gets exactly the reference's
// address sequence.  Mechanism: rebuilt for sm_100a:
//   * warp aggregation with __match_any_sync / __reduce_add_sync under
//     explicit member masks, safe under independent thread scheduling;
//   * explicit PTX memory semantics: .relaxed.gpu atomics on the hot path,
//     acquire/release on locks and on head publication;
//   * every wait is bounded by %globaltimer and reports a status bit
//     instead of spinning forever;
//   * one contiguous, slab-aligned pool: pointer -> slab is a shift and a
//     range check (no address grid to read);
//   * block-size nibbles indexed by in-slab offset / 16, so hafree reads the
//     nibble and the slab descriptor in parallel;
//   * slab sets carry a one-word-per-32-words summary so a search touches
//     two words whatever the pool size.
//
// Everything here is internal; the public entry points are hamalloc/hafree
// (halloc.cu) with the unchanged halloc.h signatures.
#pragma once

#include <cuda/atomic>
#include <stdint.h>

#include "ha_types.h"
#include "ha_stamp.cuh"

namespace ha {

// ---------------------------------------------------------------------------
// device state (defined once, in halloc.cu)
// ---------------------------------------------------------------------------
extern __constant__ Config c_cfg;
extern __device__ Class g_cls[kNSizes];
// fastmod magics per size class: nchunks (x, y = low, high word), hash step (z, w)
extern __device__ uint4 g_mod[kNSizes];
extern __device__ State g_st;

// ---------------------------------------------------------------------------
// PTX helpers: explicit scope and ordering
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t lane_id() {
  uint32_t l;
  asm("mov.u32 %0, %%laneid;" : "=r"(l));
  return l;
}
__device__ __forceinline__ uint32_t lanemask_lt() {
  uint32_t m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}
__device__ __forceinline__ uint32_t sm_id() {
  uint32_t v;
  asm("mov.u32 %0, %%smid;" : "=r"(v));
  return v;
}
__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ uint32_t ld_relaxed(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ void st_relaxed(uint32_t *p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ void st_release(uint32_t *p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t atom_add(uint32_t *p, uint32_t v) {
  uint32_t o;
  asm volatile("atom.relaxed.gpu.global.add.u32 %0, [%1], %2;"
               : "=r"(o) : "l"(p), "r"(v));
  return o;
}
__device__ __forceinline__ uint32_t atom_or(uint32_t *p, uint32_t v) {
  uint32_t o;
  asm volatile("atom.relaxed.gpu.global.or.b32 %0, [%1], %2;"
               : "=r"(o) : "l"(p), "r"(v));
  return o;
}
__device__ __forceinline__ uint32_t atom_and(uint32_t *p, uint32_t v) {
  uint32_t o;
  asm volatile("atom.relaxed.gpu.global.and.b32 %0, [%1], %2;"
               : "=r"(o) : "l"(p), "r"(v));
  return o;
}
__device__ __forceinline__ void red_add(uint32_t *p, uint32_t v) {
  asm volatile("red.relaxed.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v));
}
__device__ __forceinline__ void red_or(uint32_t *p, uint32_t v) {
  asm volatile("red.relaxed.gpu.global.or.b32 [%0], %1;" ::"l"(p), "r"(v));
}
__device__ __forceinline__ void red_and(uint32_t *p, uint32_t v) {
  asm volatile("red.relaxed.gpu.global.and.b32 [%0], %1;" ::"l"(p), "r"(v));
}
__device__ __forceinline__ void fence_acq_rel() {
  asm volatile("fence.acq_rel.gpu;" ::: "memory");
}

// Slab metadata accesses (bit arrays, size nibbles, slab counters) carry an
// L2 evict-last cache policy, so that the metadata of the slabs in use stays
// in L2 while payload streams through it -- for every kernel that calls
// hamalloc / hafree, not only those launched on a stream with an access-
// policy window (ha_l2_persist_c).  Build with -DHA_L2_HINTS=0 for plain
// accesses.  (halloc's analogue: cudaFuncCachePreferL1 and ld.global.ca
// metadata loads, src/halloc.cu:279, src/utils.h:141-157.)
#ifndef HA_L2_HINTS
#define HA_L2_HINTS 1
#endif
#if HA_L2_HINTS
__device__ __forceinline__ uint64_t meta_policy() {
  uint64_t p;
  asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint32_t ld_meta(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.L2::cache_hint.u32 %0, [%1], %2;"
               : "=r"(v) : "l"(p), "l"(meta_policy()));
  return v;
}
__device__ __forceinline__ uint32_t atom_add_meta(uint32_t *p, uint32_t v) {
  uint32_t o;
  asm volatile("atom.relaxed.gpu.global.add.L2::cache_hint.u32 %0, [%1], %2, %3;"
               : "=r"(o) : "l"(p), "r"(v), "l"(meta_policy()));
  return o;
}
__device__ __forceinline__ uint32_t atom_or_meta(uint32_t *p, uint32_t v) {
  uint32_t o;
  asm volatile("atom.relaxed.gpu.global.or.L2::cache_hint.b32 %0, [%1], %2, %3;"
               : "=r"(o) : "l"(p), "r"(v), "l"(meta_policy()));
  return o;
}
__device__ __forceinline__ uint32_t atom_and_meta(uint32_t *p, uint32_t v) {
  uint32_t o;
  asm volatile("atom.relaxed.gpu.global.and.L2::cache_hint.b32 %0, [%1], %2, %3;"
               : "=r"(o) : "l"(p), "r"(v), "l"(meta_policy()));
  return o;
}
__device__ __forceinline__ void red_or_meta(uint32_t *p, uint32_t v) {
  asm volatile("red.relaxed.gpu.global.or.L2::cache_hint.b32 [%0], %1, %2;"
               ::"l"(p), "r"(v), "l"(meta_policy()));
}
__device__ __forceinline__ void red_and_meta(uint32_t *p, uint32_t v) {
  asm volatile("red.relaxed.gpu.global.and.L2::cache_hint.b32 [%0], %1, %2;"
               ::"l"(p), "r"(v), "l"(meta_policy()));
}
#else
__device__ __forceinline__ uint32_t ld_meta(const uint32_t *p) { return ld_relaxed(p); }
__device__ __forceinline__ uint32_t atom_add_meta(uint32_t *p, uint32_t v) { return atom_add(p, v); }
__device__ __forceinline__ uint32_t atom_or_meta(uint32_t *p, uint32_t v) { return atom_or(p, v); }
__device__ __forceinline__ uint32_t atom_and_meta(uint32_t *p, uint32_t v) { return atom_and(p, v); }
__device__ __forceinline__ void red_or_meta(uint32_t *p, uint32_t v) { red_or(p, v); }
__device__ __forceinline__ void red_and_meta(uint32_t *p, uint32_t v) { red_and(p, v); }
#endif

// ---------------------------------------------------------------------------
// status, bounded waits, locks
// ---------------------------------------------------------------------------
__device__ __forceinline__ void raise_status(uint32_t bit) {
  if (!(ld_relaxed(&g_st.status) & bit)) red_or(&g_st.status, bit);
}

// A wait that gives up after g_st.wait_limit_ns of %globaltimer time.
struct Deadline {
  uint64_t end;
  uint32_t polls;
  __device__ __forceinline__ Deadline() : end(0), polls(0) {}
  // true once the limit has passed; checks the clock every 16 polls
  __device__ __forceinline__ bool expired() {
    if ((++polls & 15u) != 0) return false;
    uint64_t now = globaltimer_ns();
    if (end == 0) {
      end = now + 1000ull * ld_relaxed(&g_st.wait_limit_us);
      return false;
    }
    return now >= end;
  }
  __device__ __forceinline__ void backoff() {
    __nanosleep(polls < 64 ? 32 : 256);
  }
};

__device__ __forceinline__ bool try_lock(uint32_t *m) {
  cuda::atomic_ref<uint32_t, cuda::thread_scope_device> a(*m);
  return a.exchange(1u, cuda::memory_order_acquire) == 0u;
}
// Acquires a one-word lock; false (and HA_ST_TIMEOUT raised) when the wait
// limit passes first.
__device__ __forceinline__ bool lock(uint32_t *m) {
  Deadline d;
  while (!try_lock(m)) {
    if (d.expired()) {
      raise_status(HA_ST_TIMEOUT);
      return false;
    }
    d.backoff();
  }
  return true;
}
__device__ __forceinline__ void unlock(uint32_t *m) {
  cuda::atomic_ref<uint32_t, cuda::thread_scope_device> a(*m);
  a.store(0u, cuda::memory_order_release);
}

// ---------------------------------------------------------------------------
// size classes and chunk arithmetic
// ---------------------------------------------------------------------------

// bytes -> size class 0..15: blocks are 2 or 3 units of 8 << k bytes
// (the class rule of halloc src/halloc.cu:53-67)
__device__ __forceinline__ uint32_t size_class(uint32_t n) {
  n = n < kMinBlock ? kMinBlock : n;
  uint32_t k = (32u - __clz(n)) - 5u, unit = 8u << k;
  if (n > 3u * unit) {
    k++;
    unit <<= 1;
  }
  return 2u * k + (n > 2u * unit ? 1u : 0u);
}
// tickets that share one hash slot (src/halloc.cu:101-104)
__device__ __forceinline__ uint32_t tickets_per_slot(uint32_t sid) {
  return sid < 2 ? 4u : sid < 4 ? 2u : 1u;
}
__device__ __forceinline__ Class load_class(uint32_t sid) {
  const uint4 *p = reinterpret_cast<const uint4 *>(&g_cls[sid]);
  uint4 a = __ldg(p), b = __ldg(p + 1);
  Class c;
  c.nchunks = a.x;
  c.chunk_enc = a.y;
  c.chunk_id = a.z;
  c.ncib = a.w;
  c.sparse = b.x;
  c.hash_step = b.y;
  c.roomy = b.z;
  c.busy = b.w;
  return c;
}
// encoded chunk size: (3 or 1) << 16 | shift (halloc src/size-info.h:50-70)
__device__ __forceinline__ uint32_t chunk_mul(uint32_t v, uint32_t enc) {
  return (v << (enc & 0xffffu)) * (enc >> 16);
}
__device__ __forceinline__ uint32_t chunk_div(uint32_t v, uint32_t enc) {
  if ((enc >> 16) == 3u) v /= 3u;
  return v >> (enc & 0xffffu);
}

// ---------------------------------------------------------------------------
// slab accessors
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t *ctr_of(uint32_t sb) { return &g_st.ctr[sb * kCtrStride]; }
__device__ __forceinline__ uint32_t used_of(uint32_t sb) {
  return ld_meta(ctr_of(sb)) >> kCntShift;
}
__device__ __forceinline__ uint32_t *bits_of(uint32_t sb) {
  return c_cfg.bits + ((size_t)sb << c_cfg.bit_words_sh);
}
__device__ __forceinline__ uint32_t *nibs_of(uint32_t sb) {
  return c_cfg.nibs + ((size_t)sb << c_cfg.nib_words_sh);
}
__device__ __forceinline__ char *slab_ptr(uint32_t sb) {
  return c_cfg.pool + ((size_t)sb << c_cfg.sb_sh);
}

// head words: the slab (kNone when the field is all ones) and, in head set
// 0's word of a size, the surge level (head sets 0 .. 2^level - 1 are open)
__device__ __forceinline__ uint32_t head_slab(uint32_t w) {
  const uint32_t sb = w & kSlabField;
  return sb == kSlabField ? kNone : sb;
}
__device__ __forceinline__ uint32_t head_level(uint32_t w) { return w >> kLevelShift; }
__device__ __forceinline__ uint32_t head_word(uint32_t sb, uint32_t level) {
  return (sb == kNone ? kSlabField : sb) | (level << kLevelShift);
}

// ---------------------------------------------------------------------------
// slab sets: atomic bitsets with a summary word per 32 set words
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t *set_words(uint32_t k) { return g_st.sets[k]; }
__device__ __forceinline__ uint32_t *set_sums(uint32_t k) { return g_st.sums[k]; }

// The word is written before the summary bit, with a fence between, and
// set_tidy clears the summary bit before re-reading the word, with a fence
// between: a tidy that clears a summary bit set by a concurrent put is
// ordered after that put's word write and therefore sees it and restores
// the bit.  Summary bits may be stale-set (harmless), never stale-clear.
__device__ __forceinline__ void set_put(uint32_t k, uint32_t sb) {
  uint32_t w = sb >> 5;
  red_or(&set_words(k)[w], 1u << (sb & 31));
  fence_acq_rel();
  red_or(&set_sums(k)[w >> 5], 1u << (w & 31));
  red_add(&g_st.set_epoch, 1u);
}
// Files slab sb into the free set, which keeps a count of its slabs
// (g_st.n_free; taken slabs are counted off by set_take / set_claim), for
// slabs that may be in it already.  The allocator's own paths file only
// slabs that are not, with set_put and an increment of the count: a call
// here from them costs every hamalloc a larger register frame.
__device__ __noinline__ void set_put_free(uint32_t sb) {
  const uint32_t w = sb >> 5, bit = 1u << (sb & 31);
  if (!(atom_or(&set_words(kSetFree)[w], bit) & bit)) red_add(&g_st.n_free, 1u);
  fence_acq_rel();
  red_or(&set_sums(kSetFree)[w >> 5], 1u << (w & 31));
  red_add(&g_st.set_epoch, 1u);
}
// Clears the summary bit of word w if the word is empty.
__device__ __forceinline__ void set_tidy(uint32_t k, uint32_t w) {
  uint32_t sbit = 1u << (w & 31);
  atom_and(&set_sums(k)[w >> 5], ~sbit);
  fence_acq_rel();
  if (ld_relaxed(&set_words(k)[w])) red_or(&set_sums(k)[w >> 5], sbit);
}
__device__ __forceinline__ void set_drop(uint32_t k, uint32_t sb) {
  uint32_t w = sb >> 5, bit = 1u << (sb & 31);
  uint32_t old = atom_and(&set_words(k)[w], ~bit);
  if ((old & ~bit) == 0) set_tidy(k, w);
}
// Removes slab sb from set k; false if it was not in the set.
__device__ __forceinline__ bool set_claim(uint32_t k, uint32_t sb) {
  uint32_t w = sb >> 5, bit = 1u << (sb & 31);
  uint32_t old = atom_and(&set_words(k)[w], ~bit);
  if (!(old & bit)) return false;
  if (k == kSetFree) red_add(&g_st.n_free, 0u - 1u);
  if ((old & ~bit) == 0) set_tidy(k, w);
  return true;
}
// Removes and returns the lowest slab of set k, or kNone
// (the search order of halloc src/sbset.cuh:5-35).
__device__ __noinline__ uint32_t set_take(uint32_t k) {
  uint32_t *sums = set_sums(k), *words = set_words(k);
  for (uint32_t s = 0; s < c_cfg.sum_words; s++) {
    uint32_t sw = ld_relaxed(&sums[s]);
    while (sw) {
      uint32_t w = s * 32 + (__ffs(sw) - 1);
      sw &= sw - 1;
      uint32_t word = ld_relaxed(&words[w]);
      while (word) {
        uint32_t b = __ffs(word) - 1, bit = 1u << b;
        uint32_t old = atom_and(&words[w], ~bit);
        if (old & bit) {
          if (k == kSetFree) red_add(&g_st.n_free, 0u - 1u);
          if ((old & ~bit) == 0) set_tidy(k, w);
          return w * 32 + b;
        }
        word = old & ~bit;
      }
      set_tidy(k, w);
    }
  }
  return kNone;
}

// ---------------------------------------------------------------------------
// slab state transitions (single lane; called by group leaders)
// ---------------------------------------------------------------------------

// Returns a slab with no used chunks to the free set, or, when detaching a
// head that still has chunks in use, files it as sparse.  Caller holds the
// slab lock.  (halloc src/slab.cuh:89-113)
__device__ __noinline__ void try_release(uint32_t sb, uint32_t cid, bool from_head) {
  Desc *d = &g_st.desc[sb];
  if (ld_relaxed(&d->is_head) || cid == kNone) return;
  uint32_t *c = ctr_of(sb);
  const uint32_t clear = ((kNone - cid) & kChunkField) << kChunkShift;
  for (uint32_t guard = 0;; guard++) {
    uint32_t before = atom_add(c, clear);  // chunk field := none
    if ((before >> kCntShift) == 0) {
      st_relaxed(&d->size_id, kNone);
      st_relaxed(&d->chunk_id, kNone);
      st_relaxed(&d->chunk_enc, 0);
      set_put(kSetFree, sb);  // a slab in use until now: a new member
      red_add(&g_st.n_free, 1u);
      fence_acq_rel();
      if (!from_head) set_drop(kSetSparse + cid, sb);
      return;
    }
    uint32_t again = atom_add(c, 0u - clear);  // chunk field restored
    if ((again >> kCntShift) != 0 || guard > 1024) break;
  }
  if (from_head) set_put(kSetSparse + cid, sb);
}

// Moves a non-head slab between the busy / roomy / sparse / free sets after
// its count dropped from n0 to n1 (halloc src/slab.cuh:161-224).
__device__ __noinline__ void file_after_free(uint32_t sb, uint32_t before, uint32_t change) {
  if (before & kHeadFlag) return;
  Desc *d = &g_st.desc[sb];
  uint32_t sid = ld_relaxed(&d->size_id), cid = ld_relaxed(&d->chunk_id);
  if (sid == kNone || cid == kNone) return;
  Class cl = load_class(sid);
  uint32_t n0 = before >> kCntShift, n1 = n0 - change;
  if (n1 <= cl.busy && n0 > cl.busy) {
    set_put(kSetBusy + sid, sb);
  } else if (n1 <= cl.roomy && n0 > cl.roomy) {
    set_put(kSetRoomy + sid, sb);
    fence_acq_rel();
    set_drop(kSetBusy + sid, sb);
    set_put(kSetRoomy + sid, sb);
  } else if (n1 <= cl.sparse && n0 > cl.sparse) {
    set_put(kSetSparse + cid, sb);
    fence_acq_rel();
    set_drop(kSetRoomy + sid, sb);
    set_put(kSetSparse + cid, sb);
  } else if (n1 == 0 && ((before >> kChunkShift) & kChunkField) != kChunkField) {
    if (lock(&g_st.sb_lock[sb])) {
      try_release(sb, ld_relaxed(&d->chunk_id), false);
      unlock(&g_st.sb_lock[sb]);
    }
  }
}

// Removes `n` chunks from slab sb's count, aggregated over the calling lanes
// in `mask` that name the same slab; the group leader files the slab.
__device__ __forceinline__ void count_down(uint32_t mask, uint32_t sb, uint32_t n) {
  uint32_t grp = __match_any_sync(mask, sb);
  uint32_t total = __reduce_add_sync(grp, n);
  if (lane_id() == (uint32_t)(__ffs(grp) - 1)) {
    uint32_t before = atom_add(ctr_of(sb), 0u - (total << kCntShift));
    file_after_free(sb, before, total);
  }
}

// Stops using `sb` as head and files it by occupancy.  Caller holds the slab
// lock.  The first comparison uses the ROOMY threshold of the slab's size and
// the next two read the size-table entry whose index equals the chunk id;
// both are the reference's rules (halloc src/slab.cuh:227-255) and are kept
// for identical set contents.
__device__ __noinline__ void detach(uint32_t sb) {
  Desc *d = &g_st.desc[sb];
  st_relaxed(&d->is_head, 0);
  uint32_t before = atom_add(ctr_of(sb), 0u - kHeadFlag);
  uint32_t n = before >> kCntShift;
  uint32_t sid = ld_relaxed(&d->size_id);
  if (sid >= kNSizes || n > load_class(sid).roomy) return;
  uint32_t cid = ld_relaxed(&d->chunk_id);
  if (n == 0) {
    try_release(sb, cid, true);
    return;
  }
  if (cid >= kNChunkIds) return;
  Class q = load_class(cid);
  if (n <= q.sparse)
    set_put(kSetSparse + cid, sb);
  else if (n <= q.roomy)
    set_put(kSetRoomy + sid, sb);
  else
    set_put(kSetBusy + sid, sb);
}

__device__ __forceinline__ void make_head(uint32_t sb) {
  st_relaxed(&g_st.desc[sb].is_head, 1);
  red_add(ctr_of(sb), kHeadFlag);
}

// Stops using a head of a surge set (or its prefetched slab) before it is
// busy and files it where a later head search finds it.  Unlike detach (the
// reference's rules for a busy head), a slab between the roomy and busy
// thresholds goes to the busy set of its size, so no free space is stranded
// outside every set.  Caller holds the slab lock.
__device__ __noinline__ void retire(uint32_t sb) {
  Desc *d = &g_st.desc[sb];
  st_relaxed(&d->is_head, 0);
  const uint32_t before = atom_add(ctr_of(sb), 0u - kHeadFlag);
  const uint32_t n = before >> kCntShift;
  const uint32_t sid = ld_relaxed(&d->size_id), cid = ld_relaxed(&d->chunk_id);
  if (sid >= kNSizes || cid >= kNChunkIds) return;
  if (n == 0) {
    try_release(sb, cid, true);
    return;
  }
  const Class c = load_class(sid);
  if (n <= c.sparse)
    set_put(kSetSparse + cid, sb);
  else if (n <= c.roomy)
    set_put(kSetRoomy + sid, sb);
  else if (n <= c.busy)
    set_put(kSetBusy + sid, sb);
}

// Closes surge head set hs (set 1 or above): its head and its prefetched slab
// are retired.  Unless `force`, only while the size's set-0 head word says
// the set is closed (a set opened again meanwhile keeps its head).
__device__ __noinline__ void retire_set(uint32_t hs, bool force) {
  const uint32_t sid = hs % kNSizes, set = hs / kNSizes;
  uint32_t *hlock = &g_st.head_lock[hs * kTicketStride];
  if (!lock(hlock)) return;
  if (!force && set < (1u << head_level(ld_relaxed(&g_st.head[sid])))) {
    unlock(hlock);
    return;
  }
  const uint32_t old = head_slab(ld_relaxed(&g_st.head[hs]));
  st_release(&g_st.head[hs], kSlabField);
  cuda::atomic_ref<uint32_t, cuda::thread_scope_device> cached(g_st.cached[hs]);
  const uint32_t pre = cached.exchange(kNone, cuda::memory_order_acq_rel);
  unlock(hlock);
  if (old != kNone && lock(&g_st.sb_lock[old])) {
    retire(old);
    unlock(&g_st.sb_lock[old]);
  }
  if (pre != kNone && lock(&g_st.sb_lock[pre])) {
    retire(pre);
    unlock(&g_st.sb_lock[pre]);
  }
}

// Picks the next head slab for a size: roomy slabs of the size, sparse slabs
// of its chunk size, free slabs, then busy slabs at most half way from busy
// to full (halloc src/slab.cuh:259-372).  kNone if there is none, or if a
// slab lock could not be taken in time (the slab goes back to its set).
__device__ __noinline__ uint32_t find_slab(uint32_t sid) {
  const Class c = load_class(sid);
  const uint32_t cid = c.chunk_id;
  uint32_t sb;
  while ((sb = set_take(kSetRoomy + sid)) != kNone) {
    if (!lock(&g_st.sb_lock[sb])) {
      set_put(kSetRoomy + sid, sb);
      return kNone;
    }
    Desc *d = &g_st.desc[sb];
    bool found = false;
    if (!ld_relaxed(&d->is_head) && ld_relaxed(&d->size_id) == sid) {
      if (used_of(sb) <= c.roomy) {
        found = true;
        make_head(sb);
      } else {
        set_put(kSetBusy + sid, sb);
      }
    }
    unlock(&g_st.sb_lock[sb]);
    if (found) return sb;
  }
  while ((sb = set_take(kSetSparse + cid)) != kNone) {
    if (!lock(&g_st.sb_lock[sb])) {
      set_put(kSetSparse + cid, sb);
      return kNone;
    }
    Desc *d = &g_st.desc[sb];
    bool found = false;
    if (!ld_relaxed(&d->is_head) && ld_relaxed(&d->chunk_id) == cid) {
      if (used_of(sb) <= c.sparse) {
        found = true;
        make_head(sb);
        st_relaxed(&d->size_id, sid);
      } else {
        uint32_t other = ld_relaxed(&d->size_id);
        if (other < kNSizes) set_put(kSetRoomy + other, sb);
      }
    }
    unlock(&g_st.sb_lock[sb]);
    if (found) return sb;
  }
  while ((sb = set_take(kSetFree)) != kNone) {
    if (!lock(&g_st.sb_lock[sb])) {
      set_put(kSetFree, sb);  // taken (and counted off) just above
      red_add(&g_st.n_free, 1u);
      return kNone;
    }
    Desc *d = &g_st.desc[sb];
    bool found = false;
    if (!ld_relaxed(&d->is_head)) {
      found = true;
      st_relaxed(&d->size_id, sid);
      st_relaxed(&d->chunk_id, cid);
      st_relaxed(&d->chunk_enc, c.chunk_enc);
      make_head(sb);
      red_add(ctr_of(sb), 0u - (((kNone - cid) & kChunkField) << kChunkShift));
    }
    unlock(&g_st.sb_lock[sb]);
    if (found) return sb;
  }
  while ((sb = set_take(kSetBusy + sid)) != kNone) {
    if (used_of(sb) > (c.busy + c.nchunks) / 2) continue;
    if (!lock(&g_st.sb_lock[sb])) {
      set_put(kSetBusy + sid, sb);
      return kNone;
    }
    Desc *d = &g_st.desc[sb];
    bool found = false;
    if (!ld_relaxed(&d->is_head) && ld_relaxed(&d->size_id) == sid) {
      found = true;
      make_head(sb);
    }
    unlock(&g_st.sb_lock[sb]);
    if (found) return sb;
  }
  // nothing left; with growth on, tell the host while slabs can still be backed
  if (c_cfg.growth && ld_relaxed(&g_st.committed) < c_cfg.nsbs) raise_status(HA_ST_GROW);
  return kNone;
}

// Whether any surge set of size sid holds a head or a prefetched slab (also
// a set closed by a level change whose retirement lost a race).
__device__ __noinline__ bool surge_slabs_held(uint32_t sid) {
  bool any = false;
  for (uint32_t k = 1; k < kMaxHeads; k++) {
    const uint32_t hs = k * kNSizes + sid;
    any |= head_slab(ld_relaxed(&g_st.head[hs])) != kNone;
    any |= ld_relaxed(&g_st.cached[hs]) != kNone;
  }
  return any;
}

// Closes the surge sets of every size but `own` that holds slabs in them, so
// that a search that found nothing can look again: a size that went quiet
// keeps its level until its own next head change, and its surge heads would
// otherwise hold slabs other sizes need.  A size whose set-0 lock is free
// gets level 0 written into its head word first (no warp opens its sets
// again); one whose lock is busy has its sets emptied all the same.  The
// set-0 lock of another size is only tried, never waited for.  Returns
// whether any slab was filed.
__device__ __noinline__ bool close_other_surges(uint32_t own) {
  bool any = false;
  for (uint32_t sid = 0; sid < kNSizes; sid++) {
    if (sid == own || !surge_slabs_held(sid)) continue;
    uint32_t *hlock0 = &g_st.head_lock[sid * kTicketStride];
    bool closed = false;
    if (ld_relaxed(hlock0) == 0 && try_lock(hlock0)) {
      const uint32_t w = ld_relaxed(&g_st.head[sid]);
      if (head_level(w) != 0) {
        st_release(&g_st.head[sid], head_word(head_slab(w), 0));
        red_add(&g_st.n_surge_changes, 1);
      }
      unlock(hlock0);
      closed = true;
    }
    for (uint32_t k = 1; k < kMaxHeads; k++) retire_set(k * kNSizes + sid, !closed);
    any = true;
  }
  return any;
}

// Hands a slab taken for head slot hs back to hs's prefetch slot, or, when
// another prefetch landed there first, files it again.
__device__ __noinline__ void hand_back(uint32_t hs, uint32_t sb) {
  cuda::atomic_ref<uint32_t, cuda::thread_scope_device> cached(g_st.cached[hs]);
  uint32_t expect = kNone;
  if (!cached.compare_exchange_strong(expect, sb, cuda::memory_order_acq_rel)) {
    if (lock(&g_st.sb_lock[sb])) {
      detach(sb);
      unlock(&g_st.sb_lock[sb]);
    }
  }
}

// Opens one more surge level for size sid now, keeping set 0's head slab:
// the SMs of the new sets find no head of their own and take one through
// replace_head.  Under set 0's head lock, skipped while another warp holds
// it (a head change under way makes its own decision); the same headroom
// gate as at a head change.
__device__ __forceinline__ void surge_open(uint32_t sid) {
  uint32_t *hlock = &g_st.head_lock[sid * kTicketStride];
  if (ld_relaxed(hlock) != 0 || !try_lock(hlock)) return;
  HA_PSTAT(kPsOpenLocked, 1);
  uint32_t *head = &g_st.head[sid];
  const uint32_t w = ld_relaxed(head);
  const uint32_t level = head_level(w);
  const uint32_t nfree = ld_relaxed(&g_st.n_free);
  const uint32_t committed = ld_relaxed(&g_st.committed);
  if (head_slab(w) != kNone && level < kMaxLevel &&
      (uint64_t)kSurgeFreeOpen * nfree >= committed) {
    st_release(head, head_word(head_slab(w), level + 1));
    red_add(&g_st.n_surge_changes, 1);
  }
  unlock(hlock);
}

// Counts k long-probe lanes of size sid, for 8 (the caller samples one warp
// in 8 by the SM clock `c`, the same for the whole warp), into its
// probe-storm window with a reduction: in a 1 M-thread 16-B x4 phase
// workload four warps in ten probe long without any storm, so the counting
// is kept light, and one counting warp in 64 (more bits of `c`) reads the
// count.  Once the window is full (kProbeStormUp) that warp takes it
// with an exchange and judges it: a level opens when the size gave out
// fewer than kProbeStormTickets tickets per long probe since the window
// began; either way a new window begins.  Only set 0's ticket counter is
// read: with 2^level sets open it serves that fraction of the SMs, so its
// count is scaled up by 2^level.  This function must stay a leaf (surge_open
// is inlined): with a call to a non-inlined function here, a call that never
// ran, that workload lost a third of its rate.
__device__ __noinline__ void probe_storm(uint32_t sid, uint32_t k, uint32_t c) {
  uint32_t *line = &g_st.storm[sid * kTicketStride];
  red_add(line + 2, 8u * k);
  if ((c & 0x1f8u) != 0 || ld_relaxed(line + 2) < kProbeStormUp) return;
  const uint32_t got = atomicExch(line + 2, 0u);
  if (got < kProbeStormUp) {
    // another warp judged the window just now: give these counts back
    if (got) red_add(line + 2, got);
    return;
  }
  const uint32_t tnow = ld_relaxed(&g_st.ticket[sid * kTicketStride]);
  const uint32_t level = head_level(ld_relaxed(&g_st.head[sid]));
  const bool storm = ((uint64_t)(tnow - ld_relaxed(line + 3)) << level) <
                     (uint64_t)kProbeStormTickets * got;
  st_relaxed(line + 3, tnow);
  HA_PSTAT(kPsJudge, 1);
  if (storm) HA_PSTAT(kPsStorm, 1);
  if (storm) surge_open(sid);
}

// Gives head slot hs (= set * kNSizes + size id) a new head slab once the
// current one has reached the busy threshold: the prefetched ("cached") slab
// first, then a search; the next slab is prefetched right away.  One lane
// per warp calls this.  A caller that loses the race for the slot's lock
// waits (bounded) until the head changes or the lock is released (halloc
// src/slab.cuh:378-445).
//
// The lock covers only the switch of the head.  Filing the old head and
// prefetching the next slab, which the reference also does under the lock,
// run after it is released, so other warps can use the new head meanwhile;
// a single thread still performs the reference's steps in the reference's
// order.  Two prefetches can then overlap: the loser hands its slab back.
//
// Surge sets (c_cfg.surge): when thousands of warps queue for one size's
// head (a grid far larger than its head's free space), the lock holder of
// set 0 opens more head sets for the size, each serving the SMs whose id
// modulo 2^level names it, and closes them again as the queue shrinks.  The
// level travels in set 0's head word.  A set-k slot answers kRedirect (use
// set 0) when the set is closed or finds no slab; when set 0 itself finds no
// slab while surge sets are open, it closes them all (their heads are filed
// by occupancy) and searches again, so NULL still means what it means with
// one head.  A lone thread never waits for a lock, so it never opens a set
// and gets exactly the reference's addresses.  (Probing storms open levels
// between head changes: probe_storm above.)
__device__ __noinline__ uint32_t replace_head(uint32_t hs) {
  const uint32_t sid = hs % kNSizes, set = hs / kNSizes;
  const bool surge_set = c_cfg.surge && set != 0;
  const uint32_t none = surge_set ? kRedirect : kNone;  // "no head" answer
  uint32_t *head = &g_st.head[hs];
  uint32_t *hlock = &g_st.head_lock[hs * kTicketStride];
  cuda::atomic_ref<uint32_t, cuda::thread_scope_device> cached(g_st.cached[hs]);
  const uint32_t busy = load_class(sid).busy;
  // One round trip for the head, the memo below, the lock word and (surge
  // sets) set 0's head word (test before test-and-set: while the lock is
  // held, waiting warps only read).
  const uint32_t wseen = ld_relaxed(head);
  const uint32_t epoch = ld_relaxed(&g_st.set_epoch);
  const uint32_t memo = ld_relaxed(&g_st.no_slab[hs]);
  const uint32_t held = ld_relaxed(hlock);
  const uint32_t w0 = surge_set ? ld_relaxed(&g_st.head[sid]) : 0u;
  const uint32_t seen = head_slab(wseen);
  if (surge_set && set >= (1u << head_level(w0))) return kRedirect;
  // A failed search leaves every set it looked at empty, so until a slab is
  // filed somewhere (set_epoch moves) another search would fail the same
  // way: answer at once instead of queueing for the lock to search again.
  if (memo == epoch + 1u && (seen == kNone || used_of(seen) >= busy)) return none;
  if (held == 0 && try_lock(hlock)) {
    // Under the lock, one round trip again: the head as it is now, the count
    // of the head seen before (nearly always still the head), set 0's word
    // (surge sets) and the prefetched slab, taken on the expectation that
    // the head is replaced.  The exchange comes last so that its acquire
    // does not hold up the loads.
    const uint32_t wcur = ld_relaxed(head);
    const uint32_t cur = head_slab(wcur);
    const uint32_t n_seen = seen != kNone ? used_of(seen) : 0u;
    const uint32_t w0now = surge_set ? ld_relaxed(&g_st.head[sid]) : 0u;
    uint32_t next = cached.exchange(kNone, cuda::memory_order_acquire);
    if (surge_set && set >= (1u << head_level(w0now))) {
      // the set closed while this warp came for its lock
      unlock(hlock);
      if (next != kNone && lock(&g_st.sb_lock[next])) {
        retire(next);
        unlock(&g_st.sb_lock[next]);
      }
      return kRedirect;
    }
    if (cur != kNone && (cur == seen ? n_seen : used_of(cur)) < busy) {
      // not busy after all (the reference's re-check): hand the slab back
      if (next != kNone) hand_back(hs, next);
      unlock(hlock);
      return cur;
    }
    const uint32_t level = set == 0 ? head_level(wcur) : 0u;
    uint32_t nlevel = level;
    if (next == kNone) next = find_slab(sid);
    if (next == kNone && set == 0 && c_cfg.surge && surge_slabs_held(sid)) {
      // short of slabs while surge sets hold heads: close them all, which
      // files their heads and prefetched slabs where this search finds them
      for (uint32_t k = 1; k < kMaxHeads; k++) retire_set(k * kNSizes + sid, true);
      nlevel = 0;
      next = find_slab(sid);
    }
    if (next == kNone && set == 0 && c_cfg.surge && close_other_surges(sid))
      next = find_slab(sid);
    if (next == kNone) {
      st_relaxed(&g_st.no_slab[hs], epoch + 1u);
      if (nlevel != level) st_release(head, head_word(cur, nlevel));
      unlock(hlock);
      return none;
    }
    if (set == 0 && c_cfg.surge && nlevel == level) {
      // How many warps queued for this size's heads during the old head's
      // life, and how many tickets set 0 gave out meanwhile (about the
      // allocations its head served).  Open a level when the queue is a
      // storm (kSurgeUp), or when it is long and the head served only a few
      // allocations per queued warp of its set (a head too small for the
      // grid: kSurgeTicketsUp each); close one when neither comes near.
      uint32_t *line = &g_st.storm[sid * kTicketStride];
      const uint32_t storm = atomicExch(line, 0u);
      const uint32_t tnow = ld_relaxed(&g_st.ticket[sid * kTicketStride]);
      const uint32_t tickets = tnow - ld_relaxed(line + 1);
      st_relaxed(line + 1, tnow);
      const uint32_t per_set = storm >> level;
      const bool crowded = per_set >= kSurgeQueueMin && tickets < kSurgeTicketsUp * per_set;
      const bool calm = per_set < kSurgeQueueMin / 4 || tickets >= kSurgeTicketsDown * per_set;
      // more heads hold more partly filled slabs: open a level only while a
      // quarter of the pool is free, and close one when under an eighth is
      const uint32_t nfree = ld_relaxed(&g_st.n_free);
      const uint32_t committed = ld_relaxed(&g_st.committed);
      if ((storm >= kSurgeUp || crowded) && level < kMaxLevel &&
          (uint64_t)kSurgeFreeOpen * nfree >= committed)
        nlevel = level + 1;
      else if (level > 0 &&
               ((storm < kSurgeDown && calm) || (uint64_t)kSurgeFreeClose * nfree < committed))
        nlevel = level - 1;
    }
    st_release(head, head_word(next, nlevel));
    red_add(&g_st.n_head_changes, 1);
    if (nlevel != level) red_add(&g_st.n_surge_changes, 1);
    unlock(hlock);
    if (cur != kNone) {
      if (lock(&g_st.sb_lock[cur])) {
        detach(cur);
        unlock(&g_st.sb_lock[cur]);
      }
    }
    // a level closed by the storm count: retire the heads of its sets
    for (uint32_t k = 1u << nlevel; k < (1u << level) && nlevel < level; k++)
      retire_set(k * kNSizes + sid, false);
    const uint32_t pre = find_slab(sid);
    if (pre != kNone) hand_back(hs, pre);
    return next;
  }
  // Every warp that found the head busy waits here, thousands at once when a
  // grid storms one size.  Their polls all go to the sectors of the head and
  // lock words, which the lock holder must write to end the wait, so they
  // back off to about a microsecond and read the lock word only every
  // fourth poll (the head word is what normally changes).  With surge sets
  // on, each waiting warp is counted once (up to the threshold) for the
  // lock holder's next decision.
  if (c_cfg.surge) {
    uint32_t *storm = &g_st.storm[sid * kTicketStride];
    if (ld_relaxed(storm) < kSurgeUp) red_add(storm, 1u);
  }
  Deadline dl;
  uint32_t pause = 64;
  for (uint32_t k = 0;; k++) {
    if (ld_relaxed(head) != wseen) break;
    if ((k & 3) == 0 && ld_relaxed(hlock) == 0) break;
    if (dl.expired()) {
      raise_status(HA_ST_TIMEOUT);
      return kNone;
    }
    __nanosleep(pause);
    if (pause < 1024) pause *= 2;
  }
  const uint32_t now = head_slab(ld_relaxed(head));
  return now == kNone ? none : now;
}
// ---------------------------------------------------------------------------
// allocation
// ---------------------------------------------------------------------------

// x mod d from m = floor((2^64 - 1) / d) + 1, exact for every 32-bit x and d
// (Lemire, Kaser, Kurz: "Faster remainder by direct computation", 2019).
__device__ __forceinline__ uint32_t fastmod(uint32_t x, uint64_t m, uint32_t d) {
  return (uint32_t)__umul64hi(m * x, d);
}
__device__ __forceinline__ uint64_t mod_magic(uint32_t lo, uint32_t hi) {
  return ((uint64_t)hi << 32) | lo;
}

// first probe position of a ticket: tickets_per_slot consecutive tickets
// share a slot, slots are kHashFreq blocks apart, 32-bit wraparound
// (halloc src/halloc.cu:107-122)
__device__ __forceinline__ uint32_t first_probe(uint32_t sid, uint32_t ticket, uint32_t ncib,
                                                uint64_t mn, uint32_t nchunks) {
  const uint32_t low = tickets_per_slot(sid) - 1;
  const uint32_t spread = (ticket & ~low) * kHashFreq + (ticket & low);
  return fastmod(spread * ncib, mn, nchunks);
}

// probe position after try number `round` failed (halloc
// src/slab.cuh:492-495): step ((round+1) * 64 * ncib) mod hash_step,
// position (first + (round+1) * step) mod nchunks
__device__ __forceinline__ uint32_t next_probe(uint32_t first, uint32_t round, uint32_t ncib,
                                               uint32_t nchunks, uint64_t mn, uint32_t hstep,
                                               uint64_t mh) {
  const uint32_t k = round + 1;
  const uint32_t step = fastmod(k * kStepScale * ncib, mh, hstep);
  return fastmod(first + k * step, mn, nchunks);
}

// Continues the reference's probe sequence in slab sb (halloc
// src/slab.cuh:469-498): tries `pos` as try number `round`, then the next
// positions, until a block is reserved (true), the slab count reads busy at
// an odd try, or the 32-try round ends (false).  Per lane, no warp ops.
//
// Look-ahead: the bit words of the next kLookahead positions and the slab
// count are read together (one round trip), and atom.or is issued only at
// positions whose word shows the block free.  For a thread running alone
// this makes exactly the reference's decisions -- a loaded word is what its
// atomicOr would have seen, a partly taken block is left unchanged by the
// reference's OR-and-roll-back, and the count cannot change during the
// call -- so addresses, try numbers and give-ups are identical.  Under
// concurrency a stale word only costs one more try.  Four positions: eight
// load more than they save once many warps probe a nearly full head (those
// loads queue on the same few sectors as the atomics).  `note` gets
// kProbeCalm when the call gives up at the end of a round with the count of
// its last look-ahead below the busy threshold, and kProbeLong when the
// lane's allocation has taken kLongProbeRounds look-ahead rounds or more
// (`nr` counts them across calls) in a slab under half that threshold.  `held` is a block's worth of the slab's count that the caller
// already added (its early count, kCredit): the count it reads is taken as
// that much lower -- as the reference's thread, which has counted nothing
// yet, reads it -- and the call stops after one look-ahead round with
// kProbeMore (pos and round then name the next try), so that the early
// count is used or given back soon.
constexpr uint32_t kLookahead = 4;
constexpr uint32_t kProbeCalm = 1, kProbeLong = 2, kProbeMore = 4;
__device__ __forceinline__ bool probe_from(uint32_t sb, const Class &c, uint64_t mn, uint64_t mh,
                                           uint32_t first, uint32_t block, uint32_t &pos,
                                           uint32_t &round, uint32_t held, uint32_t &nr,
                                           uint32_t &note) {
  uint32_t *bits = bits_of(sb);
  note = 0;
  for (;;) {
    nr++;
    HA_PSTAT(kPsRound, 1);
    uint32_t pp[kLookahead], ww[kLookahead];
    pp[0] = pos;
#pragma unroll
    for (uint32_t i = 1; i < kLookahead; i++)
      pp[i] = next_probe(first, round + i - 1, c.ncib, c.nchunks, mn, c.hash_step, mh);
#pragma unroll
    for (uint32_t i = 0; i < kLookahead; i++) ww[i] = ld_meta(&bits[pp[i] >> 5]);
    const uint32_t count = used_of(sb) - held;
    if (nr >= kLongProbeRounds && 2 * count < c.busy) note |= kProbeLong;
#pragma unroll
    for (uint32_t i = 0; i < kLookahead; i++) {
      const uint32_t r = round + i;  // try number of position pp[i]
      const uint32_t mask = block << (pp[i] & 31);
      if (!(ww[i] & mask)) {
        HA_PSTAT(kPsReserve, 1);
        const uint32_t old = atom_or_meta(&bits[pp[i] >> 5], mask);
        if (!(old & mask)) {
          pos = pp[i];
          round = r;
          return true;
        }
        if (~old & mask) red_and_meta(&bits[pp[i] >> 5], ~mask | (old & mask));
      }
      // try r failed
      if (r % kCountCheck == kCountCheck - 1 && count >= c.busy) {
        pos = pp[i];
        round = r;
        return false;
      }
      if ((r + 1) % kTriesPerRound >= kTriesPerRound - 1) {
        pos = pp[i];
        round = r + 1;
        if (count < c.busy) note |= kProbeCalm;
        return false;
      }
    }
    pos = next_probe(first, round + kLookahead - 1, c.ncib, c.nchunks, mn, c.hash_step, mh);
    round += kLookahead;
    if (held) {
      note |= kProbeMore;
      return false;
    }
  }
}

// Counts the blocks just reserved by the lanes of rmask, one atomic per slab
// (halloc src/slab.cuh:122-155).  Called by exactly the lanes of rmask.
// Returns false, after giving this lane's block back, when the slab no
// longer has the caller's chunk size: the lane's ncib chunks of count then
// stay added, and the caller hands them to the slow path as a credit, which
// takes them back off before its head request (no call here, so hamalloc's
// frame stays small).  Otherwise *crossed tells whether the count crossed
// the busy threshold.
__device__ __forceinline__ bool commit(uint32_t rmask, uint32_t sb, uint32_t ncib,
                                       uint32_t cid, uint32_t busy, uint32_t pos,
                                       uint32_t block, bool &crossed) {
  const uint32_t grp = __match_any_sync(rmask, sb);
  const uint32_t total = __reduce_add_sync(grp, ncib);
  const uint32_t lead = __ffs(grp) - 1;
  uint32_t before = 0;
  if (lane_id() == lead) before = atom_add_meta(ctr_of(sb), total << kCntShift);
  before = __shfl_sync(grp, before, lead);
  const bool ok = ((before >> kChunkShift) & kChunkField) == cid;
  const uint32_t n0 = before >> kCntShift;
  crossed = n0 + total >= busy && n0 < busy;
  if (!ok) red_and_meta(&bits_of(sb)[pos >> 5], ~(block << (pos & 31)));
  return ok;
}

__device__ __forceinline__ void *publish(uint32_t sb, uint32_t pos, uint32_t enc,
                                         uint32_t ncib) {
  const uint32_t off = chunk_mul(pos, enc);
  red_or_meta(&nibs_of(sb)[off >> 7], ncib << ((off >> 2) & 28));
  return slab_ptr(sb) + off;
}

// per-lane state handed from the fast attempt to the slow path
constexpr uint32_t kWant = 1;      // no block yet
constexpr uint32_t kNeedHead = 2;  // ask for a new head slab
constexpr uint32_t kMidRound = 4;  // continue the current probe call at pos
constexpr uint32_t kCredit = 8;    // a block's worth of sb's count is already this lane's
constexpr uint32_t kCreditCrossed = 16;  // that early count crossed the busy threshold

// The rest of halloc's allocation loop (src/halloc.cu:145-179 with
// src/slab.cuh:453-535), for the whole warp `warp`: new head slabs for the
// lanes that need one (one lane per size at a time), then further probe
// calls for lanes still without a block.  Every lane of `warp` calls it.
__device__ __noinline__ void *malloc_slow(uint32_t warp, uint32_t hs, uint32_t nbytes,
                                          uint32_t ticket, uint32_t sb, uint32_t pos,
                                          uint32_t round, uint32_t flags, void *p) {
  // hs: this lane's head slot (head set * kNSizes + size id)
  const uint32_t me = lane_id();
  const uint32_t sid = size_class(nbytes);
  const Class c = load_class(sid);
  const uint4 mm = __ldg(&g_mod[sid]);
  const uint64_t mn = mod_magic(mm.x, mm.y), mh = mod_magic(mm.z, mm.w);
  const uint32_t first = first_probe(sid, ticket, c.ncib, mn, c.nchunks);
  const uint32_t block = (1u << c.ncib) - 1u;
  bool want = flags & kWant, need_head = flags & kNeedHead, mid = flags & kMidRound;
  bool long_probe = false;
  // kCredit: the lane added a block's worth (ncib chunks) of sb's count with
  // no block to show for it -- malloc_small's early count for a reservation
  // that failed, or a commit in a slab that changed chunk size.  The first
  // (one look-ahead round long) probe call may use it: a block reserved in
  // sb is then already counted.  Otherwise it goes back right after that
  // call, one atomic per (warp, slab), whose returned value is looked at
  // only on the way out (a slab that is no longer a head is then filed like
  // any count-down); or, for a lane that needs a new head first, before its
  // head request, so that the old head is filed by its true count.
  uint32_t credit = (flags & kCredit) ? sb : kNone;
  const bool credit_crossed = flags & kCreditCrossed;
  uint32_t ret_before = 0, ret_total = 0, ret_sb = kNone;
  uint32_t lookahead_rounds = 0;  // this lane's, over all its probe calls
  uint32_t rounds = 0;
  for (;;) {
    if (want && ++rounds > kMaxRounds) {
      raise_status(HA_ST_LIVELOCK);
      want = false;
    }
    const bool back = credit != kNone && (need_head || !want);
    const uint32_t cmask = __ballot_sync(warp, back);
    if (back) {
      count_down(cmask, credit, c.ncib);
      credit = kNone;
    }
    // -- new head slabs -------------------------------------------------------
    uint32_t nmask = __ballot_sync(warp, need_head);
    while (nmask) {
      const uint32_t lead = __ffs(nmask) - 1;
      const uint32_t lhs = __shfl_sync(warp, hs, lead);
      uint32_t nsb = 0;
      if (me == lead) {
        HA_PSTAT(kPsHead, 1);
        nsb = replace_head(hs);
      }
      nsb = __shfl_sync(warp, nsb, lead);
      if (need_head && hs == lhs) {
        if (nsb == kRedirect) {
          // the lane's surge set closed or ran dry: go on in head set 0
          hs = sid;
          sb = head_slab(ld_relaxed(&g_st.head[hs]));
          need_head = sb == kNone;
        } else {
          sb = nsb;
          need_head = false;
          if (nsb == kNone) want = false;
        }
      }
      nmask = __ballot_sync(warp, need_head);
    }
    const uint32_t want_mask = __ballot_sync(warp, want);
    if (!want_mask) break;
    if (want) {
      bool reserved = false;
      uint32_t note = 0;
      if (sb == kNone) {
        need_head = true;
      } else {
        if (!mid) pos = first;  // a new probe call starts at the first position
        reserved = probe_from(sb, c, mn, mh, first, block, pos, round,
                              credit != kNone ? c.ncib : 0u, lookahead_rounds, note);
        long_probe |= (note & kProbeLong) != 0;
        // A round that ended in a slab below the busy threshold: the
        // reference asks for a new head here, and its re-check under the
        // head lock keeps a head that is not busy and re-reads the head
        // (src/slab.cuh:384-390,428-431).  The count is known from the
        // round's last look-ahead, so re-read the head without the lock and
        // go on probing while it is still this slab; under a probing storm
        // that spares the head lock tens of thousands of re-checks.
        if (!reserved && !(note & kProbeMore) &&
            !((note & kProbeCalm) && head_slab(ld_relaxed(&g_st.head[hs])) == sb))
          need_head = true;
      }
      mid = (note & kProbeMore) != 0;  // one look-ahead round done: go on at pos
      const bool counted = reserved && credit != kNone;
      const bool give_back = !reserved && credit != kNone;
      const uint32_t gmask = __ballot_sync(want_mask, give_back);
      if (give_back) {
        const uint32_t grp = __match_any_sync(gmask, credit);
        const uint32_t total = __reduce_add_sync(grp, c.ncib);
        if (me == (uint32_t)(__ffs(grp) - 1)) {
          ret_before = atom_add_meta(ctr_of(credit), 0u - (total << kCntShift));
          ret_total = total;
          ret_sb = credit;
        }
        credit = kNone;
      }
      const uint32_t rmask = __ballot_sync(want_mask, reserved && !counted);
      if (counted) {
        if (credit_crossed) need_head = true;
        p = publish(sb, pos, c.chunk_enc, c.ncib);
        credit = kNone;
        want = false;
      } else if (reserved) {
        bool crossed;
        if (commit(rmask, sb, c.ncib, c.chunk_id, c.busy, pos, block, crossed)) {
          if (crossed) need_head = true;
          p = publish(sb, pos, c.chunk_enc, c.ncib);
          want = false;
        } else {
          need_head = true;
          credit = sb;  // the count commit() added goes back at the loop's top
        }
      }
    }
  }
  if (ret_sb != kNone && !(ret_before & kHeadFlag)) file_after_free(ret_sb, ret_before, ret_total);
  if (!p) red_add(&g_st.n_null, 1);
  if (HA_PROBE_STORM && c_cfg.surge) {
    // one warp in 8 (by the SM clock, one lane's reading for the whole warp)
    // counts, for 8, one count per size group of its lanes that probed long;
    // the other warps skip the collectives and the call
    const uint32_t c = __shfl_sync(warp, (uint32_t)clock(), __ffs(warp) - 1);
    if ((c & 7u) == 0) {
      const uint32_t lmask = __ballot_sync(warp, long_probe);
      if (long_probe) {
        const uint32_t grp = __match_any_sync(lmask, sid);
        if (me == (uint32_t)(__ffs(grp) - 1)) probe_storm(sid, __popc(grp), c);
      }
    }
  }
  return p;
}

// Small-block allocation for the lanes of the calling warp that are active
// here; lanes may ask for different sizes.  Fast path: ticket, one probe in
// the head slab, one counter atomic per slab, the size nibble.  Everything
// else (further probes, head replacement, exhaustion) continues in
// malloc_slow exactly where the reference's loop would.
// (halloc src/halloc.cu:125-182)
// Tickets of head slot hs for the lanes of `mask` that name it: consecutive
// values in lane order, one atomic per slot and warp.
__device__ __forceinline__ uint32_t take_ticket(uint32_t mask, uint32_t hs) {
  const uint32_t grp = __match_any_sync(mask, hs);
  const uint32_t lead = __ffs(grp) - 1;
  uint32_t base = 0;
  if (lane_id() == lead) base = atom_add(&g_st.ticket[hs * kTicketStride], __popc(grp));
  base = __shfl_sync(grp, base, lead);
  return base + __popc(grp & lanemask_lt());
}

__device__ __forceinline__ void *malloc_small(uint32_t nbytes) {
  const uint32_t warp = __activemask();
  const uint32_t sid = size_class(nbytes);
  const uint4 ca = __ldg(reinterpret_cast<const uint4 *>(&g_cls[sid]));
  const uint32_t nchunks = ca.x, enc = ca.y, cid = ca.z, ncib = ca.w;
  // head slot: fixed head set of this SM with ha_set_heads_c (set 0 with the
  // reference's single head); head word and ticket in one round trip
  const uint32_t smid = sm_id();
  HA_STAMP(kStMallocIn, smid);
  uint32_t hs = (smid & (c_cfg.nheads - 1)) * kNSizes + sid;
  const uint32_t w = ld_relaxed(&g_st.head[hs]);
  uint32_t ticket = take_ticket(warp, hs);
  uint32_t sb = head_slab(w);
  HA_STAMP(kStMallocTicket, ticket ^ w);
  {
    // surge sets open for this size (set 0's word says how many): lanes on
    // the SMs of set k > 0 take that set's head and ticket instead, one
    // round trip more, only while the size is under a storm
    const uint32_t k = smid & ((1u << head_level(w)) - 1u);
    const uint32_t moved = __ballot_sync(warp, k != 0);
    if (moved && k != 0) {
      hs = k * kNSizes + sid;
      sb = head_slab(ld_relaxed(&g_st.head[hs]));
      ticket = take_ticket(moved, hs);
    }
  }
  const uint4 mm = __ldg(&g_mod[sid]);
  const uint64_t mn = mod_magic(mm.x, mm.y);
  const uint32_t first = first_probe(sid, ticket, ncib, mn, nchunks);
  const uint32_t block = (1u << ncib) - 1u;
  HA_PSTAT(kPsAlloc, 1);

  uint32_t pos = first, round = 0, flags = kWant;
  bool reserved = false;
  // The reservation's atomic, and for a one-chunk size (c_cfg.spec_mask) the
  // slab count's as well, one per (warp, slab), in the same round trip: the
  // count is added before the reservation is known to have succeeded.  Only
  // while the size has no surge set open: under a storm the counts of
  // reservations that failed would swell a head's count for a look-ahead
  // round, and the probing-storm trigger reads that count.
  const bool spec = sb != kNone && head_level(w) == 0 && ((c_cfg.spec_mask >> sid) & 1u);
  uint32_t *bw = nullptr;
  uint32_t mask = 0, old = 0;
  if (sb != kNone) {
    mask = block << (pos & 31);
    bw = &bits_of(sb)[pos >> 5];
    old = atom_or_meta(bw, mask);
  }
  const uint32_t smask = __ballot_sync(warp, spec);
  uint32_t sgrp = 0, before = 0;
  if (spec) {
    sgrp = __match_any_sync(smask, sb);
    const uint32_t lead = __ffs(sgrp) - 1;
    if (lane_id() == lead)
      before = atom_add_meta(ctr_of(sb), (uint32_t)__popc(sgrp) << kCntShift);
    before = __shfl_sync(sgrp, before, lead);
  }
  if (sb == kNone) {
    flags |= kNeedHead;
  } else {
    HA_STAMP(kStMallocProbe, old);
    if (!(old & mask)) {
      reserved = true;
    } else {
      HA_PSTAT(kPsFirstMiss, 1);
      if (~old & mask) red_and_meta(bw, ~mask | (old & mask));
      // try 0 failed: no count check at an even try; move to try 1
      const uint32_t hstep = __ldg(&g_cls[sid].hash_step);
      pos = next_probe(first, 0, ncib, nchunks, mn, hstep, mod_magic(mm.z, mm.w));
      round = 1;
      flags |= kMidRound;
    }
  }
  void *p = nullptr;
  if (spec) {
    // the early count: as commit() below, for the whole group at once.  A
    // lane whose reservation failed hands its chunk of count to the slow
    // path as a credit (kCredit), with whether the early count crossed the
    // busy threshold; so does a lane whose slab changed chunk size under it
    // (its block goes back here), which asks for a new head at once (no
    // call here, so hamalloc's frame stays small).
    HA_STAMP(kStMallocCount, before);
    const uint32_t n0 = before >> kCntShift, total = __popc(sgrp);
    const uint32_t busy = __ldg(&g_cls[sid].busy);
    const bool crossed = n0 + total >= busy && n0 < busy;
    if (((before >> kChunkShift) & kChunkField) != cid) {
      if (reserved) red_and_meta(bw, ~mask);
      reserved = false;
      flags = kWant | kNeedHead | kCredit;
    } else if (reserved) {
      p = publish(sb, pos, enc, 1u);
      flags = crossed ? kNeedHead : 0;
    } else {
      flags |= kCredit | (crossed ? kCreditCrossed : 0u);
    }
  }
  const uint32_t rmask = __ballot_sync(warp, reserved && !spec);
  if (reserved && !spec) {
    bool crossed;
    if (commit(rmask, sb, ncib, cid, __ldg(&g_cls[sid].busy), pos, block, crossed)) {
      HA_STAMP(kStMallocCount, crossed);
      p = publish(sb, pos, enc, ncib);
      flags = crossed ? kNeedHead : 0;
    } else {
      flags = kWant | kNeedHead | kCredit;
    }
  }
  if (__any_sync(warp, flags != 0)) {
    HA_STAMP(kStSlowIn, flags);
    if (flags != 0) HA_PSTAT(kPsSlow, 1);
    p = malloc_slow(warp, hs, nbytes, ticket, sb, pos, round, flags, p);
    HA_STAMP(kStSlowOut, (uint32_t)(uintptr_t)p);
  }
  HA_STAMP(kStMallocOut, (uint32_t)(uintptr_t)p);
  return p;
}

// Small-block free for every active lane of the calling warp; `off` is the
// block's offset from the start of the pool.  (halloc src/halloc.cu:211-230)
// Block starts are at least 16 B apart (24-B chunks start on 8-B
// boundaries), so in-slab offset / 16 names a block start uniquely.
__device__ __forceinline__ void free_small(uint64_t off) {
  const uint32_t sb = (uint32_t)(off >> c_cfg.sb_sh);
  const uint32_t in = (uint32_t)off & ((1u << c_cfg.sb_sh) - 1u);
  HA_STAMP(kStFreeIn, in);
  // independent loads: the block's nibble (taken and cleared) and the
  // slab's chunk size
  uint32_t *nw = &nibs_of(sb)[in >> 7];
  const uint32_t sh = (in >> 2) & 28;
  const uint32_t enc = ld_relaxed(&g_st.desc[sb].chunk_enc);
  const uint32_t old = atom_and_meta(nw, ~(15u << sh));
  const uint32_t n = (old >> sh) & 15u;
  HA_STAMP(kStFreeNibble, old ^ enc);
  const bool valid = n != 0 && enc != 0;
  if (!valid) raise_status(HA_ST_BAD_FREE);
  const uint32_t ichunk = valid ? chunk_div(in, enc) : 0;
  if (valid) red_and_meta(&bits_of(sb)[ichunk >> 5], ~(((1u << n) - 1u) << (ichunk & 31)));
  const uint32_t vmask = __ballot_sync(__activemask(), valid);
  if (valid) {
    const uint32_t grp = __match_any_sync(vmask, sb);
    const uint32_t total = __reduce_add_sync(grp, n);
    if (lane_id() == (uint32_t)(__ffs(grp) - 1)) {
      const uint32_t before = atom_add_meta(ctr_of(sb), 0u - (total << kCntShift));
      HA_STAMP(kStFreeCount, before);
      if (!(before & kHeadFlag)) file_after_free(sb, before, total);
    }
  }
  HA_STAMP(kStFreeOut, vmask);
}

}  // namespace ha
