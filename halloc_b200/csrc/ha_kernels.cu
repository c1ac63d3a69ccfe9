// ha_kernels.cu -- batch entry points of the C ABI (halloc_c.h).
//
// The kernels here are the reference's own test and benchmark kernels
// (halloc tst/common/common.h:361-412, tst/perf/priv-throughput), written
// against the public device API: they call hamalloc / hafree across the
// device-link boundary exactly as a user kernel does.
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <chrono>
#include <new>
#include <vector>

#include "halloc.h"
#include "halloc_c.h"
#include "ha_stamp.cuh"  // HA_STAMP (a no-op unless built with -DHA_STAMPS)
#include "ha_hist.cuh"

namespace {

constexpr uint32_t kMaxAllocsPerThread = 16;

cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

int launch_status() {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    fprintf(stderr, "halloc-b200: launch failed: %s\n", cudaGetErrorString(e));
    return HA_ECUDA;
  }
  return HA_OK;
}

uint32_t blocks_for(uint64_t n, uint32_t block) { return (uint32_t)((n + block - 1) / block); }

// 16 payload bytes at a block start.  Blocks of the 24-byte chunk classes
// start on 8-byte boundaries only, so the 16-byte vector access is used when
// the block is 16-byte aligned and two 8-byte accesses otherwise.
__device__ __forceinline__ void store16(void *p, uint4 v) {
  if (((uintptr_t)p & 15u) == 0) {
    *reinterpret_cast<uint4 *>(p) = v;
  } else {
    uint2 *q = reinterpret_cast<uint2 *>(p);
    q[0] = make_uint2(v.x, v.y);
    q[1] = make_uint2(v.z, v.w);
  }
}
// The read-back is a real load (ld.global.ca: cacheable in L1, never folded
// into the preceding store by the compiler); a thread reading its own write
// always sees it.
__device__ __forceinline__ uint4 load16(const void *p) {
  if (((uintptr_t)p & 15u) == 0) return __ldca(reinterpret_cast<const uint4 *>(p));
  const uint2 a = __ldca(reinterpret_cast<const uint2 *>(p));
  const uint2 b = __ldca(reinterpret_cast<const uint2 *>(p) + 1);
  return make_uint4(a.x, a.y, b.x, b.y);
}

// block-wide sums of two counters, one atomic each per block
__device__ __forceinline__ void block_add2(unsigned long long a, unsigned long long b,
                                           unsigned long long *pa, unsigned long long *pb) {
  __shared__ unsigned long long sa[32], sb[32];
  __syncthreads();  // a previous call may still be reading sa / sb
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
  }
  const uint32_t lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    sa[warp] = a;
    sb[warp] = b;
  }
  __syncthreads();
  if (warp == 0) {
    const uint32_t nw = (blockDim.x + 31) >> 5;
    a = lane < nw ? sa[lane] : 0;
    b = lane < nw ? sb[lane] : 0;
    for (int o = 16; o > 0; o >>= 1) {
      a += __shfl_down_sync(0xffffffffu, a, o);
      b += __shfl_down_sync(0xffffffffu, b, o);
    }
    if (lane == 0) {
      if (a) atomicAdd(pa, a);
      if (b) atomicAdd(pb, b);
    }
  }
}

}  // namespace

// malloc_k / malloc_corr_k of halloc tst/common/common.h:361-388
__global__ void ha_malloc_batch_k(const uint32_t *sizes, uint32_t n, uint32_t nallocs,
                                  void **ptrs, int tag) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (uint32_t a = 0; a < nallocs; a++) {
    const size_t k = (size_t)a * n + i;
    const uint32_t sz = sizes[k];
    void *p = hamalloc(sz);
    ptrs[k] = p;
    if (p && tag) *(uint32_t *)p = sz;
  }
}

// free_k of halloc tst/common/common.h:390-399
__global__ void ha_free_batch_k(void *const *ptrs, uint32_t n, uint32_t nallocs) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (uint32_t a = 0; a < nallocs; a++) hafree(ptrs[(size_t)a * n + i]);
}

// throughput_malloc_free_k of halloc tst/perf/priv-throughput/priv-throughput.cu:13-27,
// with the 16-byte payload write and checksummed read-back of each block:
// one thread's loop, adding its checksum and failed allocations to sum / nfail
template <bool kCudaHeap>
__device__ __forceinline__ void throughput_thread(uint32_t i, uint32_t sz, uint32_t nallocs,
                                                  uint32_t niters, unsigned long long &sum,
                                                  unsigned long long &nfail) {
  const uint4 word = make_uint4(i ^ 0u, i ^ 1u, i ^ 2u, i ^ 3u);
  if (nallocs == 1) {
    // one block per iteration (the plain configuration): the same steps
    // with the pointer in a register rather than the local array below
    for (uint32_t it = 0; it < niters; it++) {
      void *p = kCudaHeap ? malloc(sz) : hamalloc(sz);
      if (!p) {
        nfail++;
        continue;
      }
      store16(p, word);
      const uint4 v = load16(p);
      HA_STAMP(ha::kStUser, v.x);
      sum += (unsigned long long)v.x + v.y + v.z + v.w;
      if (kCudaHeap)
        free(p);
      else
        hafree(p);
    }
    return;
  }
  void *ps[kMaxAllocsPerThread];
  for (uint32_t it = 0; it < niters; it++) {
    for (uint32_t a = 0; a < nallocs; a++) {
      void *p = kCudaHeap ? malloc(sz) : hamalloc(sz);
      ps[a] = p;
      if (p)
        store16(p, word);
      else
        nfail++;
    }
    for (uint32_t a = 0; a < nallocs; a++) {
      void *p = ps[a];
      if (!p) continue;
      const uint4 v = load16(p);
      HA_STAMP(ha::kStUser, v.x);
      sum += (unsigned long long)v.x + v.y + v.z + v.w;
      if (kCudaHeap)
        free(p);
      else
        hafree(p);
    }
  }
}

template <bool kCudaHeap>
__global__ void ha_throughput_k(const uint32_t *sizes, uint32_t nbytes, uint32_t n,
                                uint32_t nallocs, uint32_t niters,
                                unsigned long long *out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long sum = 0, nfail = 0;
  if (i < n) throughput_thread<kCudaHeap>(i, sizes ? sizes[i] : nbytes, nallocs, niters, sum, nfail);
  block_add2(sum, nfail, out, out + 1);
}

// The private-throughput loop run by one warp with the latency stamps of an
// HA_STAMPS build switched on (kStampBytes of dynamic shared memory); the
// stamps are copied to out (kStampBytes / 4 words) at the end.
__global__ void ha_stamps_k(uint32_t nbytes, uint32_t niters, uint32_t *out) {
#ifdef HA_STAMPS
  ha::ha_stamp_smem[threadIdx.x] = 0;
  __syncwarp();
  unsigned long long sum = 0, nfail = 0;
  throughput_thread<false>(threadIdx.x, nbytes, 1, niters, sum, nfail);
  __syncwarp();
  for (uint32_t i = threadIdx.x; i < ha::kStampBytes / 4; i += 32) out[i] = ha::ha_stamp_smem[i];
#endif
}

// Totals of the mapped-transfer loop while its blocks run; the last block
// to finish takes them (and clears them for the next launch).
__device__ unsigned long long g_mapped_acc[2];
__device__ unsigned int g_mapped_done;

// The same loop for the host-buffer form with mapped transfers: sizes is a
// device view of pinned host memory (read in place over the bus, NULL for a
// fixed nbytes), and the block that finishes last stores the totals into
// d_out and into h_out, a device view of the pinned host result.
__global__ void ha_throughput_mapped_k(const uint32_t *sizes, uint32_t nbytes, uint32_t n,
                                       uint32_t nallocs, uint32_t niters,
                                       unsigned long long *d_out, unsigned long long *h_out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long sum = 0, nfail = 0;
  if (i < n) throughput_thread<false>(i, sizes ? sizes[i] : nbytes, nallocs, niters, sum, nfail);
  block_add2(sum, nfail, g_mapped_acc, g_mapped_acc + 1);  // thread 0 adds the block's totals
  if (threadIdx.x == 0) {
    __threadfence();
    if (atomicAdd(&g_mapped_done, 1u) == gridDim.x - 1) {
      __threadfence();
      const unsigned long long cs = atomicExch(&g_mapped_acc[0], 0ull);
      const unsigned long long nf = atomicExch(&g_mapped_acc[1], 0ull);
      g_mapped_done = 0;
      d_out[0] = cs;
      d_out[1] = nf;
      h_out[0] = cs;
      h_out[1] = nf;
    }
  }
}

// ---- phase workload ----------------------------------------------------------
//
// Every decision (allocate this slot? which size? free it?) and every
// payload word comes from a counter-based hash of (seed, thread, slot,
// round), so a host can replay the whole run and predict its checksums
// whatever the device scheduling was.

// "lowbias32" integer finaliser (C. Wellons, public domain hash prospector)
__device__ __forceinline__ uint32_t mix32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}
__device__ __forceinline__ uint32_t slot_hash(uint32_t seed, uint32_t i, uint32_t s,
                                              uint32_t round) {
  return mix32(((i << 2) | s) ^ (round * 0x9E3779B9u) ^ seed);
}

// A block's payload: the words base, base+1, ... over its sz bytes (sz a
// multiple of 8), written with 16-byte stores where the block's address and
// size allow them (every size but 24 B); returns the sum of the words.  The
// stores are streaming (evict-first): a payload is read back only rounds
// later, and left at normal priority the 1.2 GB of payload sectors an
// allocation round writes push the allocator's metadata out of L2.
__device__ __forceinline__ unsigned long long write_pattern(void *p, uint32_t sz,
                                                            uint32_t base) {
  unsigned long long sum = 0;
  if ((((uintptr_t)p | sz) & 15u) == 0) {
    uint4 *q = reinterpret_cast<uint4 *>(p);
    for (uint32_t w = 0; w < sz / 16; w++) {
      const uint32_t a = base + 4 * w;
      const uint4 v = make_uint4(a, a + 1, a + 2, a + 3);  // 32-bit words, wrapping
      __stcs(q + w, v);
      sum += (unsigned long long)v.x + v.y + v.z + v.w;
    }
  } else {
    uint2 *q = reinterpret_cast<uint2 *>(p);
    for (uint32_t w = 0; w < sz / 8; w++) {
      const uint32_t a = base + 2 * w;
      const uint2 v = make_uint2(a, a + 1);
      __stcs(q + w, v);
      sum += (unsigned long long)v.x + v.y;
    }
  }
  return sum;
}

// The sum of a block's words, read with 16-byte loads where possible and
// eight loads in flight: the read-back waits on DRAM about once per block.
// The loads are streaming too: this is the payload's last use.
__device__ __forceinline__ unsigned long long read_sum(const void *p, uint32_t sz) {
  unsigned long long sum = 0;
  if ((((uintptr_t)p | sz) & 15u) == 0) {
    const uint4 *q = reinterpret_cast<const uint4 *>(p);
#pragma unroll 8
    for (uint32_t w = 0; w < sz / 16; w++) {
      const uint4 v = __ldcs(q + w);
      sum += (unsigned long long)v.x + v.y + v.z + v.w;
    }
  } else {
    const uint2 *q = reinterpret_cast<const uint2 *>(p);
#pragma unroll 8
    for (uint32_t w = 0; w < sz / 8; w++) {
      const uint2 v = __ldcs(q + w);
      sum += (unsigned long long)v.x + v.y;
    }
  }
  return sum;
}

// Phase accumulators: [0] slots filled after the round, [1] failed
// allocations, [2] sum of words written, [3] sum of words read back,
// [4] allocations, [5] frees.
//
// One allocation round: every empty slot of every thread is filled with
// probability thr / 2^32 by a block of a size drawn from size_set, whose
// words are written with base, base+1, ...
__global__ void ha_phase_alloc_k(uint32_t n, uint32_t nslots, uint32_t seed, uint32_t round,
                                 uint32_t thr, const uint32_t *size_set, uint32_t nsizes,
                                 void **slots, uint32_t *slot_sz, unsigned long long *acc) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long filled = 0, nfail = 0, wsum = 0, nmal = 0;
  if (i < n) {
    for (uint32_t s = 0; s < nslots; s++) {
      const size_t k = (size_t)s * n + i;
      void *p = slots[k];
      if (!p) {
        const uint32_t h = slot_hash(seed, i, s, round);
        if (h < thr) {
          const uint32_t sz = size_set[mix32(h ^ 0xA5A5A5A5u) % nsizes];
          p = hamalloc(sz);
          if (p) {
            wsum += write_pattern(p, sz, mix32(h ^ 0x5EED5EEDu));
            slots[k] = p;
            slot_sz[k] = sz;
            nmal++;
          } else {
            nfail++;
          }
        }
      }
      if (p) filled++;
    }
  }
  block_add2(filled, nfail, acc, acc + 1);
  block_add2(wsum, nmal, acc + 2, acc + 4);
}

// One free round: every live block is read back and freed with
// probability thr / 2^32 (always when thr is 0xffffffff).
__global__ void ha_phase_free_k(uint32_t n, uint32_t nslots, uint32_t seed, uint32_t round,
                                uint32_t thr, void **slots, const uint32_t *slot_sz,
                                unsigned long long *acc) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long filled = 0, rsum = 0, nfree = 0;
  if (i < n) {
    for (uint32_t s = 0; s < nslots; s++) {
      const size_t k = (size_t)s * n + i;
      void *p = slots[k];
      if (!p) continue;
      if (thr == 0xffffffffu || slot_hash(seed, i, s, round) < thr) {
        rsum += read_sum(p, slot_sz[k]);
        hafree(p);
        slots[k] = nullptr;
        nfree++;
      } else {
        filled++;
      }
    }
  }
  block_add2(filled, rsum, acc, acc + 3);
  block_add2(nfree, 0, acc + 5, acc + 5);
}

// ---- phase workload, the reference's own form -------------------------------
//
// halloc tst/perf/phase-throughput/phase-throughput.cu:17-48 and free_rest_k
// (tst/common/common.h:403-412), with the reference's per-thread generator
// and draws (tst/common/common.h:80-117, 209-235): Thomas Wang's 32-bit
// integer hash applied to the thread's state, an integer in [a, b] from the
// low 24 bits modulo the range, a probability test against a 20-bit
// fraction.  The same draws in the same order give the same decisions.

__device__ __forceinline__ uint32_t wang_next(uint32_t &st) {
  uint32_t x = st;
  x = (x ^ 61u) ^ (x >> 16);
  x *= 9u;
  x ^= x >> 4;
  x *= 0x27d4eb2du;
  x ^= x >> 15;
  st = x;
  return x;
}
__device__ __forceinline__ uint32_t draw_in(uint32_t &st, uint32_t a, uint32_t b) {
  return a + (wang_next(st) & 0x00ffffffu) % (b - a + 1);
}
__device__ __forceinline__ bool draw_bool(uint32_t &st, float p) {
  if (0.0f < p && p < 1.0f)
    return (1.0f / (1024.0f * 1024.0f)) * (float)draw_in(st, 0, (1u << 20) - 1) <= p;
  return p >= 1.0f;
}

struct PhaseRefProbs {
  float p[4];  // [phase * 2 + holding]
};

// per-call cycles of the timed form: [0] hamalloc, [1] hafree
struct LatAcc {
  unsigned long long n[2], sum[2], min[2], max[2];
  unsigned long long hist[2][ha::kHistBuckets];
};

// acc: [0] mallocs, [1] frees, [2] failed mallocs, [3] bytes of successful mallocs.
// kTime: clock64() around every hamalloc / hafree call (the reference's
// phase-latency kernel, tst/perf/phase-latency/phase-latency.cu:18-56), the
// cycles filed in block-local histograms and added to *lat at the end.
template <bool kTime>
__global__ void ha_phase_ref_k(uint32_t n, uint32_t nallocs, uint32_t step0, uint32_t niters,
                               PhaseRefProbs pr, uint32_t smin, uint32_t smax,
                               uint32_t *states, void **slots, uint32_t *ctrs,
                               unsigned long long *acc, int rest, LatAcc *lat) {
  __shared__ unsigned long long s_hist[kTime ? 2 * ha::kHistBuckets : 1];
  __shared__ unsigned long long s_n[2], s_sum[2], s_min[2], s_max[2];
  if (kTime) {
    for (uint32_t k = threadIdx.x; k < 2 * ha::kHistBuckets; k += blockDim.x) s_hist[k] = 0;
    if (threadIdx.x < 2) {
      s_n[threadIdx.x] = s_sum[threadIdx.x] = s_max[threadIdx.x] = 0;
      s_min[threadIdx.x] = ~0ull;
    }
    __syncthreads();
  }
  auto file = [&](int kind, long long t0, long long t1) {
    const unsigned long long c = (unsigned long long)(t1 - t0);
    atomicAdd(&s_hist[kind * ha::kHistBuckets + ha::lat_bucket(c)], 1ull);
    atomicAdd(&s_n[kind], 1ull);
    atomicAdd(&s_sum[kind], c);
    atomicMin(&s_min[kind], c);
    atomicMax(&s_max[kind], c);
  };
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long nmal = 0, nfree = 0, nfail = 0, bytes = 0;
  if (i < n) {
    uint32_t ctr = ctrs[i];
    if (rest) {
      for (uint32_t k = 0; k < ctr; k++) {
        hafree(slots[(size_t)k * n + i]);
        slots[(size_t)k * n + i] = nullptr;
      }
      nfree += ctr;
      ctr = 0;
    } else {
      uint32_t st = states[i];
      for (uint32_t it = 0; it < niters; it++) {
        const uint32_t phase = (step0 + it) & 1u;
        const bool holding = ctr > 0;
        if (!draw_bool(st, pr.p[phase * 2 + (holding ? 1 : 0)])) continue;
        if (!holding) {
          for (uint32_t k = 0; k < nallocs; k++) {
            const uint32_t sz = smin == smax ? smin : draw_in(st, smin, smax);
            const long long t0 = kTime ? clock64() : 0;
            void *p = hamalloc(sz);
            if (kTime) file(0, t0, clock64());
            slots[(size_t)k * n + i] = p;
            if (p) {
              nmal++;
              bytes += sz;
            } else {
              nfail++;
            }
          }
          ctr = nallocs;
        } else {
          for (uint32_t k = 0; k < nallocs; k++) {
            const long long t0 = kTime ? clock64() : 0;
            hafree(slots[(size_t)k * n + i]);
            if (kTime) file(1, t0, clock64());
            slots[(size_t)k * n + i] = nullptr;
          }
          nfree += nallocs;
          ctr = 0;
        }
      }
      states[i] = st;
    }
    ctrs[i] = ctr;
  }
  block_add2(nmal, nfree, acc, acc + 1);
  block_add2(nfail, bytes, acc + 2, acc + 3);
  if (kTime) {
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < 2 * ha::kHistBuckets; k += blockDim.x)
      if (s_hist[k]) atomicAdd(&lat->hist[k / ha::kHistBuckets][k % ha::kHistBuckets], s_hist[k]);
    if (threadIdx.x < 2 && s_n[threadIdx.x]) {
      atomicAdd(&lat->n[threadIdx.x], s_n[threadIdx.x]);
      atomicAdd(&lat->sum[threadIdx.x], s_sum[threadIdx.x]);
      atomicMin(&lat->min[threadIdx.x], s_min[threadIdx.x]);
      atomicMax(&lat->max[threadIdx.x], s_max[threadIdx.x]);
    }
  }
}

// ---- batched workload ---------------------------------------------------------

// allocation of requests [begin, end): the block carries its request id
__device__ __forceinline__ void batched_malloc_one(uint32_t r, const uint32_t *req_size,
                                                   unsigned long long *req_ptr,
                                                   unsigned long long &nfail,
                                                   unsigned long long &nmal) {
  void *p = hamalloc(req_size[r]);
  req_ptr[r] = (unsigned long long)(uintptr_t)p;
  if (p) {
    *reinterpret_cast<unsigned long long *>(p) = r;
    nmal++;
  } else {
    nfail++;
  }
}

__device__ __forceinline__ void batched_free_req(uint32_t r, unsigned long long *req_ptr,
                                                 unsigned long long &bad,
                                                 unsigned long long &idsum,
                                                 unsigned long long &nfree) {
  void *p = (void *)(uintptr_t)req_ptr[r];
  if (!p) return;
  if (*reinterpret_cast<const unsigned long long *>(p) != r) bad++;
  idsum += r;
  nfree++;
  hafree(p);
  req_ptr[r] = 0;  // a later run (graph replay) starts from all-NULL pointers
}

__device__ __forceinline__ void batched_free_one(uint32_t k, const uint32_t *free_ids,
                                                 unsigned long long *req_ptr,
                                                 unsigned long long &bad,
                                                 unsigned long long &idsum,
                                                 unsigned long long &nfree) {
  batched_free_req(free_ids[k], req_ptr, bad, idsum, nfree);
}

__global__ void ha_bmalloc_k(uint32_t begin, uint32_t end, const uint32_t *req_size,
                             unsigned long long *req_ptr, unsigned long long *acc) {
  const uint32_t r = begin + blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long nfail = 0, nmal = 0;
  if (r < end) batched_malloc_one(r, req_size, req_ptr, nfail, nmal);
  block_add2(nfail, nmal, acc, acc + 3);
}

__global__ void ha_bfree_k(uint32_t begin, uint32_t end, const uint32_t *free_ids,
                           unsigned long long *req_ptr, unsigned long long *acc) {
  const uint32_t k = begin + blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long bad = 0, idsum = 0, nfree = 0;
  if (k < end) batched_free_one(k, free_ids, req_ptr, bad, idsum, nfree);
  block_add2(bad, idsum, acc + 1, acc + 2);
  block_add2(nfree, 0, acc + 4, acc + 4);
}

struct BatchTask {
  uint32_t begin, end;  // range of request ids (malloc) or free_ids slots (free)
  uint32_t step;        // the step (= batch of an allocation task)
  uint32_t is_free;
};

__device__ __forceinline__ uint32_t ld_acquire_u32(const unsigned int *p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u32(unsigned int *p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint64_t now_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Within a block's task, warps take 32 consecutive requests at a time from a
// shared-memory counter: a warp whose allocations were quick takes the next
// 32, so the block's barrier at the end of the task waits for at most one
// slow chunk rather than for the slowest of each thread's fixed share.
// -DHA_BPERSIST_CHUNKS=0 gives every thread the fixed strided share instead.
#ifndef HA_BPERSIST_CHUNKS
#define HA_BPERSIST_CHUNKS 1
#endif
template <typename F>
__device__ __forceinline__ void for_task_items(uint32_t begin, uint32_t end, uint32_t *next,
                                               F &&f) {
#if HA_BPERSIST_CHUNKS
  // the block size is a multiple of 32 (checked by the host), so every warp
  // is whole
  const uint32_t lane = threadIdx.x & 31u, n = end - begin;
  for (;;) {
    uint32_t c = 0;
    if (lane == 0) c = atomicAdd(next, 32u);
    c = __shfl_sync(0xffffffffu, c, 0);
    if (c >= n) break;
    if (c + lane < n) f(begin + c + lane);
  }
#else
  (void)next;
  for (uint32_t r = begin + threadIdx.x; r < end; r += blockDim.x) f(r);
#endif
}

// A free task of step s frees blocks of batches before s.  Those of batches
// before s - 1 were allocated long before (the block waits for them, which
// seldom takes long); each block of batch s - 1 waits only for the
// allocation task that made it, so a free task need not wait for the whole
// of the batch just before it.  -DHA_BPERSIST_ITEM_WAIT=0 makes every free
// task wait for all of batch s - 1 instead.
#ifndef HA_BPERSIST_ITEM_WAIT
#define HA_BPERSIST_ITEM_WAIT 1
#endif

// Persistent form.  ctl[0] = next task; ctl[1 + b] = finished allocation
// tasks of batch b; btasks[b] = allocation tasks of batch b; bdep[b] = (first
// request, first task index) of batch b; tdone[t] = 1 once allocation task t
// is finished; `items` = requests per task (the last task of a batch may
// hold fewer).  Each block remembers the batches it has already seen
// complete (tasks reach a block in step order).
__global__ void ha_bpersist_k(const BatchTask *tasks, uint32_t ntasks, const uint32_t *btasks,
                              const uint2 *bdep, uint32_t items,
                              const uint32_t *req_size, unsigned long long *req_ptr,
                              const uint32_t *free_ids, unsigned int *ctl,
                              unsigned int *tdone, unsigned long long *acc) {
  __shared__ uint32_t s_task, s_done_below, s_next;
  unsigned long long nfail = 0, nmal = 0, bad = 0, idsum = 0, nfree = 0, late = 0;
  if (threadIdx.x == 0) s_done_below = 0;
  for (;;) {
    __syncthreads();  // everyone has read s_task and is done with s_next
    if (threadIdx.x == 0) {
      s_task = atomicAdd(&ctl[0], 1u);
      s_next = 0;
    }
    __syncthreads();
    const uint32_t t = s_task;
    if (t >= ntasks) break;
    const BatchTask tk = tasks[t];
    if (tk.is_free) {
      if (threadIdx.x == 0) {
        // every allocation task of those batches was dequeued earlier by a
        // running block, so each wait ends
        const uint64_t limit = now_ns() + 2000000000ull;
        uint32_t b = s_done_below;
        while (b < tk.step) {
          if (ld_acquire_u32(&ctl[1 + b]) >= btasks[b]) {
            b++;
            continue;
          }
          if (HA_BPERSIST_ITEM_WAIT && b + 1 == tk.step) break;  // per block, below
          if (now_ns() > limit) {
            late++;
            break;
          }
          __nanosleep(128);
        }
        s_done_below = b;
      }
      __syncthreads();
      // blocks of batch step - 1, when it is not known to be complete: the
      // allocation task of each is tasks dep_task .. dep_task + dep_n - 1
      uint32_t dep_begin = 0xffffffffu, dep_task = 0, dep_n = 0;
      if (HA_BPERSIST_ITEM_WAIT && s_done_below + 1 == tk.step) {
        const uint2 d = bdep[tk.step - 1];
        dep_begin = d.x;
        dep_task = d.y;
        dep_n = btasks[tk.step - 1];
      }
      for_task_items(tk.begin, tk.end, &s_next, [&](uint32_t k) {
        const uint32_t r = free_ids[k];
        if (r >= dep_begin) {
          const uint32_t t = (r - dep_begin) / items;
          if (t < dep_n && !ld_acquire_u32(&tdone[dep_task + t])) {
            const uint64_t limit = now_ns() + 2000000000ull;
            while (!ld_acquire_u32(&tdone[dep_task + t])) {
              if (now_ns() > limit) {
                late++;
                break;
              }
              __nanosleep(64);
            }
          }
        }
        batched_free_req(r, req_ptr, bad, idsum, nfree);
      });
    } else {
      for_task_items(tk.begin, tk.end, &s_next, [&](uint32_t r) {
        batched_malloc_one(r, req_size, req_ptr, nfail, nmal);
      });
      __syncthreads();
      if (threadIdx.x == 0) {
        __threadfence();  // this block's req_ptr and payload writes before the flags
        st_relaxed_u32(&tdone[t], 1u);
        atomicAdd(&ctl[1 + tk.step], 1u);
      }
    }
  }
  block_add2(nfail, nmal, acc, acc + 3);
  block_add2(bad, idsum, acc + 1, acc + 2);
  block_add2(nfree, late, acc + 4, acc + 5);
}

// ---- batched persistent form that allocates nothing ----------------------------
//
// Some callers cannot call cudaMalloc: code that has handed all device
// memory to its own pool (cudaMalloc would fail), and latency-bound serving
// loops that must not call cudaMalloc/cudaFree because those calls
// synchronise the device and stall every other stream.  For them the
// persistent form below keeps its scratch -- the task table, the per-batch
// task counts and first tasks, the queue and completion counters, and the
// per-task done flags -- in one fixed array in device memory instead.  Every
// GPU that loads this library holds the array (about 1.3 MiB) until the
// process exits.

constexpr uint32_t kNoAllocMaxTasks = 65536;
constexpr uint32_t kNoAllocMaxBatches = 1024;
constexpr size_t kNaTasksOff = 0;
constexpr size_t kNaBtasksOff = kNaTasksOff + sizeof(BatchTask) * kNoAllocMaxTasks;
constexpr size_t kNaCtlOff = kNaBtasksOff + 4 * 1280;
constexpr size_t kNaBdepOff = kNaCtlOff + 4 * 1280;
constexpr size_t kNaDoneOff = kNaBdepOff + sizeof(uint2) * 1280;
constexpr size_t kNoAllocScratchBytes = kNaDoneOff + 4 * kNoAllocMaxTasks;
static_assert(kNoAllocMaxBatches + 2 <= 1280, "scratch regions hold nbatch + 2 words");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

// The plan's step offsets, passed by value as a kernel parameter (8 KiB, under
// the 32 KiB parameter limit): the launch copies them, so the caller's host
// arrays are free again as soon as the call returns.
struct NoAllocOffsets {
  uint32_t batch_start[kNoAllocMaxBatches + 1];
  uint32_t free_start[kNoAllocMaxBatches + 2];
};

// Builds the task table of ha_batched_prepare_c (the same order: each step's
// allocation chunks, then its free chunks) and the per-batch first request
// and first task in the scratch array, and clears the queue and completion
// counters (the host clears the done flags).  The host has checked that the
// offsets never decrease and that the table has at most kNoAllocMaxTasks
// entries; indices are 64-bit and the writes stop at the limit regardless.
__global__ void ha_noalloc_tasks_k(unsigned char *scratch, uint32_t nbatch, uint32_t items,
                                   const NoAllocOffsets off) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  BatchTask *tasks = reinterpret_cast<BatchTask *>(scratch + kNaTasksOff);
  uint32_t *btasks = reinterpret_cast<uint32_t *>(scratch + kNaBtasksOff);
  unsigned int *ctl = reinterpret_cast<unsigned int *>(scratch + kNaCtlOff);
  uint2 *bdep = reinterpret_cast<uint2 *>(scratch + kNaBdepOff);
  uint32_t n = 0;
  for (uint32_t st = 0; st <= nbatch; st++) {
    ctl[1 + st] = 0;
    if (st < nbatch) {
      btasks[st] = 0;
      bdep[st] = make_uint2(off.batch_start[st], n);
      const uint64_t b1 = off.batch_start[st + 1];
      for (uint64_t r = off.batch_start[st]; r < b1 && n < kNoAllocMaxTasks; r += items) {
        tasks[n++] = {(uint32_t)r, (uint32_t)(r + items < b1 ? r + items : b1), st, 0u};
        btasks[st]++;
      }
    }
    const uint64_t f1 = off.free_start[st + 1];
    for (uint64_t k = off.free_start[st]; k < f1 && n < kNoAllocMaxTasks; k += items)
      tasks[n++] = {(uint32_t)k, (uint32_t)(k + items < f1 ? k + items : f1), st, 1u};
  }
  ctl[0] = 0;
}

// ---- random-graph build -----------------------------------------------------
//
// Vertex u draws its out-degree d from a Poisson CDF given as 32-bit
// thresholds (d = number of thresholds <= mix32(u ^ seed)), and its k-th
// neighbour as mix32(mix32(u ^ seed ^ 0xABCDEF01) + k * 0x9E3779B9) mod n.
// One thread per vertex appends its neighbours to an int32 array from
// hamalloc, starting at capacity 2 and doubling (malloc new, copy, free old).

__device__ __forceinline__ uint32_t graph_degree(uint32_t u, uint32_t seed, const uint32_t *cdf,
                                                 uint32_t ncdf) {
  const uint32_t h = mix32(u ^ seed);
  uint32_t d = 0;
  while (d < ncdf && cdf[d] <= h) d++;
  return d;
}
__device__ __forceinline__ uint32_t graph_neighbour(uint32_t u, uint32_t k, uint32_t seed,
                                                    uint32_t n) {
  return mix32(mix32(u ^ seed ^ 0xABCDEF01u) + k * 0x9E3779B9u) % n;
}

// acc: [0] failed allocations, [1] reallocations (doublings), [2] edges
__global__ void ha_graph_build_k(uint32_t n, uint32_t seed, const uint32_t *cdf, uint32_t ncdf,
                                 unsigned long long *arr, uint32_t *deg,
                                 unsigned long long *acc) {
  const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long nfail = 0, ngrow = 0, nedge = 0;
  if (u < n) {
    const uint32_t d = graph_degree(u, seed, cdf, ncdf);
    uint32_t cap = 2, cnt = 0;
    uint32_t *a = (uint32_t *)hamalloc(cap * sizeof(uint32_t));
    if (!a) nfail++;
    for (uint32_t k = 0; k < d && a; k++) {
      if (cnt == cap) {
        uint32_t *b = (uint32_t *)hamalloc(2 * cap * sizeof(uint32_t));
        if (!b) {
          nfail++;
          break;
        }
        for (uint32_t j = 0; j < cnt; j++) b[j] = a[j];
        hafree(a);
        a = b;
        cap *= 2;
        ngrow++;
      }
      a[cnt++] = graph_neighbour(u, k, seed, n);
    }
    arr[u] = (unsigned long long)(uintptr_t)a;
    deg[u] = cnt;
    nedge = cnt;
  }
  block_add2(nfail, ngrow, acc, acc + 1);
  block_add2(nedge, 0, acc + 2, acc + 2);
}

// Copies each vertex's array into CSR columns at offsets[u] and frees it.
__global__ void ha_graph_gather_k(uint32_t n, unsigned long long *arr, const uint32_t *deg,
                                  const unsigned long long *offsets, uint32_t *cols) {
  const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
  if (u >= n) return;
  uint32_t *a = (uint32_t *)(uintptr_t)arr[u];
  if (!a) return;
  const unsigned long long o = offsets[u];
  for (uint32_t k = 0; k < deg[u]; k++) cols[o + k] = a[k];
  hafree(a);
  arr[u] = 0;
}

// serial replay on one thread
__global__ void ha_trace_k(const int64_t *ops, int64_t n, int64_t *out) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  for (int64_t i = 0; i < n; i++) {
    const int64_t op = ops[i];
    if (op >= 0) {
      out[i] = (int64_t)(uintptr_t)hamalloc((size_t)op);
    } else {
      hafree((void *)(uintptr_t)out[-(op + 1)]);
      out[i] = 0;
    }
  }
}

// distinct-address 32-bit atomic OR throughput; thread t works on word
// (t mod nwords) x stride (stride 8: every thread on its own 32-byte sector)
__global__ void ha_atomic_peak_k(uint32_t *buf, uint32_t nwords, uint32_t stride,
                                 uint32_t reps, int returning) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t *w = &buf[(size_t)(t % nwords) * stride];
  if (returning) {
    uint32_t acc0 = 0, acc1 = 0;
    for (uint32_t r = 0; r < reps; r += 2) {
      acc0 ^= atomicOr(w, 1u << (r & 31));
      acc1 ^= atomicOr(w, 2u << (r & 30));
    }
    if ((acc0 ^ acc1) == 0x9e3779b9u) buf[0] = acc0;  // keeps the results live
  } else {
    for (uint32_t r = 0; r < reps; r++) atomicOr(w, 1u << (r & 31));
  }
}

// ---- C ABI ---------------------------------------------------------------

extern "C" int ha_malloc_batch_c(const uint32_t *sizes, uint32_t nthreads, uint32_t nallocs,
                                 void **ptrs, int tag, void *stream) {
  if (!sizes || !ptrs || nallocs == 0) return HA_EINVAL;
  if (nthreads == 0) return HA_OK;
  ha_malloc_batch_k<<<blocks_for(nthreads, 128), 128, 0, as_stream(stream)>>>(
      sizes, nthreads, nallocs, ptrs, tag);
  return launch_status();
}

extern "C" int ha_free_batch_c(void *const *ptrs, uint32_t nthreads, uint32_t nallocs,
                               void *stream) {
  if (!ptrs || nallocs == 0) return HA_EINVAL;
  if (nthreads == 0) return HA_OK;
  ha_free_batch_k<<<blocks_for(nthreads, 128), 128, 0, as_stream(stream)>>>(ptrs, nthreads,
                                                                          nallocs);
  return launch_status();
}

static int throughput(bool cuda_heap, const uint32_t *sizes, uint32_t nbytes,
                      uint32_t nthreads, uint32_t block, uint32_t nallocs, uint32_t niters,
                      uint64_t *out, void *stream) {
  if (!out || block == 0 || block > 1024 || nallocs == 0 ||
      nallocs > kMaxAllocsPerThread)
    return HA_EINVAL;
  if (nthreads == 0 || niters == 0) return HA_OK;
  const uint32_t grid = blocks_for(nthreads, block);
  unsigned long long *o = reinterpret_cast<unsigned long long *>(out);
  if (cuda_heap)
    ha_throughput_k<true><<<grid, block, 0, as_stream(stream)>>>(sizes, nbytes, nthreads,
                                                               nallocs, niters, o);
  else
    ha_throughput_k<false><<<grid, block, 0, as_stream(stream)>>>(sizes, nbytes, nthreads,
                                                                nallocs, niters, o);
  return launch_status();
}

extern "C" int ha_throughput_c(const uint32_t *sizes, uint32_t nbytes, uint32_t nthreads,
                               uint32_t block, uint32_t nallocs, uint32_t niters,
                               uint64_t *out, void *stream) {
  return throughput(false, sizes, nbytes, nthreads, block, nallocs, niters, out, stream);
}

extern "C" int ha_cuda_throughput_c(const uint32_t *sizes, uint32_t nbytes, uint32_t nthreads,
                                    uint32_t block, uint32_t nallocs, uint32_t niters,
                                    uint64_t *out, void *stream) {
  return throughput(true, sizes, nbytes, nthreads, block, nallocs, niters, out, stream);
}

// The host-buffer form moves its bytes one of two ways.  Mapped: when the
// device can address both host buffers (pinned memory), one kernel reads the
// sizes in place and its last block stores the totals into the host result;
// no copy-engine transfer, no clearing step.  Copy: one CUDA graph (sizes
// in, counters cleared, the loop, results out), built on the first call and
// kept while the arguments stay the same: one launch per call instead of
// four.  The cached graph and the mapped form's totals are one per process
// and device: calls from several host threads must not overlap.
struct HostLoopGraph {
  int dev;
  const uint32_t *h_sizes;
  uint32_t *d_sizes;
  uint32_t nbytes, nthreads, block, nallocs, niters;
  uint64_t *d_out, *h_out;
  cudaGraph_t graph;
  cudaGraphExec_t exec;
};
static HostLoopGraph g_host_loop = {};

static bool same_host_loop(const HostLoopGraph &a, const HostLoopGraph &b) {
  return a.dev == b.dev && a.h_sizes == b.h_sizes && a.d_sizes == b.d_sizes &&
         a.nbytes == b.nbytes && a.nthreads == b.nthreads && a.block == b.block &&
         a.nallocs == b.nallocs && a.niters == b.niters && a.d_out == b.d_out &&
         a.h_out == b.h_out;
}

static int build_host_loop(HostLoopGraph &k) {
  cudaGraph_t g = nullptr;
  if (cudaGraphCreate(&g, 0) != cudaSuccess) return HA_ECUDA;
  cudaGraphNode_t deps[2];
  size_t ndeps = 0;
  bool ok = true;
  if (k.h_sizes)
    ok = cudaGraphAddMemcpyNode1D(&deps[ndeps++], g, nullptr, 0, k.d_sizes, k.h_sizes,
                                  (size_t)k.nthreads * 4, cudaMemcpyHostToDevice) ==
         cudaSuccess;
  cudaMemsetParams ms = {};
  ms.dst = k.d_out;
  ms.value = 0;
  ms.elementSize = 4;
  ms.width = 4;  // two 64-bit counters
  ms.height = 1;
  ms.pitch = 0;
  ok = ok && cudaGraphAddMemsetNode(&deps[ndeps++], g, nullptr, 0, &ms) == cudaSuccess;
  const uint32_t *sizes = k.h_sizes ? k.d_sizes : nullptr;
  unsigned long long *o = reinterpret_cast<unsigned long long *>(k.d_out);
  void *args[] = {(void *)&sizes, (void *)&k.nbytes, (void *)&k.nthreads, (void *)&k.nallocs,
                  (void *)&k.niters, (void *)&o};
  cudaKernelNodeParams kp = {};
  kp.func = reinterpret_cast<void *>(ha_throughput_k<false>);
  kp.gridDim = dim3(blocks_for(k.nthreads, k.block));
  kp.blockDim = dim3(k.block);
  kp.sharedMemBytes = 0;
  kp.kernelParams = args;
  cudaGraphNode_t kn = nullptr, out = nullptr;
  ok = ok && cudaGraphAddKernelNode(&kn, g, deps, ndeps, &kp) == cudaSuccess;
  ok = ok && cudaGraphAddMemcpyNode1D(&out, g, &kn, 1, k.h_out, k.d_out,
                                      2 * sizeof(uint64_t), cudaMemcpyDeviceToHost) ==
                 cudaSuccess;
  cudaGraphExec_t exec = nullptr;
  ok = ok && cudaGraphInstantiate(&exec, g, 0) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    cudaGraphDestroy(g);
    return HA_ECUDA;
  }
  k.graph = g;
  k.exec = exec;
  return HA_OK;
}

// Device view of a host buffer, or nullptr when the device cannot address it
// (pageable memory).  Asked on every call: a cached answer would outlive a
// buffer freed and replaced by pageable memory at the same address.
static const void *mapped_view(const void *h) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, h) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  return a.type == cudaMemoryTypeHost ? a.devicePointer : nullptr;
}

extern "C" int ha_throughput_host_ex_c(const uint32_t *h_sizes, uint32_t *d_sizes,
                                       uint32_t nbytes, uint32_t nthreads, uint32_t block,
                                       uint32_t nallocs, uint32_t niters, uint64_t *d_out,
                                       uint64_t *h_out, uint32_t transfer, void *stream) {
  if (!d_out || !h_out || block == 0 || block > 1024 || nallocs == 0 ||
      nallocs > kMaxAllocsPerThread || transfer > HA_XFER_MAPPED)
    return HA_EINVAL;
  if (nthreads == 0 || niters == 0) return HA_OK;
  cudaStream_t s = as_stream(stream);
  if (transfer != HA_XFER_COPY) {
    auto *mo = static_cast<unsigned long long *>(const_cast<void *>(mapped_view(h_out)));
    const auto *ms = h_sizes ? static_cast<const uint32_t *>(mapped_view(h_sizes)) : nullptr;
    if (mo && (!h_sizes || ms)) {
      ha_throughput_mapped_k<<<blocks_for(nthreads, block), block, 0, s>>>(
          ms, nbytes, nthreads, nallocs, niters, reinterpret_cast<unsigned long long *>(d_out),
          mo);
      if (launch_status() != HA_OK || cudaStreamSynchronize(s) != cudaSuccess) return HA_ECUDA;
      return HA_OK;
    }
    if (transfer == HA_XFER_MAPPED) return HA_EINVAL;
  }
  if (h_sizes && !d_sizes) return HA_EINVAL;
  HostLoopGraph want = {};
  if (cudaGetDevice(&want.dev) != cudaSuccess) return HA_ECUDA;
  want.h_sizes = h_sizes;
  want.d_sizes = d_sizes;
  want.nbytes = nbytes;
  want.nthreads = nthreads;
  want.block = block;
  want.nallocs = nallocs;
  want.niters = niters;
  want.d_out = d_out;
  want.h_out = h_out;
  if (!g_host_loop.exec || !same_host_loop(g_host_loop, want)) {
    if (g_host_loop.exec) {
      cudaGraphExecDestroy(g_host_loop.exec);
      cudaGraphDestroy(g_host_loop.graph);
      g_host_loop.exec = nullptr;
    }
    if (build_host_loop(want) != HA_OK) return HA_ECUDA;
    g_host_loop = want;
  }
  if (cudaGraphLaunch(g_host_loop.exec, s) != cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return HA_ECUDA;
  return HA_OK;
}

extern "C" int ha_throughput_host_c(const uint32_t *h_sizes, uint32_t *d_sizes,
                                    uint32_t nbytes, uint32_t nthreads, uint32_t block,
                                    uint32_t nallocs, uint32_t niters, uint64_t *d_out,
                                    uint64_t *h_out, void *stream) {
  return ha_throughput_host_ex_c(h_sizes, d_sizes, nbytes, nthreads, block, nallocs, niters,
                                 d_out, h_out, HA_XFER_AUTO, stream);
}

extern "C" int ha_phase_round_c(int kind, uint32_t nthreads, uint32_t nslots, uint32_t seed,
                                uint32_t round, uint32_t thr, const uint32_t *size_set,
                                uint32_t nsizes, void **slots, uint32_t *slot_sz, uint64_t *acc,
                                void *stream) {
  if (!slots || !slot_sz || !acc || nslots == 0 || nslots > kMaxAllocsPerThread ||
      (kind == 0 && (!size_set || nsizes == 0)) || (kind != 0 && kind != 1))
    return HA_EINVAL;
  if (nthreads == 0) return HA_OK;
  cudaStream_t s = as_stream(stream);
  if (cudaMemsetAsync(acc, 0, sizeof(uint64_t), s) != cudaSuccess) return HA_ECUDA;
  unsigned long long *a = reinterpret_cast<unsigned long long *>(acc);
  const uint32_t grid = blocks_for(nthreads, 128);
  if (kind == 0)
    ha_phase_alloc_k<<<grid, 128, 0, s>>>(nthreads, nslots, seed, round, thr, size_set, nsizes,
                                          slots, slot_sz, a);
  else
    ha_phase_free_k<<<grid, 128, 0, s>>>(nthreads, nslots, seed, round, thr, slots, slot_sz, a);
  return launch_status();
}

extern "C" int ha_phase_run_c(uint32_t nthreads, uint32_t nslots, uint32_t seed,
                              uint32_t periods, uint32_t thr_alloc, uint32_t thr_free,
                              uint64_t target_filled, uint32_t max_rounds,
                              const uint32_t *size_set, uint32_t nsizes, void **slots,
                              uint32_t *slot_sz, uint64_t *acc, ha_phase_result_t *res,
                              void *stream) {
  if (!res || !acc) return HA_EINVAL;
  cudaStream_t s = as_stream(stream);
  memset(res, 0, sizeof(*res));
  if (cudaMemsetAsync(acc, 0, 6 * sizeof(uint64_t), s) != cudaSuccess) return HA_ECUDA;
  cudaEvent_t e0, e1;
  if (cudaEventCreate(&e0) != cudaSuccess) return HA_ECUDA;
  if (cudaEventCreate(&e1) != cudaSuccess) {
    cudaEventDestroy(e0);
    return HA_ECUDA;
  }
  int rc = HA_OK;
  uint32_t round = 0;
  auto run = [&](int kind, uint32_t thr) -> int {
    if (cudaEventRecord(e0, s) != cudaSuccess) return HA_ECUDA;
    int r = ha_phase_round_c(kind, nthreads, nslots, seed, round++, thr, size_set, nsizes,
                             slots, slot_sz, acc, stream);
    if (r) return r;
    float ms = 0.f;
    if (cudaEventRecord(e1, s) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess ||
        cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess)
      return HA_ECUDA;
    res->kernel_ms += ms;
    if (kind == 0)
      res->alloc_rounds++;
    else
      res->free_rounds++;
    return cudaMemcpy(&res->filled, acc, sizeof(uint64_t), cudaMemcpyDeviceToHost) ==
                   cudaSuccess
               ? HA_OK
               : HA_ECUDA;
  };
  for (uint32_t per = 0; per < periods && rc == HA_OK; per++) {
    for (uint32_t r = 0; r < max_rounds && rc == HA_OK; r++) {
      rc = run(0, thr_alloc);
      if (rc == HA_OK && res->filled >= target_filled) break;
    }
    if (rc == HA_OK) rc = run(1, thr_free);
  }
  if (rc == HA_OK) rc = run(1, 0xffffffffu);  // the rest, as in the reference's free_rest_k
  if (rc == HA_OK &&
      cudaMemcpy(res->acc, acc, 6 * sizeof(uint64_t), cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = HA_ECUDA;
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return rc;
}

extern "C" int ha_phase_ref_step_c(uint32_t nthreads, uint32_t nallocs, uint32_t itry,
                                   uint32_t niters, const float *probs, uint32_t smin,
                                   uint32_t smax, uint32_t *states, void **slots,
                                   uint32_t *ctrs, uint64_t *acc, int rest, void *stream) {
  if (!probs || !states || !slots || !ctrs || !acc || nallocs == 0 ||
      nallocs > kMaxAllocsPerThread || smin == 0 || smin > smax)
    return HA_EINVAL;
  if (nthreads == 0) return HA_OK;
  PhaseRefProbs pr;
  for (int k = 0; k < 4; k++) pr.p[k] = probs[k];
  const uint64_t step0 = (uint64_t)itry * niters;
  ha_phase_ref_k<false><<<blocks_for(nthreads, 128), 128, 0, as_stream(stream)>>>(
      nthreads, nallocs, (uint32_t)step0, niters, pr, smin, smax, states, slots, ctrs,
      reinterpret_cast<unsigned long long *>(acc), rest, nullptr);
  return launch_status();
}

extern "C" int ha_phase_ref_latency_c(uint32_t nthreads, uint32_t nallocs, uint32_t ntries,
                                      uint32_t niters, const float *probs, uint32_t smin,
                                      uint32_t smax, uint32_t *states, void **slots,
                                      uint32_t *ctrs, uint64_t *acc, ha_latency_stats_t *out,
                                      void *stream) {
  if (!out || !acc || !probs || !states || !slots || !ctrs || nallocs == 0 ||
      nallocs > kMaxAllocsPerThread || smin == 0 || smin > smax)
    return HA_EINVAL;
  memset(out, 0, 2 * sizeof(*out));
  if (nthreads == 0) return HA_OK;
  cudaStream_t s = as_stream(stream);
  LatAcc *d_lat = nullptr;
  LatAcc *h_lat = new (std::nothrow) LatAcc;
  if (!h_lat) return HA_ECUDA;
  memset(h_lat, 0, sizeof(*h_lat));
  h_lat->min[0] = h_lat->min[1] = ~0ull;
  int rc = HA_OK;
  if (cudaMalloc(&d_lat, sizeof(LatAcc)) != cudaSuccess ||
      cudaMemcpyAsync(d_lat, h_lat, sizeof(LatAcc), cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemsetAsync(acc, 0, 4 * sizeof(uint64_t), s) != cudaSuccess)
    rc = HA_ECUDA;
  PhaseRefProbs pr;
  for (int k = 0; k < 4; k++) pr.p[k] = probs[k];
  for (uint32_t t = 0; t < ntries && rc == HA_OK; t++) {
    ha_phase_ref_k<true><<<blocks_for(nthreads, 128), 128, 0, s>>>(
        nthreads, nallocs, t * niters, niters, pr, smin, smax, states, slots, ctrs,
        reinterpret_cast<unsigned long long *>(acc), 0, d_lat);
    rc = launch_status();
  }
  if (rc == HA_OK)
    rc = ha_phase_ref_step_c(nthreads, nallocs, ntries, niters, probs, smin, smax, states,
                             slots, ctrs, acc, 1, stream);
  if (rc == HA_OK &&
      (cudaMemcpyAsync(h_lat, d_lat, sizeof(LatAcc), cudaMemcpyDeviceToHost, s) !=
           cudaSuccess ||
       cudaStreamSynchronize(s) != cudaSuccess))
    rc = HA_ECUDA;
  if (rc == HA_OK) {
    for (int k = 0; k < 2; k++) {
      out[k].n = h_lat->n[k];
      if (!h_lat->n[k]) continue;
      out[k].min_cycles = (double)h_lat->min[k];
      out[k].max_cycles = (double)h_lat->max[k];
      out[k].avg_cycles = (double)h_lat->sum[k] / (double)h_lat->n[k];
      out[k].p50_cycles = ha::percentile(h_lat->hist[k], 0.50);
      out[k].p99_cycles = ha::percentile(h_lat->hist[k], 0.99);
    }
  }
  cudaFree(d_lat);
  delete h_lat;
  return rc;
}

extern "C" int ha_phase_ref_run_c(uint32_t nthreads, uint32_t nallocs, uint32_t ntries,
                                  uint32_t niters, const float *probs, uint32_t smin,
                                  uint32_t smax, uint32_t *states, void **slots, uint32_t *ctrs,
                                  uint64_t *acc, ha_phase_ref_result_t *res, void *stream) {
  if (!res || !acc) return HA_EINVAL;
  memset(res, 0, sizeof(*res));
  cudaStream_t s = as_stream(stream);
  if (cudaMemsetAsync(acc, 0, 4 * sizeof(uint64_t), s) != cudaSuccess) return HA_ECUDA;
  std::vector<cudaEvent_t> ev;
  int rc = HA_OK;
  for (uint32_t k = 0; k < 2 * (ntries + 1) && rc == HA_OK; k++) {
    cudaEvent_t e;
    if (cudaEventCreate(&e) != cudaSuccess) rc = HA_ECUDA;
    else ev.push_back(e);
  }
  // each launch is also waited for on the host, as halloc's test does, and
  // that wall time kept beside the device time
  for (uint32_t t = 0; t <= ntries && rc == HA_OK; t++) {
    const auto w0 = std::chrono::steady_clock::now();
    if (cudaEventRecord(ev[2 * t], s) != cudaSuccess) {
      rc = HA_ECUDA;
      break;
    }
    rc = ha_phase_ref_step_c(nthreads, nallocs, t, niters, probs, smin, smax, states, slots,
                             ctrs, acc, t == ntries, stream);
    if (rc == HA_OK && cudaEventRecord(ev[2 * t + 1], s) != cudaSuccess) rc = HA_ECUDA;
    if (rc == HA_OK && cudaStreamSynchronize(s) != cudaSuccess) rc = HA_ECUDA;
    res->wall_ms +=
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - w0).count();
  }
  for (uint32_t t = 0; t <= ntries && rc == HA_OK; t++) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, ev[2 * t], ev[2 * t + 1]) != cudaSuccess) {
      rc = HA_ECUDA;
      break;
    }
    res->kernel_ms += ms;
    if (t < ntries && t % 2 == 0)
      res->alloc_phase_ms += ms;
    else
      res->free_phase_ms += ms;
  }
  if (rc == HA_OK &&
      cudaMemcpy(res->acc, acc, 4 * sizeof(uint64_t), cudaMemcpyDeviceToHost) != cudaSuccess)
    rc = HA_ECUDA;
  for (cudaEvent_t e : ev) cudaEventDestroy(e);
  return rc;
}

namespace {
// Checks a plan's step offsets before anything is launched: batch and free
// offsets never decrease and end within nreq.  With task_items != 0 it also
// counts the tasks the persistent form makes of the plan (64-bit, so no
// offset or task size can wrap it).  HA_EINVAL for a malformed plan.
int check_plan_offsets(const ha_batch_plan_t *plan, uint32_t task_items, uint64_t *ntasks) {
  const uint32_t *bs = plan->h_batch_start, *fs = plan->h_free_start;
  for (uint32_t b = 0; b < plan->nbatch; b++)
    if (bs[b + 1] < bs[b]) return HA_EINVAL;
  for (uint32_t st = 0; st <= plan->nbatch; st++)
    if (fs[st + 1] < fs[st]) return HA_EINVAL;
  if (bs[plan->nbatch] > plan->nreq || fs[plan->nbatch + 1] > plan->nreq) return HA_EINVAL;
  if (ntasks && task_items) {
    uint64_t n = 0;
    for (uint32_t st = 0; st <= plan->nbatch; st++) {
      n += ((uint64_t)fs[st + 1] - fs[st] + task_items - 1) / task_items;
      if (st < plan->nbatch) n += ((uint64_t)bs[st + 1] - bs[st] + task_items - 1) / task_items;
    }
    *ntasks = n;
  }
  return HA_OK;
}
}  // namespace

extern "C" int ha_batched_plain_c(const ha_batch_plan_t *plan, uint32_t block, void *stream) {
  if (!plan || !plan->acc || !plan->h_batch_start || !plan->h_free_start || block == 0 ||
      block > 1024 || check_plan_offsets(plan, 0, nullptr) != HA_OK)
    return HA_EINVAL;
  cudaStream_t s = as_stream(stream);
  unsigned long long *acc = reinterpret_cast<unsigned long long *>(plan->acc);
  if (cudaMemsetAsync(acc, 0, 8 * sizeof(uint64_t), s) != cudaSuccess) return HA_ECUDA;
  unsigned long long *rp = reinterpret_cast<unsigned long long *>(plan->req_ptr);
  for (uint32_t st = 0; st <= plan->nbatch; st++) {
    const uint32_t f0 = plan->h_free_start[st], f1 = plan->h_free_start[st + 1];
    if (f1 > f0)
      ha_bfree_k<<<blocks_for(f1 - f0, block), block, 0, s>>>(f0, f1, plan->free_ids, rp, acc);
    if (st < plan->nbatch) {
      const uint32_t b0 = plan->h_batch_start[st], b1 = plan->h_batch_start[st + 1];
      if (b1 > b0)
        ha_bmalloc_k<<<blocks_for(b1 - b0, block), block, 0, s>>>(b0, b1, plan->req_size, rp,
                                                                 acc);
    }
  }
  return launch_status();
}

namespace {
struct Batched {
  ha_batch_plan_t plan;
  BatchTask *tasks;
  uint32_t ntasks;
  uint32_t *btasks;  // allocation tasks per batch
  uint2 *bdep;       // first request and first task index per batch
  unsigned int *ctl; // next task, finished allocation tasks per batch, then a
                     // done flag per task
  uint32_t grid, block, items;
  cudaGraphExec_t exec;
  bool graph;
};

void enqueue_persistent(const Batched *b, cudaStream_t s) {
  unsigned long long *acc = reinterpret_cast<unsigned long long *>(b->plan.acc);
  cudaMemsetAsync(acc, 0, 8 * sizeof(uint64_t), s);
  cudaMemsetAsync(b->ctl, 0, ((size_t)b->plan.nbatch + 1 + b->ntasks) * sizeof(unsigned int),
                  s);
  ha_bpersist_k<<<b->grid, b->block, 0, s>>>(
      b->tasks, b->ntasks, b->btasks, b->bdep, b->items, b->plan.req_size,
      reinterpret_cast<unsigned long long *>(b->plan.req_ptr), b->plan.free_ids, b->ctl,
      b->ctl + b->plan.nbatch + 1, acc);
}

void release_batched(Batched *b) {
  if (!b) return;
  if (b->graph) cudaGraphExecDestroy(b->exec);
  cudaFree(b->tasks);
  cudaFree(b->btasks);
  cudaFree(b->bdep);
  cudaFree(b->ctl);
  delete b;
}
}  // namespace

extern "C" int ha_batched_prepare_c(const ha_batch_plan_t *plan, uint32_t block,
                                    uint32_t ctas_per_sm, uint32_t task_items, int use_graph,
                                    void **out) {
  if (!plan || !out || !plan->acc || !plan->h_batch_start || !plan->h_free_start ||
      block == 0 || block > 1024 || block % 32 || task_items == 0)
    return HA_EINVAL;
  *out = nullptr;
  uint64_t ntasks = 0;
  if (check_plan_offsets(plan, task_items, &ntasks) != HA_OK || ntasks > 0xffffffffull)
    return HA_EINVAL;
  // task table: for each step its allocation chunks, then its free chunks.
  // A free chunk of step s waits for every batch before s; queued after
  // batch s's allocations it is taken when batch s - 1 has long been taken
  // (and has most likely finished), so blocks seldom idle at a step.
  std::vector<BatchTask> tasks;
  std::vector<uint32_t> btasks(plan->nbatch + 1, 0);
  std::vector<uint2> bdep(plan->nbatch + 1);
  tasks.reserve((size_t)ntasks);
  for (uint32_t st = 0; st <= plan->nbatch; st++) {
    if (st < plan->nbatch) {
      bdep[st] = make_uint2(plan->h_batch_start[st], (uint32_t)tasks.size());
      const uint64_t b1 = plan->h_batch_start[st + 1];
      for (uint64_t r = plan->h_batch_start[st]; r < b1; r += task_items) {
        tasks.push_back({(uint32_t)r, (uint32_t)(r + task_items < b1 ? r + task_items : b1), st,
                         0u});
        btasks[st]++;
      }
    }
    const uint64_t f1 = plan->h_free_start[st + 1];
    for (uint64_t k = plan->h_free_start[st]; k < f1; k += task_items)
      tasks.push_back({(uint32_t)k, (uint32_t)(k + task_items < f1 ? k + task_items : f1), st, 1u});
  }
  int dev = 0, nsm = 0, fit = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, ha_bpersist_k, (int)block, 0) !=
          cudaSuccess || fit <= 0)
    return HA_ECUDA;
  Batched *b = new Batched();
  b->plan = *plan;
  b->plan.h_batch_start = nullptr;  // not kept
  b->plan.h_free_start = nullptr;
  b->ntasks = (uint32_t)tasks.size();
  b->block = block;
  b->items = task_items;
  b->grid = (uint32_t)nsm * (ctas_per_sm && ctas_per_sm < (uint32_t)fit ? ctas_per_sm : fit);
  if (cudaMalloc(&b->tasks, sizeof(BatchTask) * (tasks.empty() ? 1 : tasks.size())) !=
          cudaSuccess ||
      cudaMalloc(&b->btasks, sizeof(uint32_t) * btasks.size()) != cudaSuccess ||
      cudaMalloc(&b->bdep, sizeof(uint2) * bdep.size()) != cudaSuccess ||
      cudaMalloc(&b->ctl, ((size_t)plan->nbatch + 1 + tasks.size()) * sizeof(unsigned int)) !=
          cudaSuccess ||
      cudaMemcpy(b->tasks, tasks.data(), sizeof(BatchTask) * tasks.size(),
                 cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(b->btasks, btasks.data(), sizeof(uint32_t) * btasks.size(),
                 cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemcpy(b->bdep, bdep.data(), sizeof(uint2) * bdep.size(), cudaMemcpyHostToDevice) !=
          cudaSuccess) {
    cudaGetLastError();
    release_batched(b);
    return HA_ECUDA;
  }
  if (use_graph) {
    cudaStream_t cap;
    cudaGraph_t g;
    if (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess) {
      release_batched(b);
      return HA_ECUDA;
    }
    bool ok = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) == cudaSuccess;
    if (ok) {
      enqueue_persistent(b, cap);
      ok = cudaStreamEndCapture(cap, &g) == cudaSuccess;
    }
    if (ok) {
      ok = cudaGraphInstantiate(&b->exec, g, 0) == cudaSuccess;
      cudaGraphDestroy(g);
    }
    cudaStreamDestroy(cap);
    if (!ok) {
      cudaGetLastError();
      release_batched(b);
      return HA_ECUDA;
    }
    b->graph = true;
  }
  *out = b;
  return HA_OK;
}

extern "C" int ha_batched_launch_c(void *handle, void *stream) {
  if (!handle) return HA_EINVAL;
  Batched *b = static_cast<Batched *>(handle);
  cudaStream_t s = as_stream(stream);
  if (b->graph) {
    if (cudaGraphLaunch(b->exec, s) != cudaSuccess) return launch_status();
    return HA_OK;
  }
  enqueue_persistent(b, s);
  return launch_status();
}

extern "C" int ha_batched_release_c(void *handle) {
  if (!handle) return HA_EINVAL;
  release_batched(static_cast<Batched *>(handle));
  return HA_OK;
}

extern "C" int ha_graph_build_c(uint32_t n, uint32_t seed, const uint32_t *cdf, uint32_t ncdf,
                                uint64_t *arr, uint32_t *deg, uint64_t *acc, void *stream) {
  if (!cdf || !ncdf || !arr || !deg || !acc) return HA_EINVAL;
  if (n == 0) return HA_OK;
  cudaStream_t s = as_stream(stream);
  if (cudaMemsetAsync(acc, 0, 3 * sizeof(uint64_t), s) != cudaSuccess) return HA_ECUDA;
  ha_graph_build_k<<<blocks_for(n, 128), 128, 0, s>>>(
      n, seed, cdf, ncdf, reinterpret_cast<unsigned long long *>(arr), deg,
      reinterpret_cast<unsigned long long *>(acc));
  return launch_status();
}

extern "C" int ha_graph_gather_c(uint32_t n, uint64_t *arr, const uint32_t *deg,
                                 const uint64_t *offsets, uint32_t *cols, void *stream) {
  if (!arr || !deg || !offsets || !cols) return HA_EINVAL;
  if (n == 0) return HA_OK;
  ha_graph_gather_k<<<blocks_for(n, 128), 128, 0, as_stream(stream)>>>(
      n, reinterpret_cast<unsigned long long *>(arr), deg,
      reinterpret_cast<const unsigned long long *>(offsets), cols);
  return launch_status();
}

namespace {
constexpr int kNoAllocDevices = 64;
unsigned char *g_noalloc_addr[kNoAllocDevices];  // scratch address per device
}  // namespace

extern "C" int ha_batched_run_noalloc_c(const ha_batch_plan_t *plan, uint32_t block,
                                        uint32_t ctas_per_sm, uint32_t task_items,
                                        void *stream) {
  if (!plan || !plan->acc || !plan->h_batch_start || !plan->h_free_start || block == 0 ||
      block > 1024 || block % 32 || task_items == 0)
    return HA_EINVAL;
  if (plan->nbatch > kNoAllocMaxBatches) return HA_ERANGE;
  uint64_t ntasks = 0;
  if (check_plan_offsets(plan, task_items, &ntasks) != HA_OK) return HA_EINVAL;
  if (ntasks > kNoAllocMaxTasks) return HA_ERANGE;
  NoAllocOffsets off;
  memcpy(off.batch_start, plan->h_batch_start, (plan->nbatch + 1) * sizeof(uint32_t));
  memcpy(off.free_start, plan->h_free_start, (plan->nbatch + 2) * sizeof(uint32_t));
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocDevices) return HA_ECUDA;
  if (!g_noalloc_addr[dev]) {
    // once per device: the device address of the scratch array (in host code
    // the symbol names a host-side stand-in, not device memory)
    unsigned char *p = nullptr;
    if (cudaGetSymbolAddress((void **)&p, g_noalloc_scratch) != cudaSuccess || !p) {
      cudaGetLastError();
      return HA_ECUDA;
    }
    g_noalloc_addr[dev] = p;
  }
  unsigned char *scratch = g_noalloc_addr[dev];
  int nsm = 0, fit = 0;
  if (cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, ha_bpersist_k, (int)block, 0) !=
          cudaSuccess || fit <= 0)
    return HA_ECUDA;
  const uint32_t grid =
      (uint32_t)nsm * (ctas_per_sm && ctas_per_sm < (uint32_t)fit ? ctas_per_sm : fit);
  cudaStream_t s = as_stream(stream);
  unsigned long long *acc = reinterpret_cast<unsigned long long *>(plan->acc);
  if (cudaMemsetAsync(acc, 0, 8 * sizeof(uint64_t), s) != cudaSuccess ||
      cudaMemsetAsync(scratch + kNaDoneOff, 0, ntasks * sizeof(unsigned int), s) != cudaSuccess)
    return HA_ECUDA;
  ha_noalloc_tasks_k<<<1, 1, 0, s>>>(scratch, plan->nbatch, task_items, off);
  ha_bpersist_k<<<grid, block, 0, s>>>(
      reinterpret_cast<const BatchTask *>(scratch + kNaTasksOff), (uint32_t)ntasks,
      reinterpret_cast<const uint32_t *>(scratch + kNaBtasksOff),
      reinterpret_cast<const uint2 *>(scratch + kNaBdepOff), task_items, plan->req_size,
      reinterpret_cast<unsigned long long *>(plan->req_ptr), plan->free_ids,
      reinterpret_cast<unsigned int *>(scratch + kNaCtlOff),
      reinterpret_cast<unsigned int *>(scratch + kNaDoneOff), acc);
  return launch_status();
}

extern "C" int ha_stamps_run_c(uint32_t nbytes, uint32_t niters, uint32_t *d_out,
                               void *stream) {
#ifdef HA_STAMPS
  if (!d_out || niters == 0 || nbytes == 0 || nbytes > 3072) return HA_EINVAL;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess)
    fprintf(stderr, "halloc-b200: error pending before the stamps launch: %s\n",
            cudaGetErrorString(e));
  e = cudaFuncSetAttribute(ha_stamps_k, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)ha::kStampBytes);
  if (e != cudaSuccess) {
    fprintf(stderr, "halloc-b200: stamps kernel attribute: %s\n", cudaGetErrorString(e));
    return HA_ECUDA;
  }
  ha_stamps_k<<<1, 32, ha::kStampBytes, as_stream(stream)>>>(nbytes, niters, d_out);
  e = cudaGetLastError();
  if (e != cudaSuccess) {
    cudaFuncAttributes fa;
    memset(&fa, 0, sizeof(fa));
    cudaFuncGetAttributes(&fa, ha_stamps_k);
    cudaGetLastError();
    fprintf(stderr,
            "halloc-b200: stamps launch failed: %s (static smem %zu, max dynamic smem %d, "
            "local %zu, regs %d, max threads %d)\n",
            cudaGetErrorString(e), fa.sharedSizeBytes, fa.maxDynamicSharedSizeBytes,
            fa.localSizeBytes, fa.numRegs, fa.maxThreadsPerBlock);
    return HA_ECUDA;
  }
  return HA_OK;
#else
  (void)nbytes, (void)niters, (void)d_out, (void)stream;
  return HA_ESTATE;  // a normal build records no stamps
#endif
}

extern "C" int ha_trace_c(const int64_t *ops, int64_t n, int64_t *out, void *stream) {
  if (!ops || !out || n < 0) return HA_EINVAL;
  if (n == 0) return HA_OK;
  ha_trace_k<<<1, 1, 0, as_stream(stream)>>>(ops, n, out);
  return launch_status();
}

extern "C" int ha_atomic_peak_c(uint32_t *buf, uint32_t nwords, uint32_t nthreads,
                                uint32_t reps, int returning, void *stream) {
  return ha_atomic_peak_strided_c(buf, nwords, 1, nthreads, reps, returning, stream);
}

extern "C" int ha_atomic_peak_strided_c(uint32_t *buf, uint32_t nwords, uint32_t stride,
                                        uint32_t nthreads, uint32_t reps, int returning,
                                        void *stream) {
  if (!buf || nwords == 0 || stride == 0 || nthreads == 0 || reps == 0) return HA_EINVAL;
  ha_atomic_peak_k<<<blocks_for(nthreads, 256), 256, 0, as_stream(stream)>>>(
      buf, nwords, stride, reps, returning);
  return launch_status();
}
