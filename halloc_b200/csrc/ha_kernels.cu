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

#include "halloc.h"
#include "halloc_c.h"

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
__device__ __forceinline__ uint4 load16(const void *p) {
  if (((uintptr_t)p & 15u) == 0) return __ldcg(reinterpret_cast<const uint4 *>(p));
  const uint2 a = __ldcg(reinterpret_cast<const uint2 *>(p));
  const uint2 b = __ldcg(reinterpret_cast<const uint2 *>(p) + 1);
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
// with the 16-byte payload write and checksummed read-back of each block
template <bool kCudaHeap>
__global__ void ha_throughput_k(const uint32_t *sizes, uint32_t nbytes, uint32_t n,
                                uint32_t nallocs, uint32_t niters,
                                unsigned long long *out) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long sum = 0, nfail = 0;
  if (i < n) {
    const uint32_t sz = sizes ? sizes[i] : nbytes;
    const uint4 word = make_uint4(i ^ 0u, i ^ 1u, i ^ 2u, i ^ 3u);
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
        sum += (unsigned long long)v.x + v.y + v.z + v.w;
        if (kCudaHeap)
          free(p);
        else
          hafree(p);
      }
    }
  }
  block_add2(sum, nfail, out, out + 1);
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
            const uint32_t base = mix32(h ^ 0x5EED5EEDu);
            uint2 *q = reinterpret_cast<uint2 *>(p);
            for (uint32_t w = 0; w < sz / 8; w++) {
              const uint32_t a = base + 2 * w, b = base + 2 * w + 1;
              q[w] = make_uint2(a, b);
              wsum += (unsigned long long)a + b;
            }
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
        const uint2 *q = reinterpret_cast<const uint2 *>(p);
        const uint32_t sz = slot_sz[k];
        for (uint32_t w = 0; w < sz / 8; w++) {
          const uint2 v = __ldcg(q + w);
          rsum += (unsigned long long)v.x + v.y;
        }
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

// distinct-address 32-bit atomic OR throughput
__global__ void ha_atomic_peak_k(uint32_t *buf, uint32_t nwords, uint32_t reps,
                                 int returning) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  uint32_t *w = &buf[t % nwords];
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

extern "C" int ha_throughput_host_c(const uint32_t *h_sizes, uint32_t *d_sizes,
                                    uint32_t nbytes, uint32_t nthreads, uint32_t block,
                                    uint32_t nallocs, uint32_t niters, uint64_t *d_out,
                                    uint64_t *h_out, void *stream) {
  if (!d_out || !h_out || (h_sizes && !d_sizes)) return HA_EINVAL;
  cudaStream_t s = as_stream(stream);
  if (h_sizes &&
      cudaMemcpyAsync(d_sizes, h_sizes, (size_t)nthreads * 4, cudaMemcpyHostToDevice, s) !=
          cudaSuccess)
    return HA_ECUDA;
  if (cudaMemsetAsync(d_out, 0, 2 * sizeof(uint64_t), s) != cudaSuccess) return HA_ECUDA;
  int rc = throughput(false, h_sizes ? d_sizes : nullptr, nbytes, nthreads, block, nallocs,
                      niters, d_out, stream);
  if (rc) return rc;
  if (cudaMemcpyAsync(h_out, d_out, 2 * sizeof(uint64_t), cudaMemcpyDeviceToHost, s) !=
          cudaSuccess ||
      cudaStreamSynchronize(s) != cudaSuccess)
    return HA_ECUDA;
  return HA_OK;
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

extern "C" int ha_trace_c(const int64_t *ops, int64_t n, int64_t *out, void *stream) {
  if (!ops || !out || n < 0) return HA_EINVAL;
  if (n == 0) return HA_OK;
  ha_trace_k<<<1, 1, 0, as_stream(stream)>>>(ops, n, out);
  return launch_status();
}

extern "C" int ha_atomic_peak_c(uint32_t *buf, uint32_t nwords, uint32_t nthreads,
                                uint32_t reps, int returning, void *stream) {
  if (!buf || nwords == 0 || nthreads == 0 || reps == 0) return HA_EINVAL;
  ha_atomic_peak_k<<<blocks_for(nthreads, 256), 256, 0, as_stream(stream)>>>(buf, nwords, reps,
                                                                            returning);
  return launch_status();
}
