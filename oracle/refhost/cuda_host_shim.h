/*
 * cuda_host_shim.h -- lets the reference allocator's own CUDA C++ sources
 * (halloc 0.11, src/halloc.cu and the headers it includes) compile and run as
 * ordinary host C++.  TEST INFRASTRUCTURE ONLY: this is part of the oracle,
 * never part of the product path.
 *
 * Model of execution: every host thread that calls hamalloc()/hafree() is one
 * GPU thread that is alone in its warp (a single-lane warp).  The warp votes
 * therefore see only lane 0, and every device atomic becomes a sequentially
 * consistent host atomic, so several host threads may run the reference code
 * concurrently (that is how the multi-core CPU baseline uses it).
 *
 * The CUDA runtime calls made by ha_init() (src/halloc.cu:267-424) are
 * replaced by host memory operations.  Slab allocations are served
 * consecutively from one arena, so slab i lies at arena + i * slab size and a
 * returned pointer can be reported as (slab, byte offset).
 *
 * This file is force-included (g++ -include) before the reference sources.
 * All system headers are pulled in first, before the CUDA keywords are
 * defined away, so that no library header sees those macros.
 */
#ifndef HA_CUDA_HOST_SHIM_H_
#define HA_CUDA_HOST_SHIM_H_

#include <algorithm>
#include <assert.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <sys/types.h>
#include <type_traits>

/* ---- CUDA keywords: plain host code ------------------------------------ */
#define __device__
#define __host__
#define __global__
#define __constant__
#define __shared__
#define __forceinline__ inline
#define __noinline__ __attribute__((noinline))

/* ---- integer min/max with CUDA's mixed-type overload behaviour ---------- */
template <class A, class B>
static inline typename std::common_type<A, B>::type max(A a, B b) {
  typedef typename std::common_type<A, B>::type T;
  return (T)a > (T)b ? (T)a : (T)b;
}
template <class A, class B>
static inline typename std::common_type<A, B>::type min(A a, B b) {
  typedef typename std::common_type<A, B>::type T;
  return (T)a < (T)b ? (T)a : (T)b;
}

/* ---- device atomics as host atomics ------------------------------------ */
static inline unsigned atomicAdd(unsigned *p, unsigned v) {
  return __atomic_fetch_add(p, v, __ATOMIC_SEQ_CST);
}
static inline int atomicAdd(int *p, int v) {
  return __atomic_fetch_add(p, v, __ATOMIC_SEQ_CST);
}
static inline unsigned long long atomicAdd(unsigned long long *p,
                                           unsigned long long v) {
  return __atomic_fetch_add(p, v, __ATOMIC_SEQ_CST);
}
static inline unsigned atomicSub(unsigned *p, unsigned v) {
  return __atomic_fetch_sub(p, v, __ATOMIC_SEQ_CST);
}
static inline int atomicSub(int *p, int v) {
  return __atomic_fetch_sub(p, v, __ATOMIC_SEQ_CST);
}
static inline unsigned atomicOr(unsigned *p, unsigned v) {
  return __atomic_fetch_or(p, v, __ATOMIC_SEQ_CST);
}
static inline unsigned atomicAnd(unsigned *p, unsigned v) {
  return __atomic_fetch_and(p, v, __ATOMIC_SEQ_CST);
}
static inline unsigned atomicExch(unsigned *p, unsigned v) {
  return __atomic_exchange_n(p, v, __ATOMIC_SEQ_CST);
}
static inline void __threadfence(void) {
  __atomic_thread_fence(__ATOMIC_SEQ_CST);
}

/* ---- warp intrinsics for a single-lane warp (lane 0) -------------------- */
static inline unsigned __ballot(int pred) { return pred ? 1u : 0u; }
static inline int __any(int pred) { return pred != 0; }
static inline int __ffs(int x) { return __builtin_ffs(x); }
static inline int __popc(unsigned x) { return __builtin_popcount(x); }
static inline int __clz(int x) {
  return x == 0 ? 32 : __builtin_clz((unsigned)x);
}

/* ---- CUDA runtime subset used by ha_init() ------------------------------ */
typedef int cudaError_t;
enum { cudaSuccess = 0, cudaErrorMemoryAllocation = 2 };
enum cudaFuncCache { cudaFuncCachePreferNone = 0, cudaFuncCachePreferL1 = 2 };
enum cudaLimit { cudaLimitMallocHeapSize = 2 };
enum cudaMemcpyKind { cudaMemcpyHostToDevice = 1, cudaMemcpyDeviceToHost = 2 };
struct cudaDeviceProp {
  size_t totalGlobalMem;
};
typedef void *cudaStream_t;

/* Parameters of the simulated device, set by the oracle wrapper before
   ha_init() runs (see refhost_api.cpp). */
struct ha_shim_device_t {
  size_t total_mem;      /* reported as cudaDeviceProp::totalGlobalMem */
  char *arena;           /* slab arena */
  size_t arena_chunk;    /* slab size served from the arena */
  size_t arena_nchunks;  /* capacity in slabs */
  size_t arena_next;     /* next free slab index */
  void *other[64];       /* non-arena allocations, released on reset */
  int nother;
  size_t heap_limit;     /* what ha_init asked for the CUDA heap */
};
extern ha_shim_device_t ha_shim_dev;

static inline const char *cudaGetErrorString(cudaError_t e) {
  return e == cudaSuccess ? "no error" : "host shim error";
}
static inline cudaError_t cudaGetDevice(int *dev) {
  *dev = 0;
  return cudaSuccess;
}
static inline cudaError_t cudaGetDeviceProperties(cudaDeviceProp *p, int) {
  p->totalGlobalMem = ha_shim_dev.total_mem;
  return cudaSuccess;
}
static inline cudaError_t cudaDeviceSetCacheConfig(int) { return cudaSuccess; }
static inline cudaError_t cudaDeviceSetLimit(int, size_t v) {
  ha_shim_dev.heap_limit = v;
  return cudaSuccess;
}
static inline cudaError_t cudaMalloc(void **p, size_t n) {
  if (ha_shim_dev.arena && n == ha_shim_dev.arena_chunk &&
      ha_shim_dev.arena_next < ha_shim_dev.arena_nchunks) {
    *p = ha_shim_dev.arena + ha_shim_dev.arena_next++ * n;
    return cudaSuccess;
  }
  if (ha_shim_dev.nother >= 64) return cudaErrorMemoryAllocation;
  size_t rounded = (n + 4095) & ~(size_t)4095;
  void *q = aligned_alloc(4096, rounded ? rounded : 4096);
  if (!q) return cudaErrorMemoryAllocation;
  ha_shim_dev.other[ha_shim_dev.nother++] = q;
  *p = q;
  return cudaSuccess;
}
static inline cudaError_t cudaMemset(void *p, int v, size_t n) {
  memset(p, v, n);
  return cudaSuccess;
}
static inline cudaError_t cudaMemcpy(void *d, const void *s, size_t n, int) {
  memcpy(d, s, n);
  return cudaSuccess;
}
static inline cudaError_t cudaStreamSynchronize(cudaStream_t) {
  return cudaSuccess;
}

#endif /* HA_CUDA_HOST_SHIM_H_ */
