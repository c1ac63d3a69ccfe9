// ha_serve.cu -- serving loop: a host-fed job stream served by continuous
// batching in one persistent kernel (ha_serve_run_c, halloc_c.h).
//
// Jobs are ids; every parameter derives from a hash of (seed, id), so a
// job's result does not depend on what else runs beside it.  A host thread
// releases ids at Poisson arrival times through a counter in mapped host
// memory.  Each thread of the persistent kernel owns one job slot; a warp
// claims released jobs for its empty slots while the slab pool is at most
// `occupancy_limit` full, then advances every active job by one step:
// grow by 1..32 blocks of 256 B (hamalloc, linked through the blocks), and
// after the job's lifetime read its blocks back and hafree them, a bounded
// number per step.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <chrono>
#include <random>
#include <vector>

#include "halloc.h"
#include "halloc_c.h"
#include "ha_hist.cuh"

namespace {

using ha::bucket_value;
using ha::lat_bucket;
using ha::percentile;

struct ServeCtl {  // mapped host memory
  uint32_t released;   // host: ids order[0 .. released) may be claimed
  uint32_t ended;      // host: nothing more will be released
  uint32_t grow_req;   // device: a block could not be had, back more slabs
  uint32_t grow_done;  // host: the pool cannot grow any more
};

struct ServeDev {  // device memory
  uint32_t claimed;        // next index of order[] to hand out
  uint32_t released_seen;  // largest host release count a warp has read
  unsigned long long live_blocks, peak_live;
  unsigned long long jobs_done, allocs, failures, refusals, timeouts, waits;
  unsigned long long cycles, nanos;
  unsigned long long hist[HA_SERVE_HIST];
};

struct ServeParams {
  const uint32_t *order;
  uint32_t norder;
  uint32_t seed;
  uint32_t block_bytes;
  float log_min, log_span;  // log-uniform job length
  float mean_life;
  uint32_t grow_min, grow_span;
  unsigned long long live_limit;  // admission: live blocks must be <= this
  unsigned long long *results;
  ServeCtl *ctl;  // device view of the mapped host struct
  ServeDev *dev;
  uint32_t grow;  // 1: a growing pool, a job waits for memory instead of failing
};

// steps a job may wait for the pool to grow before its request counts as
// failed (bounds the kernel when the pool cannot grow in time)
constexpr uint32_t kMaxStalls = 1u << 16;

__device__ __forceinline__ uint32_t mix32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}
__device__ __forceinline__ uint32_t ld_acquire_sys(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.acquire.sys.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ uint64_t now_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// log-linear latency bucket: 16 buckets per power of two

struct Job {
  uint32_t id, target, blocks, steps, life, h;
  uint32_t step_blocks;  // blocks added in the current step
  uint32_t stalls;       // attempts of the current step that waited for memory
};

__device__ __forceinline__ void job_start(Job &j, uint32_t id, const ServeParams &P) {
  j.id = id;
  j.h = mix32(P.seed ^ mix32(id));
  const float u1 = ((float)j.h + 0.5f) * 2.3283064e-10f;
  const float len = expf(P.log_min + u1 * P.log_span);
  j.target = max(1u, (uint32_t)ceilf(len / (float)P.block_bytes));
  const float u2 = ((float)mix32(j.h ^ 0x51ED270Bu) + 0.5f) * 2.3283064e-10f;
  j.life = max(1u, (uint32_t)ceilf(-P.mean_life * logf(u2)));
  j.blocks = 0;
  j.steps = 0;
  j.step_blocks = 0;
  j.stalls = 0;
}

__device__ __forceinline__ void st_release_sys(uint32_t *p, uint32_t v) {
  asm volatile("st.release.sys.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t *p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long *p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p));
  return v;
}

constexpr uint32_t kDrainPerStep = 64;  // blocks a finished job frees per step

// Each warp runs its own loop: claim released jobs for its empty slots
// (while the pool is under the admission limit), then give every slot one
// bounded step -- grow by up to grow_max blocks, or, once the job's lifetime
// is over, read back and free up to kDrainPerStep of its blocks.  No step
// waits for other warps.
__global__ void __launch_bounds__(1024) ha_serve_k(ServeParams P) {
  __shared__ unsigned long long s_hist[HA_SERVE_HIST];
  for (uint32_t i = threadIdx.x; i < HA_SERVE_HIST; i += blockDim.x) s_hist[i] = 0;
  __syncthreads();
  const uint64_t ns0 = now_ns();
  const long long cyc0 = clock64();
  const uint32_t lane = threadIdx.x & 31;
  Job j;
  j.id = 0xffffffffu;
  bool draining = false;
  void *head = nullptr;
  unsigned long long vsum = 0, my_allocs = 0, my_fail = 0, my_done = 0, my_refused = 0,
                     my_waits = 0;
  uint64_t idle_since = 0;
  for (;;) {
    // ---- admission, one claim per warp -------------------------------------
    const bool empty = j.id == 0xffffffffu;
    const uint32_t em = __ballot_sync(0xffffffffu, empty);
    uint32_t base = 0, k = 0;
    if (em && lane == 0) {
      if (ld_relaxed_u64(&P.dev->live_blocks) > P.live_limit) {
        my_refused++;
      } else {
        uint32_t c = ld_relaxed_u32(&P.dev->claimed);
        // once every job is claimed, neither counter can offer one more
        uint32_t r = c < P.norder ? min(ld_relaxed_u32(&P.dev->released_seen), P.norder) : c;
        if (r <= c && c < P.norder) {  // nothing known to be claimable: look at the host counter
          r = min(ld_acquire_sys(&P.ctl->released), P.norder);
          if (r > c) atomicMax(&P.dev->released_seen, r);
        }
        while (r > c) {
          const uint32_t want = min((uint32_t)__popc(em), r - c);
          const uint32_t got = atomicCAS(&P.dev->claimed, c, c + want);
          if (got == c) {
            base = c;
            k = want;
            break;
          }
          c = got;
        }
      }
    }
    base = __shfl_sync(0xffffffffu, base, 0);
    k = __shfl_sync(0xffffffffu, k, 0);
    if (empty) {
      const uint32_t rank = __popc(em & ((1u << lane) - 1));
      if (rank < k) {
        job_start(j, P.order[base + rank], P);
        draining = false;
        head = nullptr;
        vsum = 0;
      }
    }
    // ---- one bounded step of this lane's job --------------------------------
    uint32_t grown = 0, freed = 0;
    if (j.id != 0xffffffffu) {
      if (!draining) {
        const uint32_t g =
            P.grow_min + mix32(j.h + j.steps * 0x9E3779B9u) % P.grow_span;
        bool stalled = false;
        while (j.step_blocks < g && j.blocks < j.target) {
          const long long t0 = clock64();
          void *p = hamalloc(P.block_bytes);
          const long long t1 = clock64();
          atomicAdd(&s_hist[lat_bucket((unsigned long long)(t1 - t0))], 1ull);
          my_allocs++;
          if (!p) {
            if (P.grow && j.stalls < kMaxStalls && !ld_acquire_sys(&P.ctl->grow_done)) {
              // ask the host for more slabs; this step resumes later
              if (!ld_acquire_sys(&P.ctl->grow_req)) st_release_sys(&P.ctl->grow_req, 1u);
              my_waits++;
              j.stalls++;
              stalled = true;
            } else {
              my_fail++;
            }
            break;
          }
          *reinterpret_cast<void **>(p) = head;
          reinterpret_cast<uint32_t *>(p)[2] = mix32(j.id * 0x27D4EB2Fu + j.blocks);
          head = p;
          j.blocks++;
          j.step_blocks++;
          grown++;
        }
        if (!stalled) {
          j.step_blocks = 0;
          j.stalls = 0;
          if (++j.steps >= j.life) draining = true;
        }
      } else {
        for (uint32_t i = 0; i < kDrainPerStep && head; i++) {
          void *nx = *reinterpret_cast<void **>(head);
          vsum += reinterpret_cast<const uint32_t *>(head)[2];
          hafree(head);
          head = nx;
          freed++;
        }
        if (!head) {
          P.results[2 * (size_t)j.id] = j.blocks;
          P.results[2 * (size_t)j.id + 1] = vsum;
          my_done++;
          j.id = 0xffffffffu;
          draining = false;
        }
      }
    }
    // live-block count, one atomic per warp
    long long delta = (long long)grown - (long long)freed;
    for (int o = 16; o > 0; o >>= 1) delta += __shfl_down_sync(0xffffffffu, delta, o);
    if (lane == 0 && delta) {
      const unsigned long long now =
          atomicAdd(&P.dev->live_blocks, (unsigned long long)delta) + (unsigned long long)delta;
      if (delta > 0) atomicMax(&P.dev->peak_live, now);
    }
    // ---- leave when the stream has ended and this warp is idle ---------------
    const uint32_t active = __ballot_sync(0xffffffffu, j.id != 0xffffffffu);
    if (active == 0 && k == 0) {
      uint32_t leave = 0;
      if (lane == 0) {
        if (ld_acquire_sys(&P.ctl->ended) &&
            ld_relaxed_u32(&P.dev->claimed) >= P.norder) {
          leave = 1;
        } else {
          const uint64_t t = now_ns();
          if (!idle_since) idle_since = t;
          if (t - idle_since > 5000000000ull) {  // nothing to do for 5 s
            atomicAdd(&P.dev->timeouts, 1ull);
            leave = 1;
          } else {
            __nanosleep(2000);
          }
        }
      }
      if (__shfl_sync(0xffffffffu, leave, 0)) break;
    } else {
      idle_since = 0;
    }
  }
  // ---- totals ---------------------------------------------------------------
  for (int o = 16; o > 0; o >>= 1) {
    my_allocs += __shfl_down_sync(0xffffffffu, my_allocs, o);
    my_fail += __shfl_down_sync(0xffffffffu, my_fail, o);
    my_done += __shfl_down_sync(0xffffffffu, my_done, o);
    my_refused += __shfl_down_sync(0xffffffffu, my_refused, o);
    my_waits += __shfl_down_sync(0xffffffffu, my_waits, o);
  }
  if (lane == 0) {
    if (my_allocs) atomicAdd(&P.dev->allocs, my_allocs);
    if (my_fail) atomicAdd(&P.dev->failures, my_fail);
    if (my_done) atomicAdd(&P.dev->jobs_done, my_done);
    if (my_refused) atomicAdd(&P.dev->refusals, my_refused);
    if (my_waits) atomicAdd(&P.dev->waits, my_waits);
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < HA_SERVE_HIST; i += blockDim.x)
    if (s_hist[i]) atomicAdd(&P.dev->hist[i], s_hist[i]);
  if (threadIdx.x == 0) {
    atomicAdd(&P.dev->cycles, (unsigned long long)(clock64() - cyc0));
    atomicAdd(&P.dev->nanos, (unsigned long long)(now_ns() - ns0));
  }
}

}  // namespace

extern "C" int ha_serve_run_c(const ha_serve_cfg_t *cfg, ha_serve_result_t *out, void *stream) {
  if (!cfg || !out || !cfg->results || cfg->block_bytes < 16 || cfg->block_bytes > 3072 ||
      cfg->min_len == 0 || cfg->max_len < cfg->min_len || cfg->grow_min == 0 ||
      cfg->grow_max < cfg->grow_min || !(cfg->lambda > 0) || !(cfg->mean_life > 0) ||
      cfg->cta_threads == 0 || cfg->cta_threads > 1024 || cfg->cta_threads % 32)
    return HA_EINVAL;
  ha_stats_t st;
  int rc = ha_stats_c(&st);
  if (rc) return rc;
  const uint32_t n = cfg->job_ids ? cfg->njob_ids : cfg->njobs;
  memset(out, 0, sizeof(*out));
  if (n == 0) return HA_OK;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);

  std::vector<uint32_t> order(n);
  for (uint32_t i = 0; i < n; i++) order[i] = cfg->job_ids ? cfg->job_ids[i] : i;
  for (uint32_t i = 0; i < n; i++)
    if (order[i] >= cfg->njobs) return HA_EINVAL;  // results has 2*njobs words

  uint32_t *d_order = nullptr;
  ServeDev *d_dev = nullptr;
  ServeCtl *h_ctl = nullptr, *d_ctl = nullptr;
  auto cleanup = [&]() {
    cudaFree(d_order);
    cudaFree(d_dev);
    if (h_ctl) cudaFreeHost(h_ctl);
  };
  if (cudaMalloc(&d_order, n * sizeof(uint32_t)) != cudaSuccess ||
      cudaMalloc(&d_dev, sizeof(ServeDev)) != cudaSuccess ||
      cudaHostAlloc(&h_ctl, sizeof(ServeCtl), cudaHostAllocMapped) != cudaSuccess ||
      cudaHostGetDevicePointer((void **)&d_ctl, h_ctl, 0) != cudaSuccess ||
      cudaMemcpy(d_order, order.data(), n * sizeof(uint32_t), cudaMemcpyHostToDevice) !=
          cudaSuccess ||
      cudaMemset(d_dev, 0, sizeof(ServeDev)) != cudaSuccess) {
    cudaGetLastError();
    cleanup();
    return HA_ECUDA;
  }
  __atomic_store_n(&h_ctl->released, 0u, __ATOMIC_RELEASE);
  __atomic_store_n(&h_ctl->ended, 0u, __ATOMIC_RELEASE);
  __atomic_store_n(&h_ctl->grow_req, 0u, __ATOMIC_RELEASE);
  __atomic_store_n(&h_ctl->grow_done, 0u, __ATOMIC_RELEASE);
  if (cfg->prereleased) {  // a closed batch: every job known before the launch
    __atomic_store_n(&h_ctl->released, n, __ATOMIC_RELEASE);
    __atomic_store_n(&h_ctl->ended, 1u, __ATOMIC_RELEASE);
  }

  // Poisson arrival times (seconds from the start)
  std::mt19937_64 rng(cfg->seed * 0x9E3779B97F4A7C15ull + 1);
  std::exponential_distribution<double> gap(cfg->lambda);
  std::vector<double> arrive(n);
  double t = 0;
  for (uint32_t i = 0; i < n; i++) arrive[i] = (t += gap(rng));

  int dev = 0, nsm = 0, fit = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&fit, ha_serve_k, (int)cfg->cta_threads, 0) !=
          cudaSuccess ||
      fit <= 0) {
    cleanup();
    return HA_ECUDA;
  }
  const uint32_t per_sm =
      cfg->ctas_per_sm && cfg->ctas_per_sm < (uint32_t)fit ? cfg->ctas_per_sm : (uint32_t)fit;

  ServeParams P;
  P.order = d_order;
  P.norder = n;
  P.seed = cfg->seed;
  P.block_bytes = cfg->block_bytes;
  P.log_min = logf((float)cfg->min_len);
  P.log_span = logf((float)cfg->max_len) - P.log_min;
  P.mean_life = (float)cfg->mean_life;
  P.grow_min = cfg->grow_min;
  P.grow_span = cfg->grow_max - cfg->grow_min + 1;
  P.live_limit = (unsigned long long)(cfg->occupancy_limit * (double)st.pool_bytes) /
                 cfg->block_bytes;
  P.results = reinterpret_cast<unsigned long long *>(cfg->results);
  P.ctl = d_ctl;
  P.dev = d_dev;
  P.grow = cfg->grow_bytes && st.growth ? 1u : 0u;

  // growth requests are served on a stream of their own while the kernel runs
  cudaStream_t side = nullptr;
  if (P.grow && cudaStreamCreateWithFlags(&side, cudaStreamNonBlocking) != cudaSuccess) {
    cleanup();
    return HA_ECUDA;
  }
  uint64_t grows = 0, grown = 0;
  double grow_s = 0;
  auto serve_growth = [&]() {
    if (!P.grow || !__atomic_load_n(&h_ctl->grow_req, __ATOMIC_ACQUIRE)) return;
    const auto g0 = std::chrono::steady_clock::now();
    uint64_t added = 0;
    int r = ha_grow_c(cfg->grow_bytes, side, &added);
    // the request stands until the new slabs are in the free set: requests
    // made meanwhile are the same request
    if (r == HA_OK && cudaStreamSynchronize(side) != cudaSuccess) r = HA_ECUDA;
    if (r == HA_OK) {
      grows++;
      grown += added;
    } else {
      __atomic_store_n(&h_ctl->grow_done, 1u, __ATOMIC_RELEASE);
    }
    __atomic_store_n(&h_ctl->grow_req, 0u, __ATOMIC_RELEASE);
    grow_s += std::chrono::duration<double>(std::chrono::steady_clock::now() - g0).count();
  };

  ha_serve_k<<<nsm * per_sm, cfg->cta_threads, 0, s>>>(P);
  if (cudaGetLastError() != cudaSuccess) {
    if (side) cudaStreamDestroy(side);
    cleanup();
    return HA_ECUDA;
  }
  // release jobs at their arrival times
  const auto t0 = std::chrono::steady_clock::now();
  uint32_t released = cfg->prereleased ? n : 0;
  while (released < n) {
    const double now =
        std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    uint32_t r = released;
    while (r < n && arrive[r] <= now) r++;
    if (r != released) {
      released = r;
      __atomic_store_n(&h_ctl->released, released, __ATOMIC_RELEASE);
    }
    serve_growth();
  }
  __atomic_store_n(&h_ctl->ended, 1u, __ATOMIC_RELEASE);
  cudaError_t e;
  if (P.grow) {
    while ((e = cudaStreamQuery(s)) == cudaErrorNotReady) serve_growth();
    if (cudaStreamSynchronize(side) != cudaSuccess) e = cudaErrorUnknown;
    cudaStreamDestroy(side);
  } else {
    e = cudaStreamSynchronize(s);
  }
  const double secs =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  ServeDev hd;
  if (e != cudaSuccess || cudaMemcpy(&hd, d_dev, sizeof(hd), cudaMemcpyDeviceToHost) !=
                              cudaSuccess) {
    cudaGetLastError();
    cleanup();
    return HA_ECUDA;
  }
  out->seconds = secs;
  out->cycles_per_ns = hd.nanos ? (double)hd.cycles / (double)hd.nanos : 0;
  out->jobs_done = hd.jobs_done;
  out->allocs = hd.allocs;
  out->alloc_failures = hd.failures;
  out->refusals = hd.refusals;
  out->peak_live_blocks = hd.peak_live;
  out->timeouts = hd.timeouts;
  out->alloc_waits = hd.waits;
  out->grows = grows;
  out->grown_bytes = grown;
  out->grow_seconds = grow_s;
  memcpy(out->hist, hd.hist, sizeof(hd.hist));
  out->p50_cycles = percentile(hd.hist, 0.50);
  out->p99_cycles = percentile(hd.hist, 0.99);
  for (int i = HA_SERVE_HIST - 1; i >= 0; i--)
    if (hd.hist[i]) {
      out->max_cycles = bucket_value(i + 1);
      break;
    }
  cleanup();
  return HA_OK;
}
