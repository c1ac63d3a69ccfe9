// halloc.cu -- public entry points of halloc-b200 and its host init layer.
//
// Device: hamalloc / hafree with halloc.h's signatures and C++ linkage,
// resolved at device-link time (-rdc) exactly like the original library.
// Host: ha_init / ha_shutdown / ha_extfrag (C++ API of halloc.h) and the
// init / statistics half of the C ABI (halloc_c.h).
#define HALLOCLIB_COMPILING

#include <cuda.h>  // driver API types; the functions come from cudaGetDriverEntryPoint
#include <cuda_runtime.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <new>

#include "halloc.h"
#include "halloc_c.h"
#include "ha_core.cuh"

static_assert(sizeof(halloc_opts_t) == sizeof(ha_opts_c),
              "halloc_opts_t and ha_opts_c must share one layout");
static_assert(offsetof(halloc_opts_t, sb_sz_sh) == offsetof(ha_opts_c, sb_sz_sh),
              "halloc_opts_t and ha_opts_c must share one layout");

namespace ha {
__constant__ Config c_cfg;
__device__ Class g_cls[kNSizes];
__device__ uint4 g_mod[kNSizes];
__device__ State g_st;

// statistics scratch, written by stats_k
struct StatsOut {
  unsigned long long used_chunks, used_bytes, free_bytes, ideal_bytes;
  unsigned int free_slabs, head_slabs;
};
__device__ StatsOut g_stats_out;
__device__ unsigned long long g_max_alloc;
// ha_trim_c scratch: candidate chunks in (first slab, slab count), the
// indices of the released ones out
__device__ uint2 g_trim_chunks[kMaxSlabs];
__device__ uint32_t g_trim_out[kMaxSlabs];
__device__ uint32_t g_trim_n, g_trim_slabs;
#if HA_PROBE_STATS
__device__ unsigned long long g_pstats[kPsCopies * kPsStride];
#endif
}  // namespace ha

// ---------------------------------------------------------------------------
// device entry points
// ---------------------------------------------------------------------------

__device__ __noinline__ void *hamalloc(size_t nbytes) {
  if (nbytes > ha::kMaxBlock) return malloc(nbytes);
  if (ha::c_cfg.nsbs == 0) return nullptr;  // not initialised
  return ha::malloc_small((uint32_t)nbytes);
}

__device__ __noinline__ void hafree(void *p) {
  if (!p) return;
  uint64_t off = (uint64_t)((const char *)p - ha::c_cfg.pool);
  if (off < ha::c_cfg.pool_bytes)
    ha::free_small(off);
  else
    free(p);
}

__global__ void ha_adopt_k(uint32_t first, uint32_t count);

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------
namespace {

struct HostDev {
  bool init;
  char *raw_pool;
  char *pool;
  uint64_t pool_bytes;
  uint32_t *meta;
  size_t meta_bytes;
  uint64_t heap_bytes;
  uint32_t nsbs, sb_sh;
  bool heap_ok;
  size_t persist_bytes;
  // growth (ha_set_growth_c): the pool is a reserved address range backed
  // on demand by chunks, one device allocation each (a handle costs about a
  // millisecond to create and map whatever its size, so a grow backs its
  // whole request with one); backed[u] marks the units in a chunk
  bool growth;
  unsigned long long va;
  uint64_t unit_bytes;
  uint32_t spu;  // slabs per unit
  uint32_t nunits;
  uint8_t *backed;
  struct Chunk {
    uint32_t first, n;  // units
    unsigned long long handle;
  } *chunks;
  uint32_t nchunks;
};
constexpr int kMaxDevices = 64;
HostDev g_dev[kMaxDevices];
// hash-step scale for the next init, in percent (100 = the reference rule)
uint32_t g_hash_scale_pct = 100;
// head slabs per size for the next init (1 = the reference policy)
uint32_t g_nheads = 1;
bool g_nheads_set = false;  // ha_set_heads_c was called

// Head slabs per size for an init.  A program written against halloc.h alone
// cannot call ha_set_heads_c; HALLOC_HEADS in its environment (a power of
// two up to kMaxHeads) sets the same knob.  An ha_set_heads_c call wins.
uint32_t heads_for_init() {
  if (g_nheads_set) return g_nheads;
  const char *e = getenv("HALLOC_HEADS");
  if (!e || !*e) return g_nheads;
  char *end = nullptr;
  const unsigned long v = strtoul(e, &end, 10);
  if (*end || v == 0 || v > ha::kMaxHeads || (v & (v - 1))) {
    fprintf(stderr, "halloc-b200: HALLOC_HEADS=%s ignored (a power of two from 1 to %u)\n", e,
            (unsigned)ha::kMaxHeads);
    return g_nheads;
  }
  return (uint32_t)v;
}
// bytes backed at the next init, 0 = the whole pool (no growth)
uint64_t g_growth_initial = 0;
// surge head sets for the next init: -1 = from HALLOC_SURGE (default on)
int g_surge = -1;

// Whether an init with `nheads` head slabs per size opens surge head sets
// under contention: only with the single head of the reference policy.  A
// program written against halloc.h alone turns them off with HALLOC_SURGE=0
// in its environment; an ha_set_surge_c call wins.
uint32_t surge_for_init(uint32_t nheads) {
  if (nheads != 1) return 0;
  if (g_surge >= 0) return (uint32_t)g_surge;
  const char *e = getenv("HALLOC_SURGE");
  if (!e || !*e) return 1;
  if (!strcmp(e, "0")) return 0;
  if (!strcmp(e, "1")) return 1;
  fprintf(stderr, "halloc-b200: HALLOC_SURGE=%s ignored (0 or 1)\n", e);
  return 1;
}

uint32_t decode_head(uint32_t w) {
  const uint32_t sb = w & ha::kSlabField;
  return sb == ha::kSlabField ? ha::kNone : sb;
}

#define HA_CK(call)                                   \
  do {                                                \
    cudaError_t e_ = (call);                          \
    if (e_ != cudaSuccess) {                          \
      fprintf(stderr, "halloc-b200: %s failed: %s\n", \
              #call, cudaGetErrorString(e_));         \
      return HA_ECUDA;                                \
    }                                                 \
  } while (0)

HostDev *current(int *dev_out = nullptr) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return nullptr;
  if (dev_out) *dev_out = dev;
  return &g_dev[dev];
}

// largest prime p in [3, n) dividing neither n nor nb; 0 if none
// (the hash-step rule of halloc src/utils.cu:8-24)
uint32_t prime_below(uint32_t n, uint32_t nb) {
  for (uint32_t p = n - 1; p >= 3 && p < n; p--) {
    bool prime = true;
    for (uint32_t d = 2; (uint64_t)d * d <= p; d++)
      if (p % d == 0) {
        prime = false;
        break;
      }
    if (prime && n % p && nb % p) return p;
  }
  return 0;
}

uint32_t chunk_enc(uint32_t bytes) {
  uint32_t three = bytes % 3 == 0, base = three ? bytes / 3 : bytes, sh = 0;
  while ((1u << sh) < base) sh++;
  return (three ? 3u : 1u) << 16 | sh;
}

// the size-class table of halloc src/halloc.cu:363-394
bool build_classes(ha::Class *cls, uint32_t sb_bytes, const ha_opts_c &o) {
  for (uint32_t sid = 0; sid < ha::kNSizes; sid++) {
    ha::Class &c = cls[sid];
    uint32_t unit = 8u << (sid / 2), block = (sid & 1 ? 3 : 2) * unit;
    uint32_t per_slot = sid < 2 ? 4u : sid < 4 ? 2u : 1u;
    uint32_t nblocks = sb_bytes / block / per_slot * per_slot;
    c.chunk_id = (sid & 1) + (sid < ha::kNSizes / 2 ? 0 : 2);
    uint32_t cbytes = (c.chunk_id & 1 ? 3 : 2) * (c.chunk_id >= 2 ? 128 : 8);
    c.chunk_enc = chunk_enc(cbytes);
    c.ncib = block / cbytes;
    c.nchunks = nblocks * c.ncib;
    uint64_t span = (uint64_t)(nblocks / 256 + nblocks / 64) * g_hash_scale_pct / 100;
    if (span < 4) span = 4;
    if (span > nblocks) span = nblocks;
    uint32_t p = prime_below((uint32_t)span, nblocks);
    if (!p) return false;
    c.hash_step = c.ncib * p;
    c.roomy = (uint32_t)(o.roomy_fraction * c.nchunks);
    c.busy = (uint32_t)(o.busy_fraction * c.nchunks);
    c.sparse = (uint32_t)(o.sparse_fraction * c.nchunks);
  }
  return true;
}

// fastmod magic of a 32-bit divisor: floor((2^64 - 1) / d) + 1
uint64_t mod_magic(uint32_t d) { return ~0ull / d + 1; }

void build_magics(const ha::Class *cls, uint4 *mod) {
  for (uint32_t sid = 0; sid < ha::kNSizes; sid++) {
    uint64_t mn = mod_magic(cls[sid].nchunks), mh = mod_magic(cls[sid].hash_step);
    mod[sid] = make_uint4((uint32_t)mn, (uint32_t)(mn >> 32), (uint32_t)mh, (uint32_t)(mh >> 32));
  }
}

bool valid_fraction(double f) { return f >= 0.0 && f <= 1.0; }

// ---- virtual memory management (driver API through the runtime's entry
// points, so that the library needs no link against libcuda) --------------
struct Vmm {
  CUresult (*reserve)(CUdeviceptr *, size_t, size_t, CUdeviceptr, unsigned long long);
  CUresult (*free_va)(CUdeviceptr, size_t);
  CUresult (*create)(CUmemGenericAllocationHandle *, size_t, const CUmemAllocationProp *,
                     unsigned long long);
  CUresult (*release)(CUmemGenericAllocationHandle);
  CUresult (*map)(CUdeviceptr, size_t, size_t, CUmemGenericAllocationHandle,
                  unsigned long long);
  CUresult (*unmap)(CUdeviceptr, size_t);
  CUresult (*set_access)(CUdeviceptr, size_t, const CUmemAccessDesc *, size_t);
  CUresult (*granularity)(size_t *, const CUmemAllocationProp *,
                          CUmemAllocationGranularity_flags);
};

const Vmm *vmm() {
  static Vmm v;
  static int state = 0;  // 0 not tried, 1 ok, -1 unavailable
  if (state == 0) {
    struct {
      const char *name;
      void **fn;
    } tab[] = {{"cuMemAddressReserve", (void **)&v.reserve},
               {"cuMemAddressFree", (void **)&v.free_va},
               {"cuMemCreate", (void **)&v.create},
               {"cuMemRelease", (void **)&v.release},
               {"cuMemMap", (void **)&v.map},
               {"cuMemUnmap", (void **)&v.unmap},
               {"cuMemSetAccess", (void **)&v.set_access},
               {"cuMemGetAllocationGranularity", (void **)&v.granularity}};
    state = 1;
    for (auto &t : tab) {
      cudaDriverEntryPointQueryResult q;
      if (cudaGetDriverEntryPointByVersion(t.name, t.fn, 12000, cudaEnableDefault, &q) !=
              cudaSuccess ||
          q != cudaDriverEntryPointSuccess || !*t.fn) {
        cudaGetLastError();
        state = -1;
      }
    }
  }
  return state == 1 ? &v : nullptr;
}

CUmemAllocationProp unit_prop(int dev) {
  CUmemAllocationProp p;
  memset(&p, 0, sizeof(p));
  p.type = CU_MEM_ALLOCATION_TYPE_PINNED;
  p.location.type = CU_MEM_LOCATION_TYPE_DEVICE;
  p.location.id = dev;
  return p;
}

// Backs units [u, u + n) of h's pool with one allocation; false on a CUDA
// error (nothing left half done).
bool back_chunk(HostDev *h, int dev, uint32_t u, uint32_t n) {
  const Vmm *v = vmm();
  const CUmemAllocationProp prop = unit_prop(dev);
  const size_t bytes = (size_t)n * h->unit_bytes;
  CUmemGenericAllocationHandle hd = 0;
  if (v->create(&hd, bytes, &prop, 0) != CUDA_SUCCESS) return false;
  const CUdeviceptr at = (CUdeviceptr)(h->va + (uint64_t)u * h->unit_bytes);
  if (v->map(at, bytes, 0, hd, 0) != CUDA_SUCCESS) {
    v->release(hd);
    return false;
  }
  CUmemAccessDesc acc;
  memset(&acc, 0, sizeof(acc));
  acc.location = prop.location;
  acc.flags = CU_MEM_ACCESS_FLAGS_PROT_READWRITE;
  if (v->set_access(at, bytes, &acc, 1) != CUDA_SUCCESS) {
    v->unmap(at, bytes);
    v->release(hd);
    return false;
  }
  h->chunks[h->nchunks++] = {u, n, (unsigned long long)hd};
  memset(h->backed + u, 1, n);
  return true;
}

// Unbacks chunk i (the last chunk takes its place in the list).
void unback_chunk(HostDev *h, uint32_t i) {
  const Vmm *v = vmm();
  const HostDev::Chunk c = h->chunks[i];
  v->unmap((CUdeviceptr)(h->va + (uint64_t)c.first * h->unit_bytes),
           (size_t)c.n * h->unit_bytes);
  v->release((CUmemGenericAllocationHandle)c.handle);
  memset(h->backed + c.first, 0, c.n);
  h->chunks[i] = h->chunks[--h->nchunks];
}

// Unbacks every chunk and frees the reserved range.
void release_pool_range(HostDev *h) {
  const Vmm *v = vmm();
  if (!v || !h->va) return;
  while (h->nchunks) unback_chunk(h, h->nchunks - 1);
  v->free_va((CUdeviceptr)h->va, (size_t)h->nunits * h->unit_bytes);
  delete[] h->backed;
  delete[] h->chunks;
  h->backed = nullptr;
  h->chunks = nullptr;
  h->va = 0;
}

int shutdown_impl() {
  int dev;
  HostDev *h = current(&dev);
  if (!h) return HA_ECUDA;
  if (!h->init) return HA_ESTATE;
  HA_CK(cudaDeviceSynchronize());
  ha::Config zero;
  memset(&zero, 0, sizeof(zero));
  HA_CK(cudaMemcpyToSymbol(ha::c_cfg, &zero, sizeof(zero)));
  if (h->growth)
    release_pool_range(h);
  else
    HA_CK(cudaFree(h->raw_pool));
  HA_CK(cudaFree(h->meta));
  if (h->persist_bytes) {
    cudaCtxResetPersistingL2Cache();
    cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, 0);
    cudaGetLastError();
  }
  memset(h, 0, sizeof(*h));
  return HA_OK;
}

int init_impl(const ha_opts_c &o) {
  int dev;
  HostDev *h = current(&dev);
  if (!h) return HA_ECUDA;
  if (h->init) return HA_ESTATE;
  if (o.memory == 0 || o.sb_sz_sh < 20 || o.sb_sz_sh > 24 ||
      !(o.halloc_fraction > 0.0 && o.halloc_fraction <= 1.0) ||
      !valid_fraction(o.busy_fraction) || !valid_fraction(o.roomy_fraction) ||
      !valid_fraction(o.sparse_fraction))
    return HA_EINVAL;
  cudaDeviceProp prop;
  HA_CK(cudaGetDeviceProperties(&prop, dev));
  const uint32_t sb_sh = (uint32_t)o.sb_sz_sh, sb_bytes = 1u << sb_sh;
  uint64_t memory = o.memory;
  uint64_t cap = 3ull * prop.totalGlobalMem / 4ull;
  if (memory > cap) memory = cap;
  uint64_t slab_mem = (uint64_t)(o.halloc_fraction * (double)memory);
  uint64_t heap_mem = memory - slab_mem;
  uint64_t nsbs = slab_mem >> sb_sh;
  if (nsbs == 0) return HA_EINVAL;
  if (nsbs > ha::kMaxSlabs) return HA_ERANGE;

  ha::Class cls[ha::kNSizes];
  if (!build_classes(cls, sb_bytes, o)) return HA_EINVAL;
  uint4 mod[ha::kNSizes];
  build_magics(cls, mod);

  // CUDA heap for blocks above 3072 bytes.  The size cannot change once a
  // kernel of this context has used in-kernel malloc; the allocator still
  // works then, with the heap it has.
  bool heap_ok = cudaDeviceSetLimit(cudaLimitMallocHeapSize, heap_mem) == cudaSuccess;
  cudaGetLastError();

  char *raw = nullptr, *pool = nullptr;
  uint32_t *meta = nullptr;
  // growth: reserve the whole range, back the first units
  HostDev grow;
  memset(&grow, 0, sizeof(grow));
  uint32_t committed = (uint32_t)nsbs;
  if (g_growth_initial) {
    const Vmm *v = vmm();
    if (!v) return HA_ECUDA;
    const CUmemAllocationProp prop = unit_prop(dev);
    size_t gran = 0;
    if (v->granularity(&gran, &prop, CU_MEM_ALLOC_GRANULARITY_MINIMUM) != CUDA_SUCCESS ||
        gran == 0)
      return HA_ECUDA;
    const uint64_t unit = gran > sb_bytes ? gran : sb_bytes;
    if (unit % gran || unit % sb_bytes) return HA_EINVAL;
    grow.growth = true;
    grow.unit_bytes = unit;
    grow.spu = (uint32_t)(unit >> sb_sh);
    grow.nunits = (uint32_t)((nsbs << sb_sh) / unit);
    if (grow.nunits == 0) return HA_EINVAL;
    nsbs = (uint64_t)grow.nunits * grow.spu;
    grow.backed = new (std::nothrow) uint8_t[grow.nunits]();
    grow.chunks = new (std::nothrow) HostDev::Chunk[grow.nunits];
    if (!grow.backed || !grow.chunks) {
      delete[] grow.backed;
      delete[] grow.chunks;
      return HA_ECUDA;
    }
    CUdeviceptr va = 0;
    if (v->reserve(&va, (size_t)grow.nunits * unit, unit, 0, 0) != CUDA_SUCCESS) {
      delete[] grow.backed;
      delete[] grow.chunks;
      return HA_ECUDA;
    }
    grow.va = va;
    uint64_t want = (g_growth_initial + unit - 1) / unit;
    if (want > grow.nunits) want = grow.nunits;
    if (!back_chunk(&grow, dev, 0, (uint32_t)want)) {
      release_pool_range(&grow);
      return HA_ECUDA;
    }
    committed = (uint32_t)want * grow.spu;
    pool = (char *)va;
  }
  const uint64_t pool_bytes = nsbs << sb_sh;
  if (!grow.growth) {
    if (cudaMalloc(&raw, pool_bytes + sb_bytes) != cudaSuccess) {
      cudaGetLastError();
      return HA_ECUDA;
    }
    pool = (char *)(((uintptr_t)raw + sb_bytes - 1) & ~(uintptr_t)(sb_bytes - 1));
  }
  auto free_pool = [&]() {
    if (grow.growth)
      release_pool_range(&grow);
    else
      cudaFree(raw);
  };
  const size_t bit_words = (size_t)nsbs << (sb_sh - 9);
  const size_t nib_words = (size_t)nsbs << (sb_sh - 7);
  const size_t meta_bytes = (bit_words + nib_words) * 4;
  if (cudaMalloc(&meta, meta_bytes) != cudaSuccess) {
    cudaGetLastError();
    free_pool();
    return HA_ECUDA;
  }
  int rc = HA_OK;
  ha::State *st = new (std::nothrow) ha::State;
  if (!st) rc = HA_ECUDA;
  if (rc == HA_OK) {
    memset(st, 0, sizeof(*st));
    for (uint32_t s = 0; s < ha::kMaxHeads * ha::kNSizes; s++) {
      st->ticket[s * ha::kTicketStride] = ha::kFirstTicket;
      st->head[s] = ha::kSlabField;  // no head, surge level 0
      st->cached[s] = ha::kNone;
    }
    st->wait_limit_us = ha::kDefaultWaitUs;
    st->committed = committed;
    st->n_free = committed;  // every backed slab starts in the free set
    for (uint32_t sb = 0; sb < nsbs; sb++) {
      st->ctr[sb * ha::kCtrStride] = ha::kCtrInit;
      st->desc[sb].size_id = ha::kNone;
      st->desc[sb].chunk_id = ha::kNone;
      if (sb >= committed) continue;  // not backed yet: in no set
      st->sets[ha::kSetFree][sb >> 5] |= 1u << (sb & 31);
      st->sums[ha::kSetFree][sb >> 10] |= 1u << ((sb >> 5) & 31);
    }
    ha::Config cfg;
    memset(&cfg, 0, sizeof(cfg));
    cfg.pool = pool;
    cfg.pool_bytes = pool_bytes;
    cfg.bits = meta;
    cfg.nibs = meta + bit_words;
    cfg.nsbs = (uint32_t)nsbs;
    cfg.sb_sh = sb_sh;
    cfg.bit_words_sh = sb_sh - 9;
    cfg.nib_words_sh = sb_sh - 7;
    cfg.set_words = (uint32_t)((nsbs + 31) / 32);
    cfg.sum_words = (cfg.set_words + 31) / 32;
    cfg.nheads = heads_for_init();
    cfg.surge = surge_for_init(cfg.nheads);
    cfg.growth = grow.growth ? 1 : 0;
    if (HA_SPEC_COMMIT) {
      const uint64_t resident =
          (uint64_t)prop.multiProcessorCount * (uint64_t)prop.maxThreadsPerMultiProcessor;
      for (uint32_t s = 0; s < ha::kNSizes; s++)
        if (cls[s].ncib == 1 && cls[s].nchunks + resident < (1ull << (32 - ha::kCntShift)))
          cfg.spec_mask |= 1u << s;
    }
    if (cudaMemset(meta, 0, meta_bytes) != cudaSuccess ||
        cudaMemcpyToSymbol(ha::g_cls, cls, sizeof(cls)) != cudaSuccess ||
        cudaMemcpyToSymbol(ha::g_mod, mod, sizeof(mod)) != cudaSuccess ||
        cudaMemcpyToSymbol(ha::g_st, st, sizeof(*st)) != cudaSuccess ||
        cudaMemcpyToSymbol(ha::c_cfg, &cfg, sizeof(cfg)) != cudaSuccess ||
        cudaDeviceSynchronize() != cudaSuccess) {
      cudaGetLastError();
      rc = HA_ECUDA;
    }
  }
  delete st;
  if (rc != HA_OK) {
    free_pool();
    cudaFree(meta);
    return rc;
  }
  // persisting-L2 carve-out for the slab metadata (a context limit; it is
  // released by ha_shutdown and by context teardown)
  size_t persist = 0;
  if (prop.persistingL2CacheMaxSize > 0) {
    persist = meta_bytes < (size_t)prop.persistingL2CacheMaxSize
                  ? meta_bytes
                  : (size_t)prop.persistingL2CacheMaxSize;
    if (cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, persist) != cudaSuccess) {
      cudaGetLastError();
      persist = 0;
    }
  }
  h->init = true;
  h->raw_pool = raw;
  h->pool = pool;
  h->pool_bytes = pool_bytes;
  h->meta = meta;
  h->meta_bytes = meta_bytes;
  h->heap_bytes = heap_mem;
  h->nsbs = (uint32_t)nsbs;
  h->sb_sh = sb_sh;
  h->heap_ok = heap_ok;
  h->persist_bytes = persist;
  if (grow.growth) {
    // load the adopt kernel now: with lazy module loading its first launch
    // would otherwise wait for kernels already running, and ha_grow_c is
    // meant to be called while a persistent kernel waits for the slabs
    cudaFuncAttributes fa;
    if (cudaFuncGetAttributes(&fa, ha_adopt_k) != cudaSuccess) cudaGetLastError();
  }
  h->growth = grow.growth;
  h->va = grow.va;
  h->unit_bytes = grow.growth ? grow.unit_bytes : pool_bytes;
  h->spu = grow.spu;
  h->nunits = grow.nunits;
  h->backed = grow.backed;
  h->chunks = grow.chunks;
  h->nchunks = grow.nchunks;
  return HA_OK;
}

ha_opts_c to_c(const halloc_opts_t &o) {
  ha_opts_c c;
  c.memory = o.memory;
  c.halloc_fraction = o.halloc_fraction;
  c.busy_fraction = o.busy_fraction;
  c.roomy_fraction = o.roomy_fraction;
  c.sparse_fraction = o.sparse_fraction;
  c.sb_sz_sh = o.sb_sz_sh;
  return c;
}

}  // namespace

// ---- growth kernels ----------------------------------------------------------

// newly backed slabs [first, first + count) join the free set
__global__ void ha_adopt_k(uint32_t first, uint32_t count) {
  using namespace ha;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < count) set_put_free(first + i);
  if (i == 0) red_add(&g_st.committed, count);
}

// One thread per candidate chunk g_trim_chunks[i] (first slab, slab count):
// takes every slab of the chunk out of the free set; the chunk is released
// when all of them were there and are empty, non-head slabs with no chunk
// size, and when it fits in max_slabs; otherwise the slabs taken go back.
// Released chunks are listed in g_trim_out[0 .. g_trim_n).
// Closes every size's surge head sets (ha_close_surges_c): level 0 in each
// size's set-0 head word, then the heads and prefetched slabs of sets 1..
// filed by occupancy.  One thread; every lock wait is bounded.
__global__ void ha_close_surges_k() {
  using namespace ha;
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  for (uint32_t sid = 0; sid < kNSizes; sid++) {
    uint32_t *hlock0 = &g_st.head_lock[sid * kTicketStride];
    if (lock(hlock0)) {
      const uint32_t w = ld_relaxed(&g_st.head[sid]);
      if (head_level(w) != 0) {
        st_release(&g_st.head[sid], head_word(head_slab(w), 0));
        red_add(&g_st.n_surge_changes, 1);
      }
      unlock(hlock0);
    }
    for (uint32_t k = 1; k < kMaxHeads; k++) retire_set(k * kNSizes + sid, true);
  }
}

__global__ void ha_trim_k(uint32_t ncand, uint32_t max_slabs) {
  using namespace ha;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ncand) return;
  const uint32_t first = g_trim_chunks[i].x, n = g_trim_chunks[i].y;
  uint32_t taken = 0;
  bool ok = true;
  for (; taken < n; taken++)
    if (!set_claim(kSetFree, first + taken)) {
      ok = false;
      break;
    }
  for (uint32_t k = 0; k < n && ok; k++) {
    const uint32_t sb = first + k, c = ld_relaxed(ctr_of(sb));
    ok = (c >> kCntShift) == 0 && !(c & kHeadFlag) &&
         ((c >> kChunkShift) & kChunkField) == kChunkField &&
         !ld_relaxed(&g_st.desc[sb].is_head);
  }
  if (ok) {
    const uint32_t before = atomicAdd(&g_trim_slabs, n);
    if (before + n <= max_slabs) {
      g_trim_out[atomicAdd(&g_trim_n, 1u)] = i;
      red_add(&g_st.committed, 0u - n);
      return;
    }
    atomicSub(&g_trim_slabs, n);
  }
  for (uint32_t k = 0; k < taken; k++) set_put_free(first + k);
}

// ---- statistics kernels ----------------------------------------------------

// one thread per slab: used chunks/bytes, free and head slabs
// (the per-slab sum of halloc src/statistics.cuh:34-48, as a reduction)
__global__ void ha_stats_k(int ideal) {
  using namespace ha;
  __shared__ unsigned long long s_chunks, s_bytes, s_free, s_ideal;
  __shared__ unsigned int s_fslabs, s_hslabs;
  if (threadIdx.x == 0) {
    s_chunks = s_bytes = s_free = s_ideal = 0;
    s_fslabs = s_hslabs = 0;
  }
  __syncthreads();
  uint32_t sb = blockIdx.x * blockDim.x + threadIdx.x;
  if (sb < c_cfg.nsbs) {
    uint32_t used = ld_relaxed(ctr_of(sb)) >> kCntShift;
    uint32_t enc = ld_relaxed(&g_st.desc[sb].chunk_enc);
    uint64_t ubytes = enc ? (uint64_t)chunk_mul(used, enc) : 0;
    uint64_t sbb = 1ull << c_cfg.sb_sh;
    atomicAdd(&s_chunks, (unsigned long long)used);
    atomicAdd(&s_bytes, (unsigned long long)ubytes);
    atomicAdd(&s_free, (unsigned long long)(sbb - ubytes));
    if (ideal && enc == 0) atomicAdd(&s_ideal, (unsigned long long)sbb);
    if ((ld_relaxed(&g_st.sets[kSetFree][sb >> 5]) >> (sb & 31)) & 1u) atomicAdd(&s_fslabs, 1u);
    if (ld_relaxed(&g_st.desc[sb].is_head)) atomicAdd(&s_hslabs, 1u);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    atomicAdd(&g_stats_out.used_chunks, s_chunks);
    atomicAdd(&g_stats_out.used_bytes, s_bytes);
    atomicAdd(&g_stats_out.free_bytes, s_free);
    atomicAdd(&g_stats_out.ideal_bytes, s_ideal);
    atomicAdd(&g_stats_out.free_slabs, s_fslabs);
    atomicAdd(&g_stats_out.head_slabs, s_hslabs);
  }
}

// largest block the CUDA heap can give, by bisection on in-kernel malloc
// (halloc src/statistics.cuh:14-30; like the original it reports the last
// midpoint tried)
__global__ void ha_max_alloc_k(unsigned long long heap) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  unsigned long long hi = heap, lo = 0, mid = 0;
  const unsigned long long step = 1ull << 20;
  while (hi - lo > step) {
    mid = (hi + lo) / 2;
    void *p = malloc(mid);
    if (p) {
      lo = mid;
      free(p);
    } else {
      hi = mid;
    }
  }
  ha::g_max_alloc = mid;
}

namespace {
int run_stats(int ideal, ha::StatsOut *out) {
  HostDev *h = current();
  if (!h) return HA_ECUDA;
  if (!h->init) return HA_ESTATE;
  ha::StatsOut zero;
  memset(&zero, 0, sizeof(zero));
  HA_CK(cudaMemcpyToSymbol(ha::g_stats_out, &zero, sizeof(zero)));
  ha_stats_k<<<(h->nsbs + 127) / 128, 128>>>(ideal);
  HA_CK(cudaGetLastError());
  HA_CK(cudaMemcpyFromSymbol(out, ha::g_stats_out, sizeof(*out)));
  return HA_OK;
}
}  // namespace

// ---- C++ API (halloc.h) ------------------------------------------------------

void ha_init(halloc_opts_t opts) {
  HostDev *h = current();
  if (h && h->init) shutdown_impl();
  ha_opts_c c = to_c(opts);
  int rc = init_impl(c);
  if (rc != HA_OK) {
    fprintf(stderr, "halloc-b200: ha_init failed (%d)\n", rc);
    exit(-1);
  }
}

void ha_shutdown(void) { shutdown_impl(); }

double ha_extfrag(bool ideal) { return ha_extfrag_c(ideal ? 1 : 0); }

// ---- C ABI: init / stats layer ----------------------------------------------

extern "C" int ha_init_c(const ha_opts_c *opts) {
  if (!opts) return HA_EINVAL;
  return init_impl(*opts);
}

extern "C" int ha_shutdown_c(void) { return shutdown_impl(); }

extern "C" double ha_extfrag_c(int ideal) {
  HostDev *h = current();
  if (!h || !h->init) return -1.0;
  unsigned long long zero = 0;
  if (cudaMemcpyToSymbol(ha::g_max_alloc, &zero, sizeof(zero)) != cudaSuccess) return -1.0;
  ha_max_alloc_k<<<1, 32>>>(h->heap_bytes);
  if (cudaGetLastError() != cudaSuccess) return -1.0;
  ha::StatsOut s;
  if (run_stats(ideal, &s) != HA_OK) return -1.0;
  unsigned long long max_alloc = 0;
  if (cudaMemcpyFromSymbol(&max_alloc, ha::g_max_alloc, sizeof(max_alloc)) != cudaSuccess)
    return -1.0;
  double free_mem = (double)s.free_bytes + (double)h->heap_bytes;
  double best = (double)max_alloc + (double)s.ideal_bytes;
  return free_mem > 0 ? 1.0 - best / free_mem : 0.0;
}

extern "C" int ha_stats_c(ha_stats_t *out) {
  if (!out) return HA_EINVAL;
  HostDev *h = current();
  if (!h) return HA_ECUDA;
  if (!h->init) return HA_ESTATE;
  ha::StatsOut s;
  int rc = run_stats(0, &s);
  if (rc) return rc;
  uint32_t head[ha::kNSizes], cached[ha::kNSizes], misc[7];
  HA_CK(cudaMemcpyFromSymbol(head, ha::g_st, sizeof(head), offsetof(ha::State, head)));
  HA_CK(cudaMemcpyFromSymbol(cached, ha::g_st, sizeof(cached), offsetof(ha::State, cached)));
  HA_CK(cudaMemcpyFromSymbol(misc, ha::g_st, sizeof(misc), offsetof(ha::State, status)));
  memset(out, 0, sizeof(*out));
  out->pool_base = (uint64_t)(uintptr_t)h->pool;
  out->pool_bytes = h->pool_bytes;
  out->cuda_heap_bytes = h->heap_bytes;
  out->used_chunks = s.used_chunks;
  out->used_bytes = s.used_bytes;
  out->nsbs = h->nsbs;
  out->sb_sz = 1u << h->sb_sh;
  out->free_slabs = s.free_slabs;
  out->head_slabs = s.head_slabs;
  out->status = misc[0];
  out->n_head_changes = misc[2];
  out->n_null = misc[3];
  out->heap_limit_ok = h->heap_ok ? 1 : 0;
  for (uint32_t k = 0; k < ha::kNSizes; k++) {
    out->head[k] = decode_head(head[k]);
    out->surge_level[k] = head[k] >> ha::kLevelShift;
  }
  memcpy(out->cached, cached, sizeof(cached));
  out->n_surge_changes = misc[5];
  out->free_count = misc[6];
  out->growth = h->growth ? 1 : 0;
  out->committed_slabs = misc[4];
  out->unit_bytes = h->unit_bytes;
  return HA_OK;
}

extern "C" int ha_set_growth_c(uint64_t initial_bytes) {
  g_growth_initial = initial_bytes;
  return HA_OK;
}

extern "C" int ha_grow_c(uint64_t bytes, void *stream, uint64_t *added_bytes) {
  if (added_bytes) *added_bytes = 0;
  int dev;
  HostDev *h = current(&dev);
  if (!h) return HA_ECUDA;
  if (!h->init || !h->growth) return HA_ESTATE;
  uint64_t want = (bytes + h->unit_bytes - 1) / h->unit_bytes;
  if (want == 0) want = 1;
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  uint64_t added = 0;
  // lowest unbacked runs first, one chunk per run
  for (uint32_t u = 0; u < h->nunits && added < want;) {
    if (h->backed[u]) {
      u++;
      continue;
    }
    uint32_t n = 0;
    while (u + n < h->nunits && !h->backed[u + n] && added + n < want) n++;
    if (!back_chunk(h, dev, u, n)) break;
    const uint32_t count = n * h->spu;
    ha_adopt_k<<<(count + 127) / 128, 128, 0, s>>>(u * h->spu, count);
    if (cudaGetLastError() != cudaSuccess) return HA_ECUDA;
    added += n;
    u += n;
  }
  if (added_bytes) *added_bytes = added * h->unit_bytes;
  if (added == 0) {
    for (uint32_t u = 0; u < h->nunits; u++)
      if (!h->backed[u]) return HA_ECUDA;  // there was room: a CUDA call failed
    return HA_ERANGE;
  }
  return HA_OK;
}

extern "C" int ha_close_surges_c(void *stream) {
  HostDev *h = current();
  if (!h) return HA_ECUDA;
  if (!h->init) return HA_ESTATE;
  ha_close_surges_k<<<1, 1, 0, reinterpret_cast<cudaStream_t>(stream)>>>();
  HA_CK(cudaGetLastError());
  return HA_OK;
}

extern "C" int ha_trim_c(uint64_t max_bytes, void *stream, uint64_t *released_bytes) {
  if (released_bytes) *released_bytes = 0;
  HostDev *h = current();
  if (!h) return HA_ECUDA;
  if (!h->init || !h->growth) return HA_ESTATE;
  const uint64_t max_units = max_bytes / h->unit_bytes;
  if (max_units == 0 || h->nchunks == 0) return HA_OK;
  const uint64_t max_slabs64 = max_units * h->spu;
  const uint32_t max_slabs = max_slabs64 > 0xffffffffull ? 0xffffffffu : (uint32_t)max_slabs64;
  const uint32_t ncand = h->nchunks;
  uint2 *cand = new (std::nothrow) uint2[ncand];
  uint32_t *out = new (std::nothrow) uint32_t[ncand];
  if (!cand || !out) {
    delete[] cand;
    delete[] out;
    return HA_ECUDA;
  }
  for (uint32_t i = 0; i < ncand; i++)
    cand[i] = make_uint2(h->chunks[i].first * h->spu, h->chunks[i].n * h->spu);
  cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  uint32_t zero2[2] = {0, 0}, n = 0;
  int rc = HA_OK;
  if (cudaMemcpyToSymbolAsync(ha::g_trim_chunks, cand, ncand * sizeof(uint2), 0,
                              cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyToSymbolAsync(ha::g_trim_n, &zero2[0], sizeof(uint32_t), 0,
                              cudaMemcpyHostToDevice, s) != cudaSuccess ||
      cudaMemcpyToSymbolAsync(ha::g_trim_slabs, &zero2[1], sizeof(uint32_t), 0,
                              cudaMemcpyHostToDevice, s) != cudaSuccess)
    rc = HA_ECUDA;
  if (rc == HA_OK) {
    // surge heads hold slabs that would otherwise be wholly free
    ha_close_surges_k<<<1, 1, 0, s>>>();
    ha_trim_k<<<(ncand + 127) / 128, 128, 0, s>>>(ncand, max_slabs);
    if (cudaGetLastError() != cudaSuccess ||
        cudaMemcpyFromSymbolAsync(&n, ha::g_trim_n, sizeof(n), 0, cudaMemcpyDeviceToHost, s) !=
            cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess)
      rc = HA_ECUDA;
  }
  if (rc == HA_OK && n) {
    if (cudaMemcpyFromSymbolAsync(out, ha::g_trim_out, n * sizeof(uint32_t), 0,
                                  cudaMemcpyDeviceToHost, s) != cudaSuccess ||
        cudaStreamSynchronize(s) != cudaSuccess) {
      rc = HA_ECUDA;
    } else {
      // released chunks by their index in the candidate list; unback the
      // highest index first so that swapping the last chunk into a freed
      // place never moves a chunk still to be released
      uint64_t units = 0;
      for (uint32_t k = 0; k < n; k++) units += h->chunks[out[k]].n;
      for (uint32_t a = 0; a < n; a++)
        for (uint32_t b = a + 1; b < n; b++)
          if (out[b] > out[a]) {
            const uint32_t t = out[a];
            out[a] = out[b];
            out[b] = t;
          }
      for (uint32_t k = 0; k < n; k++) unback_chunk(h, out[k]);
      if (released_bytes) *released_bytes = units * h->unit_bytes;
    }
  }
  delete[] cand;
  delete[] out;
  return rc;
}

extern "C" uint32_t ha_status_c(void) {
  uint32_t st = 0;
  if (cudaMemcpyFromSymbol(&st, ha::g_st, sizeof(st), offsetof(ha::State, status)) !=
      cudaSuccess) {
    cudaGetLastError();
    return 0xffffffffu;
  }
  return st;
}

extern "C" int ha_clear_status_c(void) {
  uint32_t z = 0;
  HA_CK(cudaMemcpyToSymbol(ha::g_st, &z, sizeof(z), offsetof(ha::State, status)));
  return HA_OK;
}

extern "C" int ha_set_wait_limit_c(uint32_t microseconds) {
  if (microseconds == 0) return HA_EINVAL;
  HA_CK(cudaMemcpyToSymbol(ha::g_st, &microseconds, sizeof(microseconds),
                           offsetof(ha::State, wait_limit_us)));
  return HA_OK;
}

extern "C" int ha_dump_state_c(const ha_state_dump_t *d) {
  if (!d) return HA_EINVAL;
  HostDev *h = current();
  if (!h) return HA_ECUDA;
  if (!h->init) return HA_ESTATE;
  HA_CK(cudaDeviceSynchronize());
  ha::State *st = new (std::nothrow) ha::State;
  if (!st) return HA_ECUDA;
  if (cudaMemcpyFromSymbol(st, ha::g_st, sizeof(*st)) != cudaSuccess) {
    delete st;
    return HA_ECUDA;
  }
  const uint32_t n = h->nsbs, nw = (n + 31) / 32;
  for (uint32_t s = 0; s < ha::kNSizes; s++) {
    if (d->tickets) d->tickets[s] = st->ticket[s * ha::kTicketStride];
    if (d->heads) d->heads[s] = decode_head(st->head[s]);
    if (d->cached) d->cached[s] = st->cached[s];
  }
  for (uint32_t sb = 0; sb < n; sb++) {
    if (d->counters) d->counters[sb] = st->ctr[sb * ha::kCtrStride];
    if (d->size_id) d->size_id[sb] = st->desc[sb].size_id;
    if (d->chunk_id) d->chunk_id[sb] = st->desc[sb].chunk_id;
    if (d->is_head) d->is_head[sb] = st->desc[sb].is_head;
    if (d->chunk_enc) d->chunk_enc[sb] = st->desc[sb].chunk_enc;
  }
  if (d->sets)
    for (uint32_t k = 0; k < ha::kNSets; k++)
      memcpy(d->sets + (size_t)k * nw, st->sets[k], nw * 4);
  delete st;
  if (d->size_infos) HA_CK(cudaMemcpyFromSymbol(d->size_infos, ha::g_cls, sizeof(ha::Class) * ha::kNSizes));
  const size_t bit_words = (size_t)n << (h->sb_sh - 9);
  const size_t nib_words = (size_t)n << (h->sb_sh - 7);
  if (d->bits) HA_CK(cudaMemcpy(d->bits, h->meta, bit_words * 4, cudaMemcpyDeviceToHost));
  if (d->nibbles)
    HA_CK(cudaMemcpy(d->nibbles, h->meta + bit_words, nib_words * 4, cudaMemcpyDeviceToHost));
  return HA_OK;
}

extern "C" int ha_set_heads_c(uint32_t nheads) {
  if (nheads == 0 || nheads > ha::kMaxHeads || (nheads & (nheads - 1))) return HA_EINVAL;
  g_nheads = nheads;
  g_nheads_set = true;
  return HA_OK;
}

extern "C" int ha_set_surge_c(int on) {
  if (on < -1 || on > 1) return HA_EINVAL;
  g_surge = on;
  return HA_OK;
}

extern "C" int ha_set_hash_scale_c(uint32_t percent) {
  if (percent < 10 || percent > 1000) return HA_EINVAL;
  g_hash_scale_pct = percent;
  return HA_OK;
}

#if HA_PROBE_STATS
// Instrumented builds only: the probe counters (ha_stamp.cuh ProbeStat order)
// summed over their copies into out[0 .. kPsCount - 1]; reset != 0 zeroes
// them.  Waits for the device.
extern "C" int ha_probe_stats_c(unsigned long long *out, int reset) {
  if (!out) return HA_EINVAL;
  unsigned long long h[ha::kPsCopies * ha::kPsStride];
  HA_CK(cudaDeviceSynchronize());
  HA_CK(cudaMemcpyFromSymbol(h, ha::g_pstats, sizeof(h)));
  for (uint32_t i = 0; i < ha::kPsCount; i++) {
    out[i] = 0;
    for (uint32_t c = 0; c < ha::kPsCopies; c++) out[i] += h[c * ha::kPsStride + i];
  }
  if (reset) {
    memset(h, 0, sizeof(h));
    HA_CK(cudaMemcpyToSymbol(ha::g_pstats, h, sizeof(h)));
  }
  return HA_OK;
}
#endif

extern "C" int ha_debug_set_head_lock_c(uint32_t size_id, uint32_t held) {
  if (size_id >= ha::kNSizes || held > 1) return HA_EINVAL;
  HostDev *h = current();
  if (!h) return HA_ECUDA;
  if (!h->init) return HA_ESTATE;
  HA_CK(cudaDeviceSynchronize());
  HA_CK(cudaMemcpyToSymbol(ha::g_st, &held, sizeof(held),
                           offsetof(ha::State, head_lock) +
                               sizeof(uint32_t) * size_id * ha::kTicketStride));
  return HA_OK;
}

extern "C" int ha_l2_persist_c(void *stream) {
  HostDev *h = current();
  if (!h) return HA_ECUDA;
  if (!h->init) return HA_ESTATE;
  if (!h->persist_bytes) return HA_OK;  // no persisting L2 on this device
  int dev;
  HA_CK(cudaGetDevice(&dev));
  int max_window = 0;
  HA_CK(cudaDeviceGetAttribute(&max_window, cudaDevAttrMaxAccessPolicyWindowSize, dev));
  cudaStreamAttrValue v;
  memset(&v, 0, sizeof(v));
  size_t win = h->meta_bytes < (size_t)max_window ? h->meta_bytes : (size_t)max_window;
  v.accessPolicyWindow.base_ptr = h->meta;
  v.accessPolicyWindow.num_bytes = win;
  v.accessPolicyWindow.hitRatio = win ? (float)fmin(1.0, (double)h->persist_bytes / (double)win) : 0.f;
  v.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
  v.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
  HA_CK(cudaStreamSetAttribute((cudaStream_t)stream, cudaStreamAttributeAccessPolicyWindow, &v));
  return HA_OK;
}
