// ha_samples.cu -- the reference's sample programs as workloads of the C ABI
// (halloc_c.h): grid-points (samples/grid-points/grid-points.cu) and
// add-strings (samples/add-strings/add-strings.cu).  Each step is its own
// entry point so that a caller can time it; the check entry points read the
// results back on the device for the tests.
#include <cuda_runtime.h>
#include <limits.h>
#include <stdint.h>
#include <stdio.h>

#include "halloc.h"
#include "halloc_c.h"

namespace {

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

__device__ __forceinline__ uint32_t mix32(uint32_t x) {
  x ^= x >> 16;
  x *= 0x7feb352du;
  x ^= x >> 15;
  x *= 0x846ca68bu;
  x ^= x >> 16;
  return x;
}

// ---- grid-points -------------------------------------------------------------
//
// One thread per point: a 16-byte list node from hamalloc (or from a
// pre-allocated array, the sample's comparison mode) is pushed onto the list
// of the point's grid cell with an atomic exchange
// (grid-points.cu:82-137).  One thread per cell then walks the cell's list
// and frees its nodes (grid-points.cu:101-153).

struct PointNode {
  int ip;
  PointNode *next;
};
static_assert(sizeof(PointNode) == 16, "one 16-byte block per node");

__device__ __forceinline__ uint32_t cell_of(const float *pts, uint32_t ip, uint32_t ncells) {
  const int nc = (int)ncells;
  int c[3];
  for (int d = 0; d < 3; d++) {
    const int v = (int)floorf(pts[3 * (size_t)ip + d] * (float)nc);
    c[d] = max(min(v, nc - 1), 0);
  }
  return (uint32_t)(c[0] + nc * (c[1] + nc * c[2]));
}

__global__ void ha_grid_insert_k(uint32_t n, uint32_t ncells, const float *__restrict__ pts,
                                 PointNode **grid, PointNode *pre, unsigned long long *nfail) {
  const uint32_t ip = blockIdx.x * blockDim.x + threadIdx.x;
  if (ip >= n) return;
  PointNode *node = pre ? pre + ip : static_cast<PointNode *>(hamalloc(sizeof(PointNode)));
  if (!node) {
    atomicAdd(nfail, 1ull);
    return;
  }
  node->ip = (int)ip;
  unsigned long long *cell = reinterpret_cast<unsigned long long *>(grid + cell_of(pts, ip, ncells));
  // publish the node after its fields: the exchange is a release
  __threadfence();
  const unsigned long long old = atomicExch(cell, (unsigned long long)(uintptr_t)node);
  node->next = reinterpret_cast<PointNode *>((uintptr_t)old);
}

// per cell: number of points and the sum of mix32(point index)
__global__ void ha_grid_check_k(uint32_t ncells3, PointNode *const *grid, uint32_t *count,
                                unsigned long long *hsum) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ncells3) return;
  uint32_t c = 0;
  unsigned long long h = 0;
  for (const PointNode *p = grid[i]; p && c <= (1u << 30); p = p->next) {
    c++;
    h += mix32((uint32_t)p->ip);
  }
  count[i] = c;
  hsum[i] = h;
}

__global__ void ha_grid_free_k(uint32_t ncells3, PointNode **grid, int pre) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= ncells3) return;
  PointNode *p = grid[i];
  grid[i] = nullptr;
  if (pre) return;
  while (p) {
    PointNode *nx = p->next;
    hafree(p);
    p = nx;
  }
}

// ---- add-strings -------------------------------------------------------------
//
// Strings of spaces, zero-terminated, in blocks from hamalloc; every block is
// at least 8-byte aligned and a multiple of 8 bytes long, so strings are read
// and written as 64-bit words (add-strings.cu:71-205).

// first zero byte of v (8 when none)
__device__ __forceinline__ uint32_t zero_byte(uint64_t v) {
  const uint64_t t = (v - 0x0101010101010101ull) & ~v & 0x8080808080808080ull;
  return t ? (uint32_t)(__ffsll((long long)t) - 1) >> 3 : 8u;
}

__device__ __forceinline__ uint32_t dstrlen(const uint64_t *s) {
  for (uint32_t k = 0;; k++) {
    const uint32_t z = zero_byte(s[k]);
    if (z < 8) return 8 * k + z;
  }
}

__global__ void ha_strings_alloc_k(uint32_t n, const int *__restrict__ lens, char **strs,
                                   unsigned long long *nfail) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t l = (uint32_t)lens[i];
  // l + 1 bytes rounded up to whole words: the same size class for blocks up
  // to 3 KiB, and room for the last word in CUDA's heap above that
  uint64_t *s = static_cast<uint64_t *>(hamalloc(8 * (l / 8 + 1)));
  strs[i] = reinterpret_cast<char *>(s);
  if (!s) {
    atomicAdd(nfail, 1ull);
    return;
  }
  const uint32_t words = l / 8 + 1;  // the word holding the zero byte is the last
  for (uint32_t k = 0; k + 1 < words; k++) s[k] = 0x2020202020202020ull;
  const uint32_t tail = l % 8;       // spaces in the last word
  s[words - 1] = tail ? 0x2020202020202020ull >> (8 * (8 - tail)) : 0ull;
}

// c = a followed by b: word k of c takes a's word k while a covers it, then
// a's tail and b's head, then b's words shifted by a's length modulo 8
__global__ void ha_strings_concat_k(uint32_t n, char **c, char *const *a, char *const *b,
                                    unsigned long long *nfail) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t *sa = reinterpret_cast<const uint64_t *>(a[i]);
  const uint64_t *sb = reinterpret_cast<const uint64_t *>(b[i]);
  if (!sa || !sb) {
    c[i] = nullptr;
    atomicAdd(nfail, 1ull);
    return;
  }
  const uint32_t la = dstrlen(sa), lb = dstrlen(sb), lc = la + lb;
  uint64_t *sc = static_cast<uint64_t *>(hamalloc(8 * (lc / 8 + 1)));
  c[i] = reinterpret_cast<char *>(sc);
  if (!sc) {
    atomicAdd(nfail, 1ull);
    return;
  }
  const uint32_t bwords = lb / 8 + 1;  // words of b up to and including its zero byte
  auto bword = [&](uint32_t j) -> uint64_t { return j < bwords ? sb[j] : 0ull; };
  const uint32_t sh = la % 8, ka = la / 8;
  const uint32_t cwords = lc / 8 + 1;
  for (uint32_t k = 0; k < cwords; k++) {
    uint64_t w;
    if (k < ka) {
      w = sa[k];
    } else if (k == ka) {
      const uint64_t keep = sh ? sa[k] & ((1ull << (8 * sh)) - 1) : 0ull;
      w = keep | (bword(0) << (8 * sh));
    } else {
      const uint32_t j = k - ka;  // b bytes from 8 * j - sh
      w = sh ? (bword(j - 1) >> (8 * (8 - sh))) | (bword(j) << (8 * sh)) : bword(j);
    }
    if (k == cwords - 1) {  // clear whatever follows the zero byte
      const uint32_t z = lc % 8;
      w &= z ? ((1ull << (8 * z)) - 1) : 0ull;
    }
    sc[k] = w;
  }
}

__global__ void ha_strings_free_k(uint32_t n, char **strs) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  hafree(strs[i]);
  strs[i] = nullptr;
}

// counts strings that are not la[i] + lb[i] spaces followed by a zero byte
__global__ void ha_strings_check_k(uint32_t n, char *const *c, const int *la, const int *lb,
                                   unsigned long long *bad) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const char *s = c[i];
  const uint32_t want = (uint32_t)(la[i] + lb[i]);
  bool ok = s != nullptr;
  for (uint32_t k = 0; ok && k < want; k++) ok = s[k] == ' ';
  if (ok) ok = s[want] == 0;
  if (!ok) atomicAdd(bad, 1ull);
}

}  // namespace

extern "C" int ha_grid_insert_c(uint32_t n, uint32_t ncells, const float *pts, void **grid,
                                void *pre_nodes, uint64_t *nfail, void *stream) {
  if (!pts || !grid || !nfail || ncells == 0 || ncells > 1024) return HA_EINVAL;
  if (n == 0) return HA_OK;
  ha_grid_insert_k<<<blocks_for(n, 128), 128, 0, as_stream(stream)>>>(
      n, ncells, pts, reinterpret_cast<PointNode **>(grid),
      static_cast<PointNode *>(pre_nodes), reinterpret_cast<unsigned long long *>(nfail));
  return launch_status();
}

extern "C" int ha_grid_check_c(uint32_t ncells, void *const *grid, uint32_t *count,
                               uint64_t *hsum, void *stream) {
  if (!grid || !count || !hsum || ncells == 0 || ncells > 1024) return HA_EINVAL;
  const uint32_t n3 = ncells * ncells * ncells;
  ha_grid_check_k<<<blocks_for(n3, 128), 128, 0, as_stream(stream)>>>(
      n3, reinterpret_cast<PointNode *const *>(grid), count,
      reinterpret_cast<unsigned long long *>(hsum));
  return launch_status();
}

extern "C" int ha_grid_free_c(uint32_t ncells, void **grid, int pre_nodes, void *stream) {
  if (!grid || ncells == 0 || ncells > 1024) return HA_EINVAL;
  const uint32_t n3 = ncells * ncells * ncells;
  ha_grid_free_k<<<blocks_for(n3, 128), 128, 0, as_stream(stream)>>>(
      n3, reinterpret_cast<PointNode **>(grid), pre_nodes);
  return launch_status();
}

extern "C" int ha_strings_alloc_c(uint32_t n, const int *lens, char **strs, uint64_t *nfail,
                                  void *stream) {
  if (!lens || !strs || !nfail) return HA_EINVAL;
  if (n == 0) return HA_OK;
  ha_strings_alloc_k<<<blocks_for(n, 128), 128, 0, as_stream(stream)>>>(
      n, lens, strs, reinterpret_cast<unsigned long long *>(nfail));
  return launch_status();
}

extern "C" int ha_strings_concat_c(uint32_t n, char **c, char *const *a, char *const *b,
                                   uint64_t *nfail, void *stream) {
  if (!c || !a || !b || !nfail) return HA_EINVAL;
  if (n == 0) return HA_OK;
  ha_strings_concat_k<<<blocks_for(n, 128), 128, 0, as_stream(stream)>>>(
      n, c, a, b, reinterpret_cast<unsigned long long *>(nfail));
  return launch_status();
}

extern "C" int ha_strings_free_c(uint32_t n, char **strs, void *stream) {
  if (!strs) return HA_EINVAL;
  if (n == 0) return HA_OK;
  ha_strings_free_k<<<blocks_for(n, 128), 128, 0, as_stream(stream)>>>(n, strs);
  return launch_status();
}

extern "C" int ha_strings_check_c(uint32_t n, char *const *c, const int *la, const int *lb,
                                  uint64_t *bad, void *stream) {
  if (!c || !la || !lb || !bad) return HA_EINVAL;
  if (n == 0) return HA_OK;
  ha_strings_check_k<<<blocks_for(n, 128), 128, 0, as_stream(stream)>>>(
      n, c, la, lb, reinterpret_cast<unsigned long long *>(bad));
  return launch_status();
}
