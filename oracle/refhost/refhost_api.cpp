/*
 * refhost_api.cpp -- the reference allocator itself (halloc 0.11,
 * src/halloc.cu with every header it includes), compiled unchanged as host
 * C++ and wrapped in a C API for replay and state inspection.
 * TEST INFRASTRUCTURE ONLY (oracle): never linked into the product.
 *
 * Build: oracle/Makefile, target ref.  The reference tree is put on the
 * include path behind -I-, so "halloc.cu" below and every header it includes
 * come from the reference, except utils.h and statistics.cuh, which the
 * oracle/refhost directory replaces (inline PTX and kernel launches cannot
 * compile for the host; see those files).  cuda_host_shim.h is
 * force-included first.
 *
 * Every caller thread acts as one GPU thread alone in its warp.
 *
 * Deviations from running on a GPU, all outside the small-block path:
 *  - blocks > 3072 B come from the host's malloc (src/halloc.cu:185-187) and
 *    ref_free() returns them with free() directly instead of going through
 *    hafree(): the reference's grid lookup (src/grid.cuh:65-71) has no range
 *    check and would read outside sb_grid_g for such pointers;
 *  - the simulated device memory is chosen so that the 3/4 cap of
 *    src/halloc.cu:282 does not bind and the grid offset of
 *    src/halloc.cu:336-340 stays inside the 16384-cell grid.
 */
#include "halloc.cu"

#include <pthread.h>
#include <time.h>

ha_shim_device_t ha_shim_dev;

namespace {
char *g_arena = nullptr;
uint g_sb_sz = 0, g_nsbs = 0;
const int kMaxLarge = 1 << 16;
void *g_large[kMaxLarge];
int g_nlarge = 0;

void release_all() {
  for (int i = 0; i < ha_shim_dev.nother; i++) free(ha_shim_dev.other[i]);
  ha_shim_dev.nother = 0;
  free(g_arena);
  g_arena = nullptr;
  for (int i = 0; i < g_nlarge; i++) free(g_large[i]);
  g_nlarge = 0;
}

double now_s() {
  timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return ts.tv_sec + 1e-9 * ts.tv_nsec;
}
}  // namespace

extern "C" {

/* Initialises the reference allocator; returns the number of slabs, or -1
   when the configuration cannot be represented by the reference's grid. */
int ref_init(unsigned long long memory, double halloc_fraction,
             double busy_fraction, double roomy_fraction,
             double sparse_fraction, int sb_sz_sh) {
  release_all();
  uint sb_sz = 1u << sb_sz_sh;
  unsigned long long total = memory / 3 * 4 + 4ull * sb_sz;
  total = (total + sb_sz - 1) / sb_sz * sb_sz;
  unsigned long long hmem = (unsigned long long)(halloc_fraction * memory);
  uint nsbs = (uint)(hmem / sb_sz);
  if (nsbs == 0 || nsbs > MAX_NSBS) return -1;
  if (total / sb_sz + nsbs + 1 > 2ull * MAX_NSBS) return -1;
  g_arena = (char *)aligned_alloc(sb_sz, (size_t)nsbs * sb_sz);
  if (!g_arena) return -1;
  memset(&ha_shim_dev, 0, sizeof(ha_shim_dev));
  ha_shim_dev.total_mem = total;
  ha_shim_dev.arena = g_arena;
  ha_shim_dev.arena_chunk = sb_sz;
  ha_shim_dev.arena_nchunks = nsbs;
  g_sb_sz = sb_sz;
  g_nsbs = nsbs;
  halloc_opts_t opts(memory);
  opts.halloc_fraction = halloc_fraction;
  opts.busy_fraction = busy_fraction;
  opts.roomy_fraction = roomy_fraction;
  opts.sparse_fraction = sparse_fraction;
  opts.sb_sz_sh = sb_sz_sh;
  ha_init(opts);
  return (int)nsbs;
}

void ref_shutdown(void) {
  ha_shutdown();
  release_all();
}

/* >= 0: byte offset of the block from the start of slab 0;
   -1: NULL; <= -2: handle -(2 + i) of a large (CUDA-heap) block. */
long long ref_malloc(unsigned long long nbytes) {
  void *p = hamalloc((size_t)nbytes);
  if (!p) return -1;
  char *c = (char *)p;
  if (c >= g_arena && c < g_arena + (size_t)g_nsbs * g_sb_sz)
    return (long long)(c - g_arena);
  if (g_nlarge >= kMaxLarge) {
    free(p);
    return -1;
  }
  g_large[g_nlarge] = p;
  return -2 - (long long)g_nlarge++;
}

void ref_free(long long h) {
  if (h >= 0) {
    hafree(g_arena + h);
  } else if (h == -1) {
    hafree(nullptr);
  } else {
    long long i = -2 - h;
    if (i < g_nlarge && g_large[i]) {
      free(g_large[i]);
      g_large[i] = nullptr;
    }
  }
}

/* Replays a trace.  op >= 0: hamalloc(op bytes); op < 0: hafree() of the
   block returned by op index -(op + 1).  out[i] is the result of op i
   (ref_malloc encoding) for a malloc, and 0 for a free. */
void ref_run_ops(const long long *ops, long long n, long long *out) {
  for (long long i = 0; i < n; i++) {
    if (ops[i] >= 0) {
      out[i] = ref_malloc((unsigned long long)ops[i]);
    } else {
      ref_free(out[-(ops[i] + 1)]);
      out[i] = 0;
    }
  }
}

/* ---- state inspection -------------------------------------------------- */
unsigned ref_nsbs(void) { return nsbs_g; }
unsigned ref_nsizes(void) { return nsizes_g; }

void ref_get_size_infos(unsigned *out /* nsizes x 8 */) {
  for (uint i = 0; i < nsizes_g; i++) {
    const size_info_t &s = size_infos_g[i];
    unsigned *o = out + 8 * i;
    o[0] = s.nchunks;
    o[1] = s.chunk_sz;
    o[2] = s.chunk_id;
    o[3] = s.nchunks_in_block;
    o[4] = s.sparse_threshold;
    o[5] = s.hash_step;
    o[6] = s.roomy_threshold;
    o[7] = s.busy_threshold;
  }
}

void ref_get_tickets(unsigned *out /* nsizes */) {
  for (uint i = 0; i < nsizes_g; i++) out[i] = counters_g[i];
}

void ref_get_heads(unsigned *head, unsigned *cached /* nsizes each */) {
  for (uint i = 0; i < nsizes_g; i++) {
    head[i] = head_sbs_g[0][i];
    cached[i] = cached_sbs_g[0][i];
  }
}

void ref_get_slabs(unsigned *counter, unsigned *size_id, unsigned *chunk_id,
                   unsigned *is_head, unsigned *chunk_sz /* nsbs each */) {
  for (uint i = 0; i < nsbs_g; i++) {
    counter[i] = sb_counters_g[i];
    size_id[i] = sbs_g[i].size_id;
    chunk_id[i] = sbs_g[i].chunk_id;
    is_head[i] = sbs_g[i].is_head;
    chunk_sz[i] = sbs_g[i].chunk_sz;
  }
}

/* Set words 0..nwords-1: free set, then sparse[0..3], roomy[0..nsizes-1],
   busy[0..nsizes-1], each nwords long. */
void ref_get_sets(unsigned *out, unsigned nwords) {
  unsigned *o = out;
  for (uint w = 0; w < nwords; w++) *o++ = free_sbs_g[w];
  for (uint c = 0; c < 4; c++)
    for (uint w = 0; w < nwords; w++) *o++ = sparse_sbs_g[c][w];
  for (uint s = 0; s < nsizes_g; s++)
    for (uint w = 0; w < nwords; w++) *o++ = roomy_sbs_g[s][w];
  for (uint s = 0; s < nsizes_g; s++)
    for (uint w = 0; w < nwords; w++) *o++ = busy_sbs_g[s][w];
}

void ref_get_bits(unsigned sb, unsigned *out, unsigned nwords) {
  const uint *b = sb_block_bits(sb);
  for (uint w = 0; w < nwords; w++) out[w] = b[w];
}

void ref_get_alloc_sizes(unsigned sb, unsigned *out, unsigned nwords) {
  const uint *a = sb_alloc_sizes(sb);
  for (uint w = 0; w < nwords; w++) out[w] = a[w];
}

/* ---- multi-core run of the plain throughput workload ------------------ */
struct plain_arg_t {
  unsigned t0, t1, niters, nbytes;
  unsigned long long checksum, nfail;
};

static void *plain_worker(void *vp) {
  plain_arg_t *a = (plain_arg_t *)vp;
  unsigned long long sum = 0, nfail = 0;
  for (unsigned t = a->t0; t < a->t1; t++) {
    for (unsigned it = 0; it < a->niters; it++) {
      unsigned *p = (unsigned *)hamalloc(a->nbytes);
      if (!p) {
        nfail++;
        continue;
      }
      for (unsigned k = 0; k < 4; k++) p[k] = t ^ k;
      for (unsigned k = 0; k < 4; k++) sum += ((volatile unsigned *)p)[k];
      hafree(p);
    }
  }
  a->checksum = sum;
  a->nfail = nfail;
  return nullptr;
}

/* Runs nthreads logical GPU threads x niters malloc/write/read/free
   iterations of nbytes (>= 16) on nworkers host threads, each worker taking
   a contiguous slice of logical threads.  Returns wall seconds. */
double ref_plain_run(unsigned nthreads, unsigned niters, unsigned nbytes,
                     int nworkers, unsigned long long *checksum,
                     unsigned long long *nfail) {
  if (nworkers < 1) nworkers = 1;
  if (nworkers > 512) nworkers = 512;
  pthread_t th[512];
  plain_arg_t args[512];
  for (int w = 0; w < nworkers; w++) {
    args[w].t0 = (unsigned)((unsigned long long)nthreads * w / nworkers);
    args[w].t1 = (unsigned)((unsigned long long)nthreads * (w + 1) / nworkers);
    args[w].niters = niters;
    args[w].nbytes = nbytes;
  }
  double t0 = now_s();
  for (int w = 0; w < nworkers; w++)
    pthread_create(&th[w], nullptr, plain_worker, &args[w]);
  for (int w = 0; w < nworkers; w++) pthread_join(th[w], nullptr);
  double dt = now_s() - t0;
  unsigned long long s = 0, f = 0;
  for (int w = 0; w < nworkers; w++) {
    s += args[w].checksum;
    f += args[w].nfail;
  }
  *checksum = s;
  *nfail = f;
  return dt;
}

}  // extern "C"
