#ifndef HALLOC_C_H_
#define HALLOC_C_H_

/*
 * halloc_c.h -- C ABI of halloc-b200 (libhalloc_b200.so).
 *
 * Plain C types only: device buffers are raw device pointers, streams are
 * cudaStream_t passed as void* (NULL = the legacy default stream).  Every
 * int-returning call gives HA_OK (0) or a negative HA_E* code and never
 * exits the process.
 *
 * The allocator itself is used from device code through hamalloc/hafree
 * (include/halloc.h).  This ABI is the host side of it: the init / stats
 * layer, and batch entry points that run the reference's own test and
 * benchmark kernels (malloc a batch, free a batch, the private-throughput
 * loop) so that a host program -- or a Python/ctypes harness -- can drive
 * the allocator without compiling device code.
 */

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- return codes -------------------------------------------------- */
#define HA_OK 0
#define HA_EINVAL (-1)   /* invalid argument or option */
#define HA_ECUDA (-2)    /* a CUDA runtime call failed */
#define HA_ESTATE (-3)   /* not initialised, or already initialised */
#define HA_ERANGE (-4)   /* a size beyond a documented limit */

/* ---- device status bits (ha_status_c) ------------------------------ */
#define HA_ST_TIMEOUT 0x1u  /* a bounded device-side wait gave up */
#define HA_ST_BAD_FREE 0x2u /* hafree of a pointer that is no live block */
#define HA_ST_LIVELOCK 0x4u /* a hamalloc exceeded its probe-round bound */
#define HA_ST_GROW 0x8u     /* no slab was left, but the pool can still grow
                               (ha_grow_c) */

/* Options: same fields, order and layout as struct halloc_opts_t
   (include/halloc.h; halloc src/halloc.h:15-34). */
typedef struct ha_opts_c {
  uint64_t memory;
  double halloc_fraction;
  double busy_fraction;
  double roomy_fraction;
  double sparse_fraction;
  int32_t sb_sz_sh;
} ha_opts_c;

/* ---- init / shutdown / statistics ---------------------------------- */

/* Initialises the allocator on the current device.  HA_ESTATE if it is
   already initialised there (call ha_shutdown_c first).
   Replaces ha_init (halloc src/halloc.cu:267-424). */
int ha_init_c(const ha_opts_c *opts);

/* Frees the allocator's device memory; blocks still held become invalid.
   Replaces ha_shutdown (halloc src/halloc.cu:426-428, a no-op there). */
int ha_shutdown_c(void);

/* External fragmentation (see ha_extfrag in include/halloc.h); negative on
   error.  Replaces ha_extfrag (halloc src/statistics.cuh:50-69). */
double ha_extfrag_c(int ideal);

typedef struct ha_stats_t {
  uint64_t pool_base;       /* device address of slab 0 */
  uint64_t pool_bytes;      /* nsbs * slab size */
  uint64_t cuda_heap_bytes; /* CUDA heap size requested by init */
  uint64_t used_chunks;     /* chunks in live small blocks */
  uint64_t used_bytes;      /* bytes in live small blocks */
  uint32_t nsbs;
  uint32_t sb_sz;
  uint32_t free_slabs;      /* slabs in the free set */
  uint32_t head_slabs;      /* slabs flagged head (heads + prefetched) */
  uint32_t status;          /* HA_ST_* bits */
  uint32_t n_head_changes;  /* head replacements since init */
  uint32_t n_null;          /* small requests answered with NULL */
  uint32_t heap_limit_ok;   /* 1 if the CUDA heap size could be set */
  uint32_t head[16];        /* head slab per size class, 0xffffffff none */
  uint32_t cached[16];      /* prefetched next head per size class */
  uint32_t growth;          /* 1 when the pool grows on demand (ha_set_growth_c) */
  uint32_t committed_slabs; /* slabs backed by device memory (nsbs without growth) */
  uint64_t unit_bytes;      /* growth / release unit, a multiple of the slab size */
  uint32_t surge_level[16]; /* per size class: 2^level head sets open (0 = one) */
  uint32_t n_surge_changes; /* surge level changes since init */
  uint32_t free_count;      /* the free set's own count of its slabs (kept by
                               its operations; equals free_slabs when no
                               kernel runs) */
} ha_stats_t;

/* Fills *out (synchronises the device).  No counterpart in the reference,
   which only had ha_extfrag. */
int ha_stats_c(ha_stats_t *out);

/* Returns the HA_ST_* bits raised since init / the last clear. */
uint32_t ha_status_c(void);
int ha_clear_status_c(void);

/* Bound, in microseconds, of every device-side wait (default 1 s). */
int ha_set_wait_limit_c(uint32_t microseconds);

/* Full allocator state in host buffers, for parity checks against the host
   replay model.  NULL members are skipped.  Sizes: tickets/heads/cached 16,
   size_infos 16*8, per-slab arrays nsbs, sets 37*ceil(nsbs/32) (free,
   sparse[4], roomy[16], busy[16]), bits nsbs*(slab/512),
   nibbles nsbs*(slab/128) (4 bits per 16 B of slab, indexed by offset/16). */
typedef struct ha_state_dump_t {
  uint32_t *tickets, *heads, *cached, *size_infos;
  uint32_t *counters, *size_id, *chunk_id, *is_head, *chunk_enc;
  uint32_t *sets, *bits, *nibbles;
} ha_state_dump_t;
int ha_dump_state_c(const ha_state_dump_t *out);

/* Pins the slab metadata (bit arrays, size nibbles) in L2 for kernels
   launched on `stream` (an access-policy window over the metadata). */
int ha_l2_persist_c(void *stream);

/* ---- slab growth and release ------------------------------------------
   halloc commits every slab at init and never gives one back (its TODO at
   src/slab.cuh:371, the unused SB_CUDA flag at src/slab.h:9-12).  With
   growth on, init reserves the address range of the whole slab pool but
   backs only the first initial_bytes with device memory (cuMemCreate /
   cuMemMap, in units of ha_stats_t.unit_bytes); the other slabs join the
   free set when ha_grow_c backs them, and ha_trim_c gives the memory of
   wholly free units back.  Addresses, the grid map and the policy are those
   of the fully committed pool.  When a head slab is needed and none is
   left while the pool can still grow, hamalloc returns NULL and raises
   HA_ST_GROW.  Grow and trim may run while kernels allocate; call them
   from one host thread per device. */

/* Applied by the next init on this process: 0 (the default) commits the
   whole pool at init; otherwise init backs initial_bytes (at least one
   unit) and the pool grows on demand. */
int ha_set_growth_c(uint64_t initial_bytes);
/* Backs at least `bytes` more of the pool (lowest units first) and adds
   their slabs to the free set on `stream`; *added_bytes (may be NULL) gets
   what was added.  HA_ERANGE when the pool is fully backed, HA_ESTATE
   without growth. */
int ha_grow_c(uint64_t bytes, void *stream, uint64_t *added_bytes);
/* Takes wholly free units (every slab in the free set, no chunk in use) out
   of the free set, up to max_bytes, and returns their device memory to
   CUDA; synchronises `stream`.  *released_bytes (may be NULL) gets what was
   released.  HA_ESTATE without growth. */
int ha_trim_c(uint64_t max_bytes, void *stream, uint64_t *released_bytes);

/* Tuning knob, applied by the next init on this process: the probe hash
   step of each size class is ncib x (largest prime below span) with span =
   (nblocks/256 + nblocks/64) x percent / 100.  100 (the default) is the
   reference's rule (halloc src/halloc.cu:384-385) and the only setting
   whose addresses match it; the autotuner may pick another. 10..1000. */
int ha_set_hash_scale_c(uint32_t percent);

/* Tuning knob, applied by the next init on this process: head slabs per
   size class, a power of two up to 8.  A warp allocates from head
   (SM id mod nheads), each head with its own ticket counter and its own
   head replacement, which spreads the hottest words and the replacement
   work over several slabs.  1 (the default) is the reference policy (its
   compile-time NHEADS, halloc src/slab.h:43) and the only setting whose
   addresses match it.  A program that uses only halloc.h sets the same knob
   with HALLOC_HEADS=<n> in its environment, read at init; a call here wins
   over the environment. */
int ha_set_heads_c(uint32_t nheads);

/* Surge head sets (on by default with one head per size; applied by the
   next init on this process).  When thousands of warps queue for one size's
   head replacement during one head's life (2,048 queued warps: a grid of
   1,024 warps can never get there), or when a long queue forms at a head
   that serves only a few allocations per queued warp (under 96), or when
   a head under half its busy threshold keeps missing first probes (2,048
   allocations needing two or more look-ahead rounds within 16 tickets
   each), the size gets 2, then 4, then 8 head slabs, each serving the SMs
   whose id modulo the set count names it -- while a quarter of the pool's
   slabs is free.
   The sets close again one level per calm head change (or while under an
   eighth of the pool is free), and all of them at once when a size runs
   short of slabs, so a NULL still means that no slab is left for the size.
   A thread alone, or any grid that neither queues that many warps nor
   probes that long, keeps the reference policy's single head and
   addresses.  0 turns them off (the
   reference policy under every load), 1 on, -1 back to the environment's
   choice; HALLOC_SURGE=0|1 in the environment does the same for programs
   that only use halloc.h.  Ignored
   when ha_set_heads_c chose more than one head.  No counterpart in the
   reference (halloc src/slab.cuh:378-445 has one head per size). */
int ha_set_surge_c(int on);

/* Closes every size's surge head sets now, on `stream`: their heads and
   prefetched slabs are filed by occupancy (empty ones to the free set), and
   each size is back to its single head until the next storm.  Open sets
   otherwise close one level per calm head change, or all at once when a
   size runs short of slabs; a program that has gone quiet can call this
   (ha_trim_c does) to see every empty slab in the free set.  Run it while
   no kernel allocates.  No counterpart in the reference. */
int ha_close_surges_c(void *stream);

/* Test hook for failure detection: sets the head-replacement lock of size
   class `size_id` to `held` (1 = held by a holder that never releases it,
   0 = free).  A hamalloc that then needs a new head for that size waits
   until the wait limit, raises HA_ST_TIMEOUT and returns NULL.  No
   counterpart in the reference (its waits are unbounded). */
int ha_debug_set_head_lock_c(uint32_t size_id, uint32_t held);

/* ---- batch entry points (device buffers) --------------------------- */

/* Thread i of nthreads performs nallocs hamalloc calls; request a of thread
   i has size sizes[a*nthreads + i] and its pointer goes to
   ptrs[a*nthreads + i].  tag != 0 writes the request size into the first
   4 bytes of each block.  Replaces malloc_k / malloc_corr_k
   (halloc tst/common/common.h:361-388). */
int ha_malloc_batch_c(const uint32_t *sizes, uint32_t nthreads,
                      uint32_t nallocs, void **ptrs, int tag, void *stream);

/* hafree of ptrs[a*nthreads + i] for every thread i and a < nallocs.
   Replaces free_k (halloc tst/common/common.h:390-399). */
int ha_free_batch_c(void *const *ptrs, uint32_t nthreads, uint32_t nallocs,
                    void *stream);

/* The private-throughput loop: nthreads threads in blocks of `block`, each
   doing niters x (nallocs x hamalloc(sizes[i]); write 16 bytes
   {i^0,i^1,i^2,i^3} to each block; read them back into a checksum;
   nallocs x hafree).  sizes may be NULL for a fixed `nbytes`.
   out[0] += checksum, out[1] += failed allocations (out is not cleared).
   Replaces throughput_malloc_free_k + PrivThroughputTest
   (halloc tst/perf/priv-throughput/priv-throughput.cu:13-63). */
int ha_throughput_c(const uint32_t *sizes, uint32_t nbytes, uint32_t nthreads,
                    uint32_t block, uint32_t nallocs, uint32_t niters,
                    uint64_t *out, void *stream);

/* The same loop end to end from host memory: h_sizes (nthreads words;
   NULL for a fixed nbytes) in, the loop, the two totals out to h_out and to
   d_out, the stream synchronised.  ha_throughput_host_ex_c with
   HA_XFER_AUTO.  No counterpart in halloc, whose tests start from device
   buffers. */
int ha_throughput_host_c(const uint32_t *h_sizes, uint32_t *d_sizes,
                         uint32_t nbytes, uint32_t nthreads, uint32_t block,
                         uint32_t nallocs, uint32_t niters, uint64_t *d_out,
                         uint64_t *h_out, void *stream);

#define HA_XFER_AUTO 0u   /* mapped when the device can address both host
                             buffers (pinned memory), else copy */
#define HA_XFER_COPY 1u   /* copy engine: h_sizes -> d_sizes, d_out cleared,
                             the loop, d_out -> h_out, as one CUDA graph built
                             on the first call and reused while the arguments
                             stay the same */
#define HA_XFER_MAPPED 2u /* one kernel reads h_sizes in place over the bus
                             and its last block stores the totals into h_out;
                             d_sizes is not used.  HA_EINVAL when a buffer
                             is not device-addressable */

/* ha_throughput_host_c with the transfer chosen (HA_XFER_*).  The cached
   graph and the mapped form's device totals are one per process and
   device: calls from several host threads must not overlap.  No counterpart
   in halloc. */
int ha_throughput_host_ex_c(const uint32_t *h_sizes, uint32_t *d_sizes,
                            uint32_t nbytes, uint32_t nthreads, uint32_t block,
                            uint32_t nallocs, uint32_t niters, uint64_t *d_out,
                            uint64_t *h_out, uint32_t transfer, void *stream);

/* The same loop with CUDA's in-kernel malloc/free instead of
   hamalloc/hafree: the comparator of the reference's benchmarks
   (halloc tst/common/cuda-malloc-wrapper.h:8-20). */
int ha_cuda_throughput_c(const uint32_t *sizes, uint32_t nbytes,
                         uint32_t nthreads, uint32_t block, uint32_t nallocs,
                         uint32_t niters, uint64_t *out, void *stream);

/* One round of the mixed-size phase workload (nthreads threads, nslots
   block slots each; slots[s*nthreads + i] is NULL when empty, slot_sz its
   block size).  kind 0 (allocation round): each empty slot is filled with
   probability thr / 2^32 by hamalloc of a size drawn from size_set[nsizes],
   and the block's 32-bit words are written base, base+1, ...; kind 1 (free
   round): each live block is read back and hafree'd with probability
   thr / 2^32 (always for thr = 0xffffffff).  Decisions, sizes and bases
   come from a hash of (seed, thread, slot, round).  acc (6 device words):
   acc[0] is set to the slots filled after the round; acc[1] += failed
   allocations, acc[2] += sum of words written, acc[3] += sum of words read
   back, acc[4] += allocations, acc[5] += frees.  Replaces
   prob_throughput_k / prob_corr_k (halloc
   tst/perf/phase-throughput/phase-throughput.cu:14-47,
   tst/corr/prob-checkptr/prob-checkptr.cu:14-45) with an occupancy-driven
   phase schedule. */
int ha_phase_round_c(int kind, uint32_t nthreads, uint32_t nslots, uint32_t seed,
                     uint32_t round, uint32_t thr, const uint32_t *size_set,
                     uint32_t nsizes, void **slots, uint32_t *slot_sz, uint64_t *acc,
                     void *stream);

typedef struct ha_phase_result_t {
  uint32_t alloc_rounds, free_rounds;
  double kernel_ms;   /* sum of the rounds' kernel times (CUDA events) */
  uint64_t filled;    /* slots filled after the last round */
  uint64_t acc[6];    /* final accumulators, as in ha_phase_round_c */
} ha_phase_result_t;

/* The whole phase workload: `periods` times (allocation rounds until at
   least target_filled slots are filled, at most max_rounds; one free
   round), then a round freeing every remaining block.  Round r uses round
   number r in the hash.  The host loop of the reference's phase-throughput
   test (halloc tst/perf/phase-throughput/phase-throughput.cu:149-192),
   driven by occupancy instead of fixed transition probabilities. */
int ha_phase_run_c(uint32_t nthreads, uint32_t nslots, uint32_t seed,
                   uint32_t periods, uint32_t thr_alloc, uint32_t thr_free,
                   uint64_t target_filled, uint32_t max_rounds,
                   const uint32_t *size_set, uint32_t nsizes, void **slots,
                   uint32_t *slot_sz, uint64_t *acc, ha_phase_result_t *res,
                   void *stream);

/* ---- phase workload, the reference's own form --------------------- */

/* One kernel launch ("try" itry) of the reference's phase-throughput test
   (halloc tst/perf/phase-throughput/phase-throughput.cu:17-48): each of
   nthreads threads runs niters iterations; in iteration it of try itry the
   phase is (itry * niters + it) % 2 (0 = allocation, 1 = free), and a thread
   holding nothing allocates nallocs blocks with probability probs[2*phase],
   a thread holding blocks frees them all with probability probs[2*phase+1].
   Sizes are drawn uniformly from [smin, smax] (no draw when equal).  All
   draws come from the thread's generator state states[i] (Thomas Wang's
   32-bit integer hash chained, tst/common/common.h:80-117), updated in
   place.  Block k of thread i is slots[k * nthreads + i]; ctrs[i] is the
   thread's number of blocks (0 or nallocs).  With rest != 0 the launch
   instead frees every block still held (free_rest_k).  acc (device, 4
   words, accumulated, not reset): mallocs, frees, failed mallocs, bytes
   requested by successful mallocs. */
int ha_phase_ref_step_c(uint32_t nthreads, uint32_t nallocs, uint32_t itry, uint32_t niters,
                        const float *probs, uint32_t smin, uint32_t smax, uint32_t *states,
                        void **slots, uint32_t *ctrs, uint64_t *acc, int rest, void *stream);

typedef struct ha_phase_ref_result_t {
  double kernel_ms;      /* all tries and the final free (CUDA events) */
  double alloc_phase_ms; /* even tries */
  double free_phase_ms;  /* odd tries and the final free */
  uint64_t acc[4];       /* as in ha_phase_ref_step_c, over the whole run */
  double wall_ms;        /* host clock around each launch and its
                            synchronisation, summed (how halloc timed it) */
} ha_phase_ref_result_t;

/* ntries tries then the final free, each launch timed with CUDA events and
   waited for (the host loop of phase-throughput.cu:76-110).  acc is reset
   first. */
int ha_phase_ref_run_c(uint32_t nthreads, uint32_t nallocs, uint32_t ntries, uint32_t niters,
                       const float *probs, uint32_t smin, uint32_t smax, uint32_t *states,
                       void **slots, uint32_t *ctrs, uint64_t *acc,
                       ha_phase_ref_result_t *res, void *stream);

/* Per-call latency, in SM clock cycles (clock64). */
typedef struct ha_latency_stats_t {
  uint64_t n;
  double min_cycles, avg_cycles, max_cycles, p50_cycles, p99_cycles;
} ha_latency_stats_t;

/* The reference's phase-latency test (halloc
   tst/perf/phase-latency/phase-latency.cu:18-56): the tries of
   ha_phase_ref_run_c with clock64() around every hamalloc and hafree
   call, then the final free (untimed).  out[0] = hamalloc, out[1] = hafree;
   percentiles from a 16-per-octave histogram. */
int ha_phase_ref_latency_c(uint32_t nthreads, uint32_t nallocs, uint32_t ntries,
                           uint32_t niters, const float *probs, uint32_t smin, uint32_t smax,
                           uint32_t *states, void **slots, uint32_t *ctrs, uint64_t *acc,
                           ha_latency_stats_t *out, void *stream);

/* ---- the reference's sample programs ------------------------------ */

/* grid-points (halloc samples/grid-points/grid-points.cu:82-153): point ip
   of n (pts: device, 3 floats per point in [0, 1]) gets a 16-byte list node,
   from hamalloc or, when pre_nodes is not NULL, from that device array of n
   nodes, pushed onto the list of its cell of the ncells^3 grid (grid: device,
   ncells^3 pointers, NULL at first).  nfail (device, 1 word, accumulated):
   nodes hamalloc could not give. */
int ha_grid_insert_c(uint32_t n, uint32_t ncells, const float *pts, void **grid,
                     void *pre_nodes, uint64_t *nfail, void *stream);
/* Per cell: the number of points and the sum of mix32(point index) ("lowbias32"
   finaliser), into device arrays of ncells^3 entries. */
int ha_grid_check_c(uint32_t ncells, void *const *grid, uint32_t *count, uint64_t *hsum,
                    void *stream);
/* One thread per cell frees the cell's nodes (unless pre_nodes) and clears
   the cell. */
int ha_grid_free_c(uint32_t ncells, void **grid, int pre_nodes, void *stream);

/* add-strings (halloc samples/add-strings/add-strings.cu:71-205): string i
   becomes lens[i] spaces and a zero byte in a block from hamalloc
   (strs: device, n pointers); concat makes c[i] = a[i] followed by b[i] in a
   new block; free releases and clears every string.  Strings are read and
   written as 64-bit words.  nfail (device, accumulated): NULL blocks. */
int ha_strings_alloc_c(uint32_t n, const int *lens, char **strs, uint64_t *nfail,
                       void *stream);
int ha_strings_concat_c(uint32_t n, char **c, char *const *a, char *const *b,
                        uint64_t *nfail, void *stream);
int ha_strings_free_c(uint32_t n, char **strs, void *stream);
/* bad (device, accumulated): strings c[i] that are not la[i] + lb[i] spaces
   and a zero byte. */
int ha_strings_check_c(uint32_t n, char *const *c, const int *la, const int *lb,
                       uint64_t *bad, void *stream);

/* ---- batched workload -------------------------------------------- */

/* A stream of allocation batches.  Step s (0 <= s <= nbatch) first frees
   the requests listed for it, then (s < nbatch) allocates the requests of
   batch s; step nbatch frees whatever is still live.  Each block carries
   its request id in its first 8 bytes, checked when it is freed. */
typedef struct ha_batch_plan_t {
  uint32_t nbatch;
  uint32_t nreq;
  const uint32_t *req_size;      /* device, nreq: bytes of request r */
  uint64_t *req_ptr;             /* device, nreq: block of request r */
  const uint32_t *free_ids;      /* device, nreq: request ids by free step */
  const uint32_t *h_batch_start; /* host, nbatch+1: batch b = requests
                                    [h_batch_start[b], h_batch_start[b+1]) */
  const uint32_t *h_free_start;  /* host, nbatch+2: step s frees
                                    free_ids[h_free_start[s] .. [s+1]);
                                    both offset arrays never decrease and
                                    end within nreq (else HA_EINVAL) */
  uint64_t *acc; /* device, 8 words: [0] failed allocations, [1] id
                    mismatches, [2] sum of freed request ids, [3]
                    allocations, [4] frees, [5] dependency-wait timeouts */
} ha_batch_plan_t;

/* Plain form: two launches per step (free kernel, malloc kernel) on
   `stream`, `block` threads per block; clears acc first.  No counterpart
   in the reference (its benchmarks launch one kernel per phase). */
int ha_batched_plain_c(const ha_batch_plan_t *plan, uint32_t block, void *stream);

/* Persistent form: ONE kernel whose resident blocks take tasks (chunks of
   task_items requests) from a queue in step order, each step's allocation
   chunks before its free chunks; a free task waits (bounded) until every
   allocation task of the earlier batches has finished.  `block` threads per block ("request group"), ctas_per_sm
   blocks per SM (0 = as many as fit).  use_graph != 0 captures
   [clear acc, reset queue, kernel] in a CUDA graph once, replayed by each
   ha_batched_launch_c.  Returns an opaque handle in *out. */
int ha_batched_prepare_c(const ha_batch_plan_t *plan, uint32_t block,
                         uint32_t ctas_per_sm, uint32_t task_items,
                         int use_graph, void **out);
int ha_batched_launch_c(void *handle, void *stream);
int ha_batched_release_c(void *handle);

/* The persistent form for callers that cannot call cudaMalloc -- code that
   has given all device memory to its own pool, or a latency-bound serving
   loop that must not call cudaMalloc/cudaFree because they synchronise the
   device.  It allocates nothing: the task table and counters live in one
   fixed array of device memory that every GPU loading this library holds
   until exit (about 1.3 MiB).  Limits: at most 65,536 tasks (ceil of each
   step's frees and of each batch's requests over task_items, summed) and
   1,024 batches, else HA_ERANGE; offsets that decrease or run past nreq
   give HA_EINVAL, checked before anything is launched.  The step offsets
   (h_batch_start, h_free_start) travel as a kernel parameter, so the host
   arrays may be reused as soon as the call returns.  The first call on a
   device looks up the array's device address, with that device current;
   make that first call before any stream capture.  Each call rebuilds the
   table and clears the counters, but all calls share the one array: calls
   that overlap on the GPU race, so serialise them (one stream, or events).
   The caller still provides the plan's buffers and acc.  No counterpart in
   the reference. */
int ha_batched_run_noalloc_c(const ha_batch_plan_t *plan, uint32_t block,
                             uint32_t ctas_per_sm, uint32_t task_items,
                             void *stream);

/* ---- random-graph build ------------------------------------------- */

/* Builds a random graph on n vertices, one device thread per vertex.
   Vertex u's out-degree is the number of entries of cdf[0..ncdf) (an
   increasing table of 32-bit thresholds of the degree distribution) that
   are <= mix32(u ^ seed); its k-th neighbour is
   mix32(mix32(u ^ seed ^ 0xABCDEF01) + k * 0x9E3779B9) mod n, with mix32
   the "lowbias32" finaliser.  The neighbours go into an int32 array from
   hamalloc that starts at capacity 2 and doubles (malloc new, copy, hafree
   old); arr[u] receives the array and deg[u] its length.  acc (3 device
   words, cleared): failed allocations, doublings, edges.  Replaces
   random_graph_build_k (halloc samples/random-graph/random-graph.cu:
   165-181), which built linked lists. */
int ha_graph_build_c(uint32_t n, uint32_t seed, const uint32_t *cdf,
                     uint32_t ncdf, uint64_t *arr, uint32_t *deg,
                     uint64_t *acc, void *stream);

/* Copies every vertex's array to cols[offsets[u] ...] (a CSR, offsets =
   exclusive prefix sum of deg) and hafree's it. */
int ha_graph_gather_c(uint32_t n, uint64_t *arr, const uint32_t *deg,
                      const uint64_t *offsets, uint32_t *cols, void *stream);

/* ---- serving loop ------------------------------------------------ */

/* A host-fed stream of jobs served by continuous batching.  Job j (an id;
   every parameter derives from a hash of (seed, j)) has a target of
   ceil(L/block_bytes) blocks, L log-uniform in [min_len, max_len]; on each
   step it gains grow_min..grow_max blocks (hamalloc(block_bytes) each,
   linked through their first 8 bytes, the next 4 bytes holding a hashed
   value) until the target, and it ends after an Exp(mean_life) number of
   steps: its blocks are read back (result = number of blocks and sum of the
   values) and hafree'd.  Arrivals are Poisson with rate `lambda` jobs/s:
   a host thread releases job ids at their arrival times through a mapped
   host counter.  One persistent kernel serves them: each thread owns a
   job slot; each warp claims released jobs for its empty slots while the
   slab pool's occupancy is at most occupancy_limit (otherwise the
   admission is refused and retried), steps its jobs independently of other
   warps (a finished job frees at most 64 blocks per step), and leaves once
   the stream has ended and its slots are empty.
   Every hamalloc's latency (clock64 cycles) goes into a log-linear
   histogram.  With job_ids != NULL only those jobs (in that order) are
   released, e.g. to serve one job alone.  No counterpart in the
   reference. */
typedef struct ha_serve_cfg_t {
  uint32_t njobs;          /* jobs in the stream (ids 0..njobs-1) */
  uint32_t seed;
  double lambda;           /* arrival rate, jobs per second */
  double occupancy_limit;  /* admission gate on slab-pool occupancy */
  double mean_life;        /* mean job lifetime in steps */
  uint32_t block_bytes;    /* bytes per block (256) */
  uint32_t min_len, max_len;
  uint32_t grow_min, grow_max;
  uint32_t cta_threads;    /* slots per persistent block */
  uint32_t ctas_per_sm;    /* 0 = as many as fit */
  const uint32_t *job_ids; /* host, optional: the ids to release, in order */
  uint32_t njob_ids;
  uint64_t *results;       /* device, 2 words per job id: blocks, value sum */
  uint64_t grow_bytes;     /* with a growing pool (ha_set_growth_c): bytes
                              backed per request of the kernel; a job whose
                              block cannot be had waits for the pool to grow.
                              0 = never grow during the run */
  uint32_t prereleased;    /* 1: every job is released (and the stream ended)
                              before the launch -- a closed batch, and a kernel
                              that waits on nothing from the host */
} ha_serve_cfg_t;

#define HA_SERVE_HIST 1024 /* histogram buckets: 16 per power of two */

typedef struct ha_serve_result_t {
  double seconds;          /* first release to kernel completion, wall */
  double cycles_per_ns;    /* SM clock seen by the kernel */
  uint64_t jobs_done, allocs, alloc_failures, refusals, peak_live_blocks;
  uint64_t timeouts;       /* idle waits that gave up */
  double p50_cycles, p99_cycles, max_cycles;
  uint64_t hist[HA_SERVE_HIST];
  uint64_t alloc_waits;    /* attempts that waited for the pool to grow */
  uint64_t grows, grown_bytes;  /* ha_grow_c calls made for the kernel */
  double grow_seconds;     /* host time in those calls, new slabs adopted */
} ha_serve_result_t;

int ha_serve_run_c(const ha_serve_cfg_t *cfg, ha_serve_result_t *out,
                   void *stream);

/* Latency breakdown of one warp (instrumented builds only): runs the
   private-throughput loop (hamalloc(nbytes), 16-byte write and read-back,
   hafree; niters iterations) with 32 threads, and copies to d_out (device,
   10,272 words) the SM clock each lane read after every dependent round
   trip of hamalloc / hafree: word l = lane l's stamp count, then 2 words
   per stamp (point id, clock low word) at 32 + 2 * (l * 160 + i).  Point
   ids: 1 hamalloc entered, 2 ticket and head back, 3 bit reservation back,
   4 slab count back, 5 hamalloc returns, 6/7 slow path in/out, 8 hafree
   entered, 9 size nibble and descriptor back, 10 count-down back, 11 hafree
   returns, 12 payload read back.  HA_ESTATE in a normal build: only the
   library built with -DHA_STAMPS (halloc_b200/build.py, stamps=True)
   records them.  No counterpart in the reference. */
int ha_stamps_run_c(uint32_t nbytes, uint32_t niters, uint32_t *d_out, void *stream);

/* Replays a trace on ONE device thread: op >= 0 is hamalloc(op);
   op < 0 is hafree of the block returned by op index -(op + 1).
   out[i] = the pointer hamalloc returned (0 for NULL) as an integer, and 0
   for a free.  No counterpart in the reference: it exists so that a serial
   address sequence can be compared with the host replay model. */
int ha_trace_c(const int64_t *ops, int64_t n, int64_t *out, void *stream);

/* L2 atomic throughput probe: every thread of `nthreads` applies `reps`
   32-bit atomic ORs to its own word of buf[nwords] (returning != 0 uses
   the returned value, like a bit-array reservation).  For the roofline
   denominator; no counterpart in the reference. */
int ha_atomic_peak_c(uint32_t *buf, uint32_t nwords, uint32_t nthreads,
                     uint32_t reps, int returning, void *stream);
/* The same with thread t on word (t mod nwords) x stride of buf (nwords x
   stride words): stride 8 puts every thread on a 32-byte sector of its
   own, as the allocator's hashed bit-array probes land. */
int ha_atomic_peak_strided_c(uint32_t *buf, uint32_t nwords, uint32_t stride,
                             uint32_t nthreads, uint32_t reps, int returning, void *stream);

#ifdef __cplusplus
}
#endif
#endif
