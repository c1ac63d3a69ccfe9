/*
 * ha_model.h -- host replay model of halloc's small-block policy.
 *
 * TEST INFRASTRUCTURE (the oracle).  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg use it; the product path never does.
 *
 * The model replays a serial sequence of hamalloc/hafree calls exactly as the
 * reference allocator (halloc 0.11) would execute them from a single thread,
 * and exposes every piece of allocator state in the reference's own encoding
 * so it can be compared word for word with the reference built for the host
 * (oracle/_ref) and with the device state of the CUDA implementation.
 *
 * Block addresses are reported as byte offsets from the start of slab 0 of a
 * pool whose slabs are laid out contiguously (slab i at i << sb_sz_sh).
 */
#ifndef HA_MODEL_H_
#define HA_MODEL_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ham ham_t;

/* Creates a model; returns NULL when the options are invalid.
   ref_scan_whole_words != 0 reproduces the reference's slab-set scan, which
   only visits nsbs/32 whole bitset words (src/sbset.cuh:17), so trailing
   slabs of a pool with nsbs % 32 != 0 are never handed out; 0 scans
   ceil(nsbs/32) words like the CUDA implementation. */
ham_t *ham_create(uint64_t memory, double halloc_fraction,
                  double busy_fraction, double roomy_fraction,
                  double sparse_fraction, int sb_sz_sh,
                  int ref_scan_whole_words);
void ham_destroy(ham_t *m);

/* >= 0: byte offset of the block; -1: NULL; <= -2: a large block
   (delegated to the CUDA heap; handle -(2 + i)). */
int64_t ham_malloc(ham_t *m, uint64_t nbytes);
/* frees a value returned by ham_malloc (-1 is hafree(NULL), a no-op) */
void ham_free(ham_t *m, int64_t h);
/* op >= 0: malloc(op); op < 0: free(out[-(op + 1)]); out[i] = result */
void ham_run_ops(ham_t *m, const int64_t *ops, int64_t n, int64_t *out);

/* size class of a request (src/halloc.cu:53-67); sizes > 3072 give -1 */
int ham_size_id(uint64_t nbytes);

uint32_t ham_nsbs(const ham_t *m);
uint32_t ham_nsizes(const ham_t *m);
uint32_t ham_bit_words(const ham_t *m);   /* bit-array words per slab */
uint32_t ham_nib_words(const ham_t *m);   /* size-nibble words per slab */
/* nsizes x {nchunks, chunk_sz (encoded), chunk_id, nchunks_in_block,
   sparse, hash_step, roomy, busy}, the order of src/size-info.h:8-26 */
void ham_get_size_infos(const ham_t *m, uint32_t *out);
void ham_get_tickets(const ham_t *m, uint32_t *out);
void ham_get_heads(const ham_t *m, uint32_t *head, uint32_t *cached);
void ham_get_slabs(const ham_t *m, uint32_t *counter, uint32_t *size_id,
                   uint32_t *chunk_id, uint32_t *is_head, uint32_t *chunk_sz);
/* free, sparse[0..3], roomy[0..nsizes-1], busy[0..nsizes-1]; nwords each */
void ham_get_sets(const ham_t *m, uint32_t *out, uint32_t nwords);
void ham_get_bits(const ham_t *m, uint32_t sb, uint32_t *out, uint32_t nwords);
void ham_get_alloc_sizes(const ham_t *m, uint32_t sb, uint32_t *out,
                         uint32_t nwords);

/* ---- CPU baselines (timed on the host cores) -------------------------- */
/* The plain workload through independent model replicas, one per worker
   thread, each on its contiguous slice of logical GPU threads.  Returns
   wall seconds; *checksum sums every word read back. */
double ham_plain_run(uint64_t memory, int sb_sz_sh, uint32_t nthreads,
                     uint32_t niters, uint32_t nbytes, int nworkers,
                     uint64_t *checksum, uint64_t *nfail);
/* The same workload through the C library's malloc/free. */
double hostmalloc_plain_run(uint32_t nthreads, uint32_t niters,
                            uint32_t nbytes, int nworkers, uint64_t *checksum,
                            uint64_t *nfail);

#ifdef __cplusplus
}
#endif
#endif
