/*
 * ha_model.c -- host replay model of halloc 0.11's small-block policy.
 *
 * TEST INFRASTRUCTURE (the oracle).  Used by tests/, by
 * __graft_entry__.smoke() as the checker and by bench.py's CPU-baseline leg;
 * never by the product path.
 *
 * A restatement in plain C of the reference's serial behaviour: one thread
 * calling hamalloc/hafree.  Each function names the reference lines it
 * follows.  State is kept in the reference's own encoding (packed slab
 * counter words, bitset sets, 4-bit size nibbles) so that it can be compared
 * word for word with the reference built for the host and with the CUDA
 * implementation's device state.
 *
 * Pinned by tests/test_oracle.py and tests/test_oracle_property.py against
 * the reference's own sources compiled for the host (oracle/_ref), and by
 * the golden traces in tests/golden/ generated from that build.
 */
#define _GNU_SOURCE
#include "ha_model.h"

#include <math.h>
#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

/* policy constants (src/halloc.cu:38-45, src/slab.h:31-48,
   src/size-info.h:28-47) */
enum {
  NSIZES = 16,             /* 2 sizes per unit x 8 units */
  NCHUNK_IDS = 4,          /* 16, 24, 256, 384 B */
  FIRST_TICKET = 0x0B0B0B0B, /* counters memset to byte 11 */
  HASH_FREQ = 11,          /* THREAD_FREQ */
  GROUP_SHIFT = 2,         /* THREAD_MOD_SH */
  TRIES_PER_ROUND = 32,    /* MAX_NTRIES */
  COUNT_CHECK_PERIOD = 2,  /* CHECK_NTRIES */
  STEP_SCALE = 64,         /* STEP_FREQ */
  MIN_BLOCK = 16,
  MAX_BLOCK = 3072
};
#define NO_SLAB 0xffffffffu
#define NO_SIZE 0xffffffffu

/* packed slab counter (src/slab.h:50-63, 120-125):
   bits 12-31 used chunks, bit 8 head flag, bits 5-7 chunk id (7 = none),
   bits 0-4 size id (left at 31 by ha_init and never changed) */
#define CNT_SHIFT 12
#define HEAD_FLAG (1u << 8)
#define CHUNK_SHIFT 5
#define CHUNK_FIELD 7u

/* set numbering inside ham.sets */
#define SET_FREE 0
#define SET_SPARSE(c) (1 + (c))
#define SET_ROOMY(s) (1 + NCHUNK_IDS + (s))
#define SET_BUSY(s) (1 + NCHUNK_IDS + NSIZES + (s))
#define NSETS (1 + NCHUNK_IDS + 2 * NSIZES)

typedef struct {
  uint32_t nchunks;     /* chunks per slab usable by this size */
  uint32_t chunk_bytes; /* 16, 24, 256 or 384 */
  uint32_t chunk_id;
  uint32_t ncib;        /* chunks in one block */
  uint32_t sparse, hash_step, roomy, busy;
  uint32_t tmod;        /* how many consecutive tickets share a hash slot */
} size_class_t;

struct ham {
  uint32_t nsbs, sb_sh, sb_bytes;
  uint32_t set_words, scan_words;
  uint32_t bit_words, nib_words;
  size_class_t cls[NSIZES];
  uint32_t ticket[NSIZES], head[NSIZES], cached[NSIZES];
  uint32_t *ctr;                         /* packed counters */
  uint32_t *d_size, *d_chunk, *d_head;   /* slab descriptors */
  uint32_t *d_chunk_enc;                 /* encoded chunk size, 0 = free */
  uint32_t *sets;                        /* NSETS x set_words */
  uint32_t *bits;                        /* nsbs x bit_words */
  uint32_t *nib;                         /* nsbs x nib_words */
  int64_t nlarge;
};

/* ---- small helpers -------------------------------------------------- */

/* chunk size encoding of src/size-info.h:50-58: (3 or 1) << 16 | shift */
static uint32_t chunk_enc(uint32_t bytes) {
  uint32_t three = bytes % 3 == 0;
  uint32_t base = three ? bytes / 3 : bytes, sh = 0;
  while ((1u << sh) < base) sh++;
  return (three ? 3u : 1u) << 16 | sh;
}

/* v / chunk size for an encoded chunk size (src/size-info.h:65-70) */
static uint32_t chunk_index(uint32_t v, uint32_t enc) {
  if ((enc >> 16) == 3u) v /= 3u;
  return v >> (enc & 0xffffu);
}

/* largest prime p in [3, n) that divides neither n nor nb
   (src/utils.cu:8-24); 0 if none */
static uint32_t prime_below(uint32_t n, uint32_t nb) {
  for (uint32_t p = n - 1; p >= 3 && p < n; p--) {
    int prime = 1;
    for (uint32_t d = 2; (uint64_t)d * d <= p; d++)
      if (p % d == 0) {
        prime = 0;
        break;
      }
    if (prime && n % p && nb % p) return p;
  }
  return 0;
}

static uint32_t *set_of(ham_t *m, int k) { return m->sets + (size_t)k * m->set_words; }
static void set_put(ham_t *m, int k, uint32_t sb) { set_of(m, k)[sb / 32] |= 1u << (sb % 32); }
static void set_drop(ham_t *m, int k, uint32_t sb) { set_of(m, k)[sb / 32] &= ~(1u << (sb % 32)); }

/* removes and returns the lowest slab of a set (src/sbset.cuh:5-35) */
static uint32_t set_take(ham_t *m, int k) {
  uint32_t *s = set_of(m, k);
  for (uint32_t w = 0; w < m->scan_words; w++)
    if (s[w]) {
      uint32_t b = (uint32_t)__builtin_ctz(s[w]);
      s[w] &= ~(1u << b);
      return w * 32 + b;
    }
  return NO_SLAB;
}

static uint32_t used(const ham_t *m, uint32_t sb) { return m->ctr[sb] >> CNT_SHIFT; }

/* ---- construction (src/halloc.cu:267-424) --------------------------- */

static uint32_t tickets_per_slot(uint32_t sid) {
  /* src/halloc.cu:101-104 */
  int sh = GROUP_SHIFT - (int)sid / 2;
  return 1u << (sh > 0 ? sh : 0);
}

static int build_classes(ham_t *m, double busy, double roomy, double sparse) {
  for (uint32_t sid = 0; sid < NSIZES; sid++) {
    size_class_t *c = &m->cls[sid];
    uint32_t unit = 8u << (sid / 2);
    uint32_t block = (sid & 1 ? 3 : 2) * unit;
    c->tmod = tickets_per_slot(sid);
    uint32_t nblocks = m->sb_bytes / block / c->tmod * c->tmod;
    c->chunk_id = (sid & 1) + (sid < NSIZES / 2 ? 0 : 2);
    c->chunk_bytes = (c->chunk_id & 1 ? 3 : 2) * (c->chunk_id >= 2 ? 128 : 8);
    c->ncib = block / c->chunk_bytes;
    c->nchunks = nblocks * c->ncib;
    uint32_t p = prime_below(nblocks / 256 + nblocks / 64, nblocks);
    if (!p) return -1;
    c->hash_step = c->ncib * p;
    /* thresholds: double x uint truncated to uint (src/halloc.cu:390-392) */
    c->roomy = (uint32_t)(roomy * c->nchunks);
    c->busy = (uint32_t)(busy * c->nchunks);
    c->sparse = (uint32_t)(sparse * c->nchunks);
  }
  return 0;
}

ham_t *ham_create(uint64_t memory, double halloc_fraction, double busy_fraction,
                  double roomy_fraction, double sparse_fraction, int sb_sz_sh,
                  int ref_scan_whole_words) {
  if (sb_sz_sh < 20 || sb_sz_sh > 24) return NULL;
  ham_t *m = (ham_t *)calloc(1, sizeof(ham_t));
  if (!m) return NULL;
  m->sb_sh = (uint32_t)sb_sz_sh;
  m->sb_bytes = 1u << sb_sz_sh;
  uint64_t pool = (uint64_t)(halloc_fraction * (double)memory);
  uint64_t nsbs = pool / m->sb_bytes;
  if (nsbs == 0 || nsbs > (1u << 20) || build_classes(m, busy_fraction,
      roomy_fraction, sparse_fraction)) {
    free(m);
    return NULL;
  }
  m->nsbs = (uint32_t)nsbs;
  m->set_words = (m->nsbs + 31) / 32;
  m->scan_words = ref_scan_whole_words ? m->nsbs / 32 : m->set_words;
  m->bit_words = m->sb_bytes / (MIN_BLOCK * 32);
  m->nib_words = m->sb_bytes / (MIN_BLOCK * 8);
  size_t n = m->nsbs;
  m->ctr = (uint32_t *)malloc(n * 4);
  m->d_size = (uint32_t *)malloc(n * 4);
  m->d_chunk = (uint32_t *)malloc(n * 4);
  m->d_head = (uint32_t *)calloc(n, 4);
  m->d_chunk_enc = (uint32_t *)calloc(n, 4);
  m->sets = (uint32_t *)calloc((size_t)NSETS * m->set_words, 4);
  m->bits = (uint32_t *)calloc(n * m->bit_words, 4);
  m->nib = (uint32_t *)calloc(n * m->nib_words, 4);
  if (!m->ctr || !m->d_size || !m->d_chunk || !m->d_head || !m->d_chunk_enc ||
      !m->sets || !m->bits || !m->nib) {
    ham_destroy(m);
    return NULL;
  }
  for (uint32_t sb = 0; sb < m->nsbs; sb++) {
    /* count 0, not head, no chunk, size field all ones (src/halloc.cu:310) */
    m->ctr[sb] = CHUNK_FIELD << CHUNK_SHIFT | 31u;
    m->d_size[sb] = NO_SIZE;
    m->d_chunk[sb] = NO_SIZE;
    set_put(m, SET_FREE, sb);
  }
  for (int s = 0; s < NSIZES; s++) {
    m->ticket[s] = FIRST_TICKET;
    m->head[s] = NO_SLAB;
    m->cached[s] = NO_SLAB;
  }
  return m;
}

void ham_destroy(ham_t *m) {
  if (!m) return;
  free(m->ctr);
  free(m->d_size);
  free(m->d_chunk);
  free(m->d_head);
  free(m->d_chunk_enc);
  free(m->sets);
  free(m->bits);
  free(m->nib);
  free(m);
}

/* ---- slab state transitions ----------------------------------------- */

/* Return a slab with no used chunks to the free set, or (when called while
   detaching a head) to the sparse set if chunks are still in use.
   src/slab.cuh:89-113 */
static void try_release(ham_t *m, uint32_t sb, uint32_t cid, int from_head) {
  if (m->d_head[sb] || cid == NO_SIZE) return;
  uint32_t clear = ((NO_SIZE - cid) & CHUNK_FIELD) << CHUNK_SHIFT;
  for (;;) {
    uint32_t before = m->ctr[sb];
    m->ctr[sb] += clear; /* chunk field := none */
    if ((before >> CNT_SHIFT) == 0) {
      m->d_size[sb] = NO_SIZE;
      m->d_chunk[sb] = NO_SIZE;
      m->d_chunk_enc[sb] = 0;
      set_put(m, SET_FREE, sb);
      if (!from_head) set_drop(m, SET_SPARSE(cid), sb);
      return;
    }
    uint32_t again = m->ctr[sb];
    m->ctr[sb] -= clear; /* chunk field restored */
    if ((again >> CNT_SHIFT) != 0) break;
  }
  if (from_head) set_put(m, SET_SPARSE(cid), sb);
}

/* Adds a block's chunks to a slab's count (single-lane form of
   src/slab.cuh:122-155).  Bit 0: the slab still has the caller's chunk size;
   bit 1: this add crossed the busy threshold. */
static uint32_t count_up(ham_t *m, uint32_t sb, uint32_t sid) {
  const size_class_t *c = &m->cls[sid];
  uint32_t before = m->ctr[sb];
  m->ctr[sb] += c->ncib << CNT_SHIFT;
  uint32_t flags = ((before >> CHUNK_SHIFT) & CHUNK_FIELD) == c->chunk_id;
  uint32_t n0 = before >> CNT_SHIFT;
  if (n0 + c->ncib >= c->busy && n0 < c->busy) flags |= 2;
  return flags;
}

/* Removes chunks from a slab's count and moves a non-head slab between the
   busy / roomy / sparse / free sets when a threshold is crossed on the way
   down (single-lane form of src/slab.cuh:161-224). */
static void count_down(ham_t *m, uint32_t sb, uint32_t nchunks) {
  uint32_t before = m->ctr[sb];
  m->ctr[sb] -= nchunks << CNT_SHIFT;
  if (before & HEAD_FLAG) return;
  uint32_t sid = m->d_size[sb], cid = m->d_chunk[sb];
  if (sid == NO_SIZE || cid == NO_SIZE) return;
  const size_class_t *c = &m->cls[sid];
  uint32_t n0 = before >> CNT_SHIFT, n1 = n0 - nchunks;
  if (n1 <= c->busy && n0 > c->busy) {
    set_put(m, SET_BUSY(sid), sb);
  } else if (n1 <= c->roomy && n0 > c->roomy) {
    set_put(m, SET_ROOMY(sid), sb);
    set_drop(m, SET_BUSY(sid), sb);
  } else if (n1 <= c->sparse && n0 > c->sparse) {
    set_put(m, SET_SPARSE(cid), sb);
    set_drop(m, SET_ROOMY(sid), sb);
  } else if (n1 == 0 && ((before >> CHUNK_SHIFT) & CHUNK_FIELD) != CHUNK_FIELD) {
    /* under the slab lock the descriptor is read again; serially it is
       unchanged */
    try_release(m, sb, m->d_chunk[sb], 0);
  }
}

/* Stops using a slab as head and files it by occupancy
   (src/slab.cuh:227-255).  The reference compares against the ROOMY
   threshold of the slab's size first, then against the sparse and roomy
   thresholds of the size-table entry whose index equals the CHUNK id
   (src/slab.cuh:378, 386-387); the model keeps both quirks. */
static void detach(ham_t *m, uint32_t sb) {
  m->d_head[sb] = 0;
  uint32_t before = m->ctr[sb];
  m->ctr[sb] -= HEAD_FLAG;
  uint32_t n = before >> CNT_SHIFT;
  uint32_t sid = m->d_size[sb];
  if (n > m->cls[sid].roomy) return;
  uint32_t cid = m->d_chunk[sb];
  if (n == 0) {
    try_release(m, sb, cid, 1);
    return;
  }
  const size_class_t *q = &m->cls[cid];
  if (n <= q->sparse)
    set_put(m, SET_SPARSE(cid), sb);
  else if (n <= q->roomy)
    set_put(m, SET_ROOMY(sid), sb);
  else
    set_put(m, SET_BUSY(sid), sb);
}

static void make_head(ham_t *m, uint32_t sb) {
  m->d_head[sb] = 1;
  m->ctr[sb] += HEAD_FLAG;
}

/* Picks a slab to become head for a size: roomy slabs of the size, then
   sparse slabs of its chunk size, then free slabs, then busy slabs of the
   size that are at most half way from busy to full (src/slab.cuh:259-372). */
static uint32_t find_slab(ham_t *m, uint32_t sid) {
  const size_class_t *c = &m->cls[sid];
  uint32_t cid = c->chunk_id, sb;
  while ((sb = set_take(m, SET_ROOMY(sid))) != NO_SLAB) {
    if (m->d_head[sb] || m->d_size[sb] != sid) continue;
    if (used(m, sb) <= c->roomy) {
      make_head(m, sb);
      return sb;
    }
    set_put(m, SET_BUSY(sid), sb);
  }
  while ((sb = set_take(m, SET_SPARSE(cid))) != NO_SLAB) {
    if (m->d_head[sb] || m->d_chunk[sb] != cid) continue;
    if (used(m, sb) <= c->sparse) {
      make_head(m, sb);
      m->d_size[sb] = sid;
      return sb;
    }
    if (m->d_size[sb] != NO_SIZE) set_put(m, SET_ROOMY(m->d_size[sb]), sb);
  }
  while ((sb = set_take(m, SET_FREE)) != NO_SLAB) {
    if (m->d_head[sb]) continue;
    m->d_size[sb] = sid;
    m->d_chunk[sb] = cid;
    m->d_chunk_enc[sb] = chunk_enc(c->chunk_bytes);
    make_head(m, sb);
    m->ctr[sb] -= ((NO_SIZE - cid) & CHUNK_FIELD) << CHUNK_SHIFT;
    return sb;
  }
  while ((sb = set_take(m, SET_BUSY(sid))) != NO_SLAB) {
    if (used(m, sb) > (c->busy + c->nchunks) / 2) continue;
    if (m->d_head[sb] || m->d_size[sb] != sid) continue;
    make_head(m, sb);
    return sb;
  }
  return NO_SLAB;
}

/* Replaces the head slab of a size when it has reached the busy threshold,
   using the prefetched ("cached") slab first and prefetching the next one
   (single-thread form of src/slab.cuh:378-445). */
static uint32_t replace_head(ham_t *m, uint32_t sid) {
  uint32_t cur = m->head[sid];
  if (cur != NO_SLAB && used(m, cur) < m->cls[sid].busy) return cur;
  uint32_t next = m->cached[sid];
  m->cached[sid] = NO_SLAB;
  if (next == NO_SLAB) next = find_slab(m, sid);
  if (next == NO_SLAB) return NO_SLAB;
  m->head[sid] = next;
  if (cur != NO_SLAB) detach(m, cur);
  m->cached[sid] = find_slab(m, sid);
  return next;
}

/* ---- allocation ----------------------------------------------------- */

int ham_size_id(uint64_t nbytes) {
  /* src/halloc.cu:53-67: blocks are 2 or 3 units of 8 << k bytes */
  if (nbytes > MAX_BLOCK) return -1;
  uint32_t n = nbytes < MIN_BLOCK ? MIN_BLOCK : (uint32_t)nbytes;
  uint32_t k = (uint32_t)(32 - __builtin_clz(n)) - 5, unit = 8u << k;
  if (n > 3 * unit) {
    k++;
    unit <<= 1;
  }
  return (int)(2 * k + (n > 2 * unit));
}

/* first probe position for a ticket (src/halloc.cu:107-122): tmod
   consecutive tickets share one slot, slots are HASH_FREQ blocks apart, all
   arithmetic wraps at 32 bits */
static uint32_t first_probe(const size_class_t *c, uint32_t ticket) {
  uint32_t low = c->tmod - 1;
  uint32_t spread = (ticket & ~low) * HASH_FREQ + (ticket & low);
  return spread * c->ncib % c->nchunks;
}

/* Tries to reserve a block in slab sb, probing from `first` with the
   ticket's step sequence; *round carries the probe count across calls
   (src/slab.cuh:453-535).  Returns the byte offset or -1. */
static int64_t probe_slab(ham_t *m, uint32_t sb, uint32_t sid, uint32_t first,
                          uint32_t *round, int *want_head) {
  const size_class_t *c = &m->cls[sid];
  if (sb == NO_SLAB) {
    *want_head = 1;
    return -1;
  }
  uint32_t *bits = m->bits + (size_t)sb * m->bit_words;
  uint32_t pos = first, block = (1u << c->ncib) - 1;
  int got = 0;
  do {
    uint32_t w = pos / 32, mask = block << (pos % 32);
    uint32_t before = bits[w];
    if (!(before & mask)) {
      bits[w] = before | mask;
      got = 1;
      break;
    }
    /* a collision leaves the word as it was */
    if (*round % COUNT_CHECK_PERIOD == COUNT_CHECK_PERIOD - 1 &&
        used(m, sb) >= c->busy)
      break;
    uint32_t k = *round + 1;
    uint32_t step = k * STEP_SCALE * c->ncib % c->hash_step;
    pos = (first + k * step) % c->nchunks;
  } while (++*round % TRIES_PER_ROUND < TRIES_PER_ROUND - 1);
  if (!got) {
    *want_head = 1;
    return -1;
  }
  uint32_t flags = count_up(m, sb, sid);
  if (!(flags & 1)) {
    /* the slab changed chunk size under us: give the block back */
    bits[pos / 32] &= ~(block << (pos % 32));
    count_down(m, sb, c->ncib);
    *want_head = 1;
    return -1;
  }
  if (flags & 2) *want_head = 1;
  uint32_t *nib = m->nib + (size_t)sb * m->nib_words;
  nib[pos / 8] |= c->ncib << (pos % 8 * 4);
  return (int64_t)sb * m->sb_bytes + (int64_t)pos * c->chunk_bytes;
}

/* src/halloc.cu:125-182, one thread alone in its warp */
static int64_t alloc_small(ham_t *m, uint32_t sid) {
  uint32_t sb = m->head[sid];
  uint32_t first = first_probe(&m->cls[sid], m->ticket[sid]++);
  uint32_t round = 0;
  for (;;) {
    int want_head = 0;
    int64_t off = probe_slab(m, sb, sid, first, &round, &want_head);
    if (want_head) {
      sb = replace_head(m, sid);
      if (off < 0 && sb == NO_SLAB) return -1;
    }
    if (off >= 0) return off;
  }
}

int64_t ham_malloc(ham_t *m, uint64_t nbytes) {
  int sid = ham_size_id(nbytes);
  if (sid < 0) return -2 - m->nlarge++;
  return alloc_small(m, (uint32_t)sid);
}

/* src/halloc.cu:211-230 (grid lookup replaced by the contiguous layout) */
void ham_free(ham_t *m, int64_t h) {
  if (h < 0) return; /* NULL, or a block of the CUDA heap */
  uint32_t sb = (uint32_t)(h >> m->sb_sh);
  if (sb >= m->nsbs) return;
  uint32_t in = (uint32_t)(h & (m->sb_bytes - 1));
  uint32_t ichunk = chunk_index(in, m->d_chunk_enc[sb]);
  if (ichunk >= m->nib_words * 8) return; /* not a block start */
  uint32_t *nib = m->nib + (size_t)sb * m->nib_words;
  uint32_t sh = ichunk % 8 * 4;
  uint32_t n = (nib[ichunk / 8] >> sh) & 15u;
  nib[ichunk / 8] &= ~(15u << sh);
  m->bits[(size_t)sb * m->bit_words + ichunk / 32] &=
      ~(((1u << n) - 1) << (ichunk % 32));
  count_down(m, sb, n);
}

void ham_run_ops(ham_t *m, const int64_t *ops, int64_t n, int64_t *out) {
  for (int64_t i = 0; i < n; i++) {
    if (ops[i] >= 0) {
      out[i] = ham_malloc(m, (uint64_t)ops[i]);
    } else {
      ham_free(m, out[-(ops[i] + 1)]);
      out[i] = 0;
    }
  }
}

/* ---- state export in the reference's encoding ----------------------- */

uint32_t ham_nsbs(const ham_t *m) { return m->nsbs; }
uint32_t ham_nsizes(const ham_t *m) { (void)m; return NSIZES; }
uint32_t ham_bit_words(const ham_t *m) { return m->bit_words; }
uint32_t ham_nib_words(const ham_t *m) { return m->nib_words; }

void ham_get_size_infos(const ham_t *m, uint32_t *out) {
  for (int s = 0; s < NSIZES; s++) {
    const size_class_t *c = &m->cls[s];
    uint32_t *o = out + 8 * s;
    o[0] = c->nchunks;
    o[1] = chunk_enc(c->chunk_bytes);
    o[2] = c->chunk_id;
    o[3] = c->ncib;
    o[4] = c->sparse;
    o[5] = c->hash_step;
    o[6] = c->roomy;
    o[7] = c->busy;
  }
}

void ham_get_tickets(const ham_t *m, uint32_t *out) {
  memcpy(out, m->ticket, sizeof(m->ticket));
}

void ham_get_heads(const ham_t *m, uint32_t *head, uint32_t *cached) {
  memcpy(head, m->head, sizeof(m->head));
  memcpy(cached, m->cached, sizeof(m->cached));
}

void ham_get_slabs(const ham_t *m, uint32_t *counter, uint32_t *size_id,
                   uint32_t *chunk_id, uint32_t *is_head, uint32_t *chunk_sz) {
  size_t n = (size_t)m->nsbs * 4;
  memcpy(counter, m->ctr, n);
  memcpy(size_id, m->d_size, n);
  memcpy(chunk_id, m->d_chunk, n);
  memcpy(is_head, m->d_head, n);
  memcpy(chunk_sz, m->d_chunk_enc, n);
}

void ham_get_sets(const ham_t *m, uint32_t *out, uint32_t nwords) {
  for (int k = 0; k < NSETS; k++)
    for (uint32_t w = 0; w < nwords; w++)
      out[(size_t)k * nwords + w] =
          w < m->set_words ? m->sets[(size_t)k * m->set_words + w] : 0;
}

void ham_get_bits(const ham_t *m, uint32_t sb, uint32_t *out, uint32_t nwords) {
  for (uint32_t w = 0; w < nwords; w++)
    out[w] = w < m->bit_words ? m->bits[(size_t)sb * m->bit_words + w] : 0;
}

void ham_get_alloc_sizes(const ham_t *m, uint32_t sb, uint32_t *out,
                         uint32_t nwords) {
  for (uint32_t w = 0; w < nwords; w++)
    out[w] = w < m->nib_words ? m->nib[(size_t)sb * m->nib_words + w] : 0;
}

/* ---- CPU baselines -------------------------------------------------- */

static double wall_s(void) {
  struct timespec ts;
  clock_gettime(CLOCK_MONOTONIC, &ts);
  return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

typedef struct {
  uint64_t memory;
  int sb_sh;
  uint32_t t0, t1, niters, nbytes;
  int use_model;
  uint64_t checksum, nfail;
} plain_job_t;

static void *plain_job(void *vp) {
  plain_job_t *j = (plain_job_t *)vp;
  ham_t *m = NULL;
  char *payload = NULL;
  if (j->use_model) {
    m = ham_create(j->memory, 0.75, 0.835, 0.6, 0.012, j->sb_sh, 0);
    if (m) payload = (char *)malloc((size_t)m->nsbs << m->sb_sh);
    if (!m || !payload) {
      j->nfail = (uint64_t)(j->t1 - j->t0) * j->niters;
      ham_destroy(m);
      return NULL;
    }
  }
  uint64_t sum = 0, nfail = 0;
  for (uint32_t t = j->t0; t < j->t1; t++) {
    for (uint32_t it = 0; it < j->niters; it++) {
      uint32_t *p;
      int64_t h = 0;
      if (m) {
        h = ham_malloc(m, j->nbytes);
        p = h >= 0 ? (uint32_t *)(payload + h) : NULL;
      } else {
        p = (uint32_t *)malloc(j->nbytes);
      }
      if (!p) {
        nfail++;
        continue;
      }
      for (uint32_t k = 0; k < 4; k++) p[k] = t ^ k;
      for (uint32_t k = 0; k < 4; k++) sum += ((volatile uint32_t *)p)[k];
      if (m)
        ham_free(m, h);
      else
        free(p);
    }
  }
  j->checksum = sum;
  j->nfail = nfail;
  free(payload);
  ham_destroy(m);
  return NULL;
}

static double plain_run(int use_model, uint64_t memory, int sb_sh,
                        uint32_t nthreads, uint32_t niters, uint32_t nbytes,
                        int nworkers, uint64_t *checksum, uint64_t *nfail) {
  if (nworkers < 1) nworkers = 1;
  if (nworkers > 256) nworkers = 256;
  pthread_t th[256];
  plain_job_t job[256];
  for (int w = 0; w < nworkers; w++) {
    plain_job_t *j = &job[w];
    memset(j, 0, sizeof(*j));
    j->memory = memory;
    j->sb_sh = sb_sh;
    j->t0 = (uint32_t)((uint64_t)nthreads * w / nworkers);
    j->t1 = (uint32_t)((uint64_t)nthreads * (w + 1) / nworkers);
    j->niters = niters;
    j->nbytes = nbytes < 16 ? 16 : nbytes;
    j->use_model = use_model;
  }
  double t0 = wall_s();
  for (int w = 0; w < nworkers; w++) pthread_create(&th[w], NULL, plain_job, &job[w]);
  for (int w = 0; w < nworkers; w++) pthread_join(th[w], NULL);
  double dt = wall_s() - t0;
  *checksum = 0;
  *nfail = 0;
  for (int w = 0; w < nworkers; w++) {
    *checksum += job[w].checksum;
    *nfail += job[w].nfail;
  }
  return dt;
}

double ham_plain_run(uint64_t memory, int sb_sz_sh, uint32_t nthreads,
                     uint32_t niters, uint32_t nbytes, int nworkers,
                     uint64_t *checksum, uint64_t *nfail) {
  return plain_run(1, memory, sb_sz_sh, nthreads, niters, nbytes, nworkers,
                   checksum, nfail);
}

double hostmalloc_plain_run(uint32_t nthreads, uint32_t niters,
                            uint32_t nbytes, int nworkers, uint64_t *checksum,
                            uint64_t *nfail) {
  return plain_run(0, 0, 22, nthreads, niters, nbytes, nworkers, checksum,
                   nfail);
}
