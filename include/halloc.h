#ifndef HALLOC_H_
#define HALLOC_H_

/*
 * halloc.h -- public C++ API of halloc-b200, a device-side allocator for
 * NVIDIA B200 (sm_100a).
 *
 * Drop-in for halloc 0.11's src/halloc.h: the option structure keeps the
 * same fields, order, defaults and layout, and the device and host entry
 * points keep the same names, signatures and C++ linkage, so a program
 * written against halloc compiles and device-links against libhalloc.a
 * unchanged:
 *
 *   nvcc -gencode arch=compute_100a,code=sm_100a -rdc=true -c prog.cu
 *   nvcc -gencode arch=compute_100a,code=sm_100a prog.o -lhalloc -o prog
 *
 * Requests of up to 3072 bytes are served from the allocator's slabs;
 * larger ones go to CUDA's in-kernel malloc/free.
 */

#include <stddef.h>

#ifdef HALLOCLIB_COMPILING
#define HALLOC_EXTERN
#else
#define HALLOC_EXTERN extern
#endif

/** allocator options (replaces halloc src/halloc.h:15-34, same layout) */
struct halloc_opts_t {
  /** bytes made available for allocation (slabs + CUDA heap); capped at
      3/4 of device memory */
  size_t memory;
  /** share of `memory` given to slabs; the rest becomes the CUDA heap used
      for requests above 3072 bytes */
  double halloc_fraction;
  /** slab occupancy at which a head slab is replaced */
  double busy_fraction;
  /** occupancy below which a slab is filed as roomy for its block size */
  double roomy_fraction;
  /** occupancy below which a slab may be reused by another block size of
      the same chunk size */
  double sparse_fraction;
  /** log2 of the slab size in bytes (20..24; default 22 = 4 MiB) */
  int sb_sz_sh;
  /** defaults: 512 MiB, 0.75, 0.835, 0.6, 0.012, 22 */
  halloc_opts_t(size_t memory = 512 * 1024 * 1024)
      : memory(memory), halloc_fraction(0.75), busy_fraction(0.835),
        roomy_fraction(0.6), sparse_fraction(0.012), sb_sz_sh(22) {}
};

/** allocates nbytes from device code; NULL when no memory is left
    (replaces halloc src/halloc.h:38) */
HALLOC_EXTERN __device__ __noinline__ void *hamalloc(size_t nbytes);

/** frees a block returned by hamalloc; NULL is ignored
    (replaces halloc src/halloc.h:41) */
HALLOC_EXTERN __device__ __noinline__ void hafree(void *p);

/** initialises the allocator on the current device; must run before any
    kernel that uses hamalloc or CUDA's in-kernel malloc.  Calling it again
    re-initialises (all blocks are released).  On failure it prints the
    reason and exits, like the original.  (replaces halloc src/halloc.h:46) */
void ha_init(halloc_opts_t opts = halloc_opts_t());

/** releases the allocator's device memory on the current device
    (replaces halloc src/halloc.h:49, which was a no-op) */
void ha_shutdown(void);

/** external fragmentation: 1 - (largest block the CUDA heap can still give)
    / (free bytes in slabs and heap).  `ideal` also counts unused slabs as
    allocatable.  (replaces halloc src/halloc.h:55) */
double ha_extfrag(bool ideal);

/* Device operator new / delete served by hamalloc / hafree when the
   program is compiled with -DHALLOC_CPP (replaces halloc src/halloc.h:71-80
   and src/halloc.cu:201-208, 258-265, disabled there).  nvcc binds a device
   new-expression to a replacement operator only when the operator's
   definition is visible in the translation unit, so the definitions are
   here, inline (nonstandard for replacement operators: nvcc warning 2620,
   suppressed).  operator new promises 16-byte alignment, and blocks of the
   24-byte-chunk size classes are only 8-byte aligned, so requests of
   17..24, 33..48, 65..96 and 129..192 bytes are served from the next
   16-byte-chunk class (32, 64, 128, 256 bytes).  The array forms, which
   halloc left commented out, are included.  Failure returns NULL. */
#if defined(HALLOC_CPP)
#pragma nv_diagnostic push
#pragma nv_diag_suppress 2620
__device__ __forceinline__ size_t ha_new_bytes(size_t n) {
  if (n > 16 && n <= 24) return 32;
  if (n > 32 && n <= 48) return 64;
  if (n > 64 && n <= 96) return 128;
  if (n > 128 && n <= 192) return 256;
  return n;
}
__device__ inline void *operator new(size_t n) { return hamalloc(ha_new_bytes(n)); }
__device__ inline void *operator new[](size_t n) { return hamalloc(ha_new_bytes(n)); }
__device__ inline void operator delete(void *p) noexcept { hafree(p); }
__device__ inline void operator delete[](void *p) noexcept { hafree(p); }
__device__ inline void operator delete(void *p, size_t) noexcept { hafree(p); }
__device__ inline void operator delete[](void *p, size_t) noexcept { hafree(p); }
#pragma nv_diagnostic pop
#endif

#endif
