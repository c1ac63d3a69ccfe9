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

/* Device operator new / delete served by hamalloc / hafree, when the
   program is compiled with -DHALLOC_CPP and linked with libhalloc_cpp.a
   (replaces halloc src/halloc.h:71-80, disabled there).  Only the scalar
   forms are replaced, as in the original. */
#if defined(HALLOC_CPP)
__device__ void *operator new(size_t nbytes);
__device__ void operator delete(void *p) noexcept;
__device__ void operator delete(void *p, size_t nbytes) noexcept;
#endif

#endif
