/*
 * Host replacement for the reference's src/utils.h, used only when the
 * reference allocator is compiled as host code for the oracle.
 *
 * The original header holds inline PTX (%laneid, ld.global.ca) and CUDA
 * runtime macros that cannot compile for the host.  This file supplies the
 * same names with host meanings:
 *   - symbol copies (cuset, cuset_arr, cuvar_memset, cuget) become memcpy /
 *     memset on the host-resident "device" globals (src/utils.h:17-50);
 *   - the spin locks (src/utils.h:86-97) keep their atomicExch protocol;
 *   - warp helpers describe a single-lane warp (src/utils.h:107-138);
 *   - ldca (src/utils.h:141-157) is a relaxed atomic load.
 * The constants keep the reference's values, since the data layout of the
 * compiled allocator depends on them.
 */
#ifndef HALLOC_UTILS_H_
#define HALLOC_UTILS_H_

#define cucheck(call)                                                      \
  {                                                                        \
    cudaError_t cucheck_err_ = (call);                                     \
    if (cucheck_err_ != cudaSuccess) {                                     \
      fprintf(stderr, "%s (%d): host shim failure in %s\n", __FILE__,      \
              __LINE__, #call);                                            \
      exit(-1);                                                            \
    }                                                                      \
  }
#define cuset(symbol, T, val)                                              \
  {                                                                        \
    T cuset_val_ = (val);                                                  \
    memcpy((void *)&(symbol), &cuset_val_, sizeof(cuset_val_));            \
  }
#define cuget(pval, symbol)                                                \
  { memcpy((pval), (void *)&(symbol), sizeof(*(pval))); }
#define cuset_arr(symbol, val)                                             \
  { memcpy((void *)&(symbol), *(val), sizeof(*(val))); }
#define cuvar_memset(symbol, val, sz)                                      \
  { memset((void *)&(symbol), (val), (sz)); }

typedef unsigned long long uint64;

#define WORD_SZ 32
#define WARP_SZ 32
#define MAX_NSBS 8192
#define SB_SET_SZ (MAX_NSBS / WORD_SZ)
#define MAX_NWARPS 32

inline int divup(int a, int b) { return (a + b - 1) / b; }

/* test-and-set lock on a 32-bit word, same protocol as the device code */
inline bool try_lock(uint *mutex) { return atomicExch(mutex, 1) == 0; }
inline void lock(uint *mutex) {
  while (!try_lock(mutex)) {
  }
}
inline void unlock(uint *mutex) {
  __threadfence();
  atomicExch(mutex, 0);
}
inline void wait_unlock(uint *mutex) {
  while (__atomic_load_n(mutex, __ATOMIC_SEQ_CST)) {
  }
}

/* a warp here has exactly one lane, lane 0 */
inline uint warp_leader(uint mask) { return __ffs(mask) - 1; }
inline uint lane_id(void) { return 0; }
inline uint warp_id(void) { return 0; }
inline uint warp_bcast(uint v, uint) { return v; }
inline uint lanemask_lt(void) { return 0; }

inline uint ldca(const uint *p) { return __atomic_load_n(p, __ATOMIC_RELAXED); }
inline uint64 ldca(const uint64 *p) {
  return __atomic_load_n(p, __ATOMIC_RELAXED);
}
inline void *ldca(void *const *p) {
  return __atomic_load_n(p, __ATOMIC_RELAXED);
}
inline void prefetch_l1(const void *) {}
inline void prefetch_l2(const void *) {}

/* defined by the reference's src/utils.cu, compiled unchanged */
uint max_prime_below(uint n, uint nb);

#endif
