/*
 * phase_draws.cpp -- runs the decision logic of halloc's phase-throughput
 * test on the host, from the reference's own test harness header
 * (tst/common/common.h: drandom, CommonOpts::next_action, next_alloc_sz),
 * compiled unchanged as host C++ under cuda_host_shim.h.  TEST
 * INFRASTRUCTURE ONLY: it pins the oracle's restatement of those draws
 * (oracle/phase.py) and is never part of the product path.
 *
 * Allocation and free are left out: the loop below is prob_throughput_k
 * (tst/perf/phase-throughput/phase-throughput.cu:17-48) with T::malloc and
 * T::free replaced by recording the size drawn, so it yields, for every
 * try, each thread's block count and the sizes of the blocks it holds.
 */
#include <vector>

/* drandom() reads the calling GPU thread's index */
struct ha_dim3 {
  unsigned x, y, z;
};
static ha_dim3 threadIdx, blockIdx, blockDim;
/* named by common.h's run_test template, never called here */
static inline cudaError_t cudaSetDevice(int) { return cudaSuccess; }

/* defines random_states_g (a plain host pointer under the shim) */
#define COMMONTEST_COMPILING
#include "common.h"

extern "C" int ref_phase_draws(const uint32_t *seeds, uint32_t nthreads, const float *probs,
                               uint32_t smin, uint32_t smax, uint32_t nallocs,
                               uint32_t ntries, uint32_t niters, uint32_t *ctr_out,
                               uint32_t *size_out, uint32_t *states_out) {
  CommonOpts o;
  o.alloc_sz = smin;
  o.max_alloc_sz = smax;
  o.distr_type = DistrUniform;
  o.niters = niters;
  o.nallocs = nallocs;
  o.probabs[0][0] = probs[0];
  o.probabs[0][1] = probs[1];
  o.probabs[1][0] = probs[2];
  o.probabs[1][1] = probs[3];
  std::vector<uint> st(seeds, seeds + nthreads), ctr(nthreads, 0);
  std::vector<uint> sz((size_t)nallocs * nthreads, 0);
  random_states_g = st.data();
  blockIdx.x = 0;
  blockDim.x = nthreads;
  for (uint32_t itry = 0; itry < ntries; itry++) {
    for (uint32_t i = 0; i < nthreads; i++) {
      threadIdx.x = i;
      uint c = ctr[i];
      for (uint32_t iter = 0; iter < niters; iter++) {
        switch (o.next_action(c > 0, itry, iter)) {
          case ActionAlloc:
            for (uint32_t k = 0; k < nallocs; k++) sz[(size_t)k * nthreads + i] = o.next_alloc_sz();
            c = nallocs;
            break;
          case ActionFree:
            for (uint32_t k = 0; k < nallocs; k++) sz[(size_t)k * nthreads + i] = 0;
            c = 0;
            break;
          case ActionNone:
            break;
        }
      }
      ctr[i] = c;
    }
    for (uint32_t i = 0; i < nthreads; i++) ctr_out[(size_t)itry * nthreads + i] = ctr[i];
    for (size_t k = 0; k < sz.size(); k++) size_out[(size_t)itry * sz.size() + k] = sz[k];
  }
  for (uint32_t i = 0; i < nthreads; i++) states_out[i] = st[i];
  return 0;
}
