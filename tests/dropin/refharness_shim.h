/* Force-included (nvcc -include) ahead of halloc's test harness library,
 * tst/common/common.cu, which is compiled from the reference tree unchanged.
 *
 * The harness opens `using namespace thrust;` at global scope.  With the
 * thrust of CUDA 12 that brings in thrust's `cuda` namespace alias, which
 * collides with ::cuda in the host stubs nvcc generates for the thrust kernels
 * the harness instantiates; and thrust::plus is cuda::std::plus, so argument-
 * dependent lookup makes its unqualified reduce() call ambiguous with
 * cuda::std::reduce.  The harness predates both.  So: the thrust headers it
 * uses are included here first (their include guards keep its own #includes
 * from re-reading them), the six thrust names it uses are gathered in a
 * namespace of their own, its `using namespace thrust;` is pointed at that
 * namespace, and its one reduce() call is qualified.  The harness's source
 * and its behaviour are otherwise untouched. */
#ifndef HALLOC_B200_REFHARNESS_SHIM_H_
#define HALLOC_B200_REFHARNESS_SHIM_H_
#include <thrust/device_ptr.h>
#include <thrust/functional.h>
#include <thrust/iterator/counting_iterator.h>
#include <thrust/logical.h>
#include <thrust/reduce.h>
#include <thrust/sort.h>
namespace halloc_b200_refharness {
using thrust::all_of;
using thrust::counting_iterator;
using thrust::device_ptr;
using thrust::plus;
using thrust::reduce;
using thrust::sort;
}  // namespace halloc_b200_refharness
#define thrust halloc_b200_refharness
#define reduce thrust::reduce
#endif
