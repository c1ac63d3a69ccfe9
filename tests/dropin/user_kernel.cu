// A user program written against the halloc API only (include/halloc.h),
// compiled with -rdc and linked with libhalloc.a: the drop-in check.
//
// Every thread builds a linked list of 16-byte nodes with hamalloc, a few
// threads also take a large (> 3 KiB) buffer from the CUDA heap through
// hamalloc, a second kernel sums and frees everything.  Prints "OK" and
// exits 0 when the sums match.
#include <halloc.h>
#include <stdio.h>
#include <stdlib.h>

struct node {
  int value;
  node *next;
};

__global__ void build_k(node **heads, void **bufs, int n, int len) {
  int i = threadIdx.x + blockIdx.x * blockDim.x;
  if (i >= n) return;
  node *h = 0;
  for (int k = 0; k < len; k++) {
    node *x = (node *)hamalloc(sizeof(node));
    if (!x) break;
    x->value = i + k;
    x->next = h;
    h = x;
  }
  heads[i] = h;
  bufs[i] = (i % 97 == 0) ? hamalloc(8192) : 0;
  if (bufs[i]) ((int *)bufs[i])[2047] = i;
}

__global__ void sum_free_k(node **heads, void **bufs, int n, unsigned long long *sum,
                           unsigned long long *bad) {
  int i = threadIdx.x + blockIdx.x * blockDim.x;
  if (i >= n) return;
  unsigned long long s = 0;
  for (node *x = heads[i]; x;) {
    node *nx = x->next;
    s += x->value;
    hafree(x);
    x = nx;
  }
  if (bufs[i]) {
    if (((int *)bufs[i])[2047] != i) atomicAdd(bad, 1ull);
    hafree(bufs[i]);
  }
  atomicAdd(sum, s);
}

int main() {
  const int n = 1 << 16, len = 6;
  ha_init(halloc_opts_t(256 << 20));
  node **heads;
  void **bufs;
  unsigned long long *d;
  cudaMalloc(&heads, n * sizeof(node *));
  cudaMalloc(&bufs, n * sizeof(void *));
  cudaMalloc(&d, 2 * sizeof(unsigned long long));
  cudaMemset(d, 0, 2 * sizeof(unsigned long long));
  build_k<<<n / 128, 128>>>(heads, bufs, n, len);
  sum_free_k<<<n / 128, 128>>>(heads, bufs, n, d, d + 1);
  unsigned long long h[2];
  cudaError_t e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) {
    printf("CUDA error %s\n", cudaGetErrorString(e));
    return 2;
  }
  unsigned long long want = 0;
  for (int i = 0; i < n; i++)
    for (int k = 0; k < len; k++) want += (unsigned long long)(i + k);
  double frag = ha_extfrag(false);
  ha_shutdown();
  if (h[0] != want || h[1] != 0) {
    printf("FAIL sum %llu want %llu bad %llu\n", h[0], want, h[1]);
    return 1;
  }
  printf("OK sum %llu extfrag %.3f\n", h[0], frag);
  return 0;
}
