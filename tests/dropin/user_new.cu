// A program that allocates device objects with new / delete, compiled with
// -DHALLOC_CPP and linked with libhalloc_cpp.a, so that device operator new
// and delete are served by the allocator.  Prints "OK" and exits 0 when every
// object was created, holds its value, was served from the allocator's slabs
// (its used-chunk count rises) and was deleted (the count returns to 0).
#include <halloc.h>
#include <halloc_c.h>
#include <stdio.h>

struct item {
  int key;
  item *next;
  __device__ item(int k, item *n) : key(k), next(n) {}
};

__global__ void make_k(item **heads, int n, int len, unsigned long long *bad) {
  int i = threadIdx.x + blockIdx.x * blockDim.x;
  if (i >= n) return;
  item *h = nullptr;
  for (int k = 0; k < len; k++) {
    item *x = new item(i * len + k, h);
    if (!x) {
      atomicAdd(bad, 1ull);
      break;
    }
    h = x;
  }
  heads[i] = h;
}

__global__ void drop_k(item **heads, int n, int len, unsigned long long *bad) {
  int i = threadIdx.x + blockIdx.x * blockDim.x;
  if (i >= n) return;
  int k = len;
  for (item *x = heads[i]; x;) {
    item *nx = x->next;
    if (x->key != i * len + --k) atomicAdd(bad, 1ull);
    delete x;
    x = nx;
  }
}

int main() {
  const int n = 1 << 15, len = 4;
  ha_init(halloc_opts_t(256 << 20));
  item **heads;
  unsigned long long *bad, hbad = 0;
  cudaMalloc(&heads, n * sizeof(item *));
  cudaMalloc(&bad, sizeof(unsigned long long));
  cudaMemset(bad, 0, sizeof(unsigned long long));
  make_k<<<n / 128, 128>>>(heads, n, len, bad);
  ha_stats_t before;
  if (ha_stats_c(&before) != HA_OK) return 3;
  drop_k<<<n / 128, 128>>>(heads, n, len, bad);
  ha_stats_t after;
  if (ha_stats_c(&after) != HA_OK) return 3;
  cudaMemcpy(&hbad, bad, sizeof(hbad), cudaMemcpyDeviceToHost);
  ha_shutdown();
  // item is 16 bytes: one 16-byte chunk each
  if (hbad || before.used_chunks != (unsigned long long)n * len || after.used_chunks != 0) {
    printf("FAIL bad %llu used before %llu after %llu\n", hbad,
           (unsigned long long)before.used_chunks, (unsigned long long)after.used_chunks);
    return 1;
  }
  printf("OK %d objects through device new/delete\n", n * len);
  return 0;
}
