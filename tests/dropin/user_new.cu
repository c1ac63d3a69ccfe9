// A program that allocates device objects with new / delete, compiled with
// -DHALLOC_CPP and linked with libhalloc.a, so that device operator new and
// delete are served by the allocator.  Prints "OK" and exits 0 when every
// object was created and holds its value, every array is 16-byte aligned,
// the objects sit in the allocator's slabs (its used-chunk count is what
// they need) and all were deleted (the count returns to 0).
#include <halloc.h>
#include <halloc_c.h>
#include <stdint.h>
#include <stdio.h>

struct item {  // 16 bytes: one 16-byte chunk
  int key;
  item *next;
  __device__ item(int k, item *n) : key(k), next(n) {}
};

// 48 bytes, 16-byte aligned: served from the 64-byte class (four chunks)
struct vec3x4 {
  float4 v[3];
};

__global__ void make_k(item **heads, vec3x4 **arrs, int n, int len,
                       unsigned long long *bad) {
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
  vec3x4 *a = new vec3x4[1];
  if (!a || ((uintptr_t)a & 15)) {
    atomicAdd(bad, 1ull);
    a = nullptr;
  } else {
    for (int j = 0; j < 3; j++) a->v[j] = make_float4(i, j, -i, -j);
  }
  arrs[i] = a;
}

__global__ void drop_k(item **heads, vec3x4 **arrs, int n, int len, unsigned long long *bad) {
  int i = threadIdx.x + blockIdx.x * blockDim.x;
  if (i >= n) return;
  int k = len;
  for (item *x = heads[i]; x;) {
    item *nx = x->next;
    if (x->key != i * len + --k) atomicAdd(bad, 1ull);
    delete x;
    x = nx;
  }
  vec3x4 *a = arrs[i];
  if (a) {
    for (int j = 0; j < 3; j++) {
      float4 w = a->v[j];
      if (w.x != i || w.y != j || w.z != -i || w.w != -j) atomicAdd(bad, 1ull);
    }
    delete[] a;
  }
}

int main() {
  const int n = 1 << 15, len = 4;
  ha_init(halloc_opts_t(256 << 20));
  item **heads;
  vec3x4 **arrs;
  unsigned long long *bad, hbad = 0;
  cudaMalloc(&heads, n * sizeof(item *));
  cudaMalloc(&arrs, n * sizeof(vec3x4 *));
  cudaMalloc(&bad, sizeof(unsigned long long));
  cudaMemset(bad, 0, sizeof(unsigned long long));
  make_k<<<n / 128, 128>>>(heads, arrs, n, len, bad);
  ha_stats_t before;
  if (ha_stats_c(&before) != HA_OK) return 3;
  drop_k<<<n / 128, 128>>>(heads, arrs, n, len, bad);
  ha_stats_t after;
  if (ha_stats_c(&after) != HA_OK) return 3;
  cudaMemcpy(&hbad, bad, sizeof(hbad), cudaMemcpyDeviceToHost);
  cudaError_t err = cudaGetLastError();
  ha_shutdown();
  const unsigned long long want = (unsigned long long)n * len + 4ull * n;
  if (err != cudaSuccess || hbad || before.used_chunks != want || after.used_chunks != 0) {
    printf("FAIL err %d bad %llu used before %llu (want %llu) after %llu\n", (int)err, hbad,
           (unsigned long long)before.used_chunks, want, (unsigned long long)after.used_chunks);
    return 1;
  }
  printf("OK %d objects and %d arrays through device new/delete\n", n * len, n);
  return 0;
}
