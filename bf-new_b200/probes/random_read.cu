// Random-read ceiling of the B200's memory system for the relaxation
// engines' access pattern: dependent random 8-byte reads (a pointer chase)
// at footprints from 32 MB to 16 GB and 1, 8 or 32 warps per SM.  Each
// thread walks 200 links of an odd-multiplier permutation of the array's
// indices (n a power of two, so the map is a bijection and every value is an
// index < n).  Prints per-load latency and the aggregate loads per second.
//
//   nvcc -gencode arch=compute_100a,code=sm_100a -O3 -o bf-new_b200/probes/random_read \
//        bf-new_b200/probes/random_read.cu && ./bf-new_b200/probes/random_read
#include <cstdio>
#include <cstdint>
#include <vector>
#include <random>
#include <cuda_runtime.h>

__global__ void init_perm(unsigned long long* a, unsigned long long n, unsigned long long stride_mult) {
  unsigned long long i = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
  unsigned long long s = gridDim.x * (unsigned long long)blockDim.x;
  for (; i < n; i += s) a[i] = (i * stride_mult + 12345ull) % n;  // stride_mult coprime with n -> permutation-ish
}

__global__ void chase(const unsigned long long* __restrict__ a, unsigned long long n, int steps,
                      unsigned long long* out, long long* cycles) {
  unsigned long long idx = (blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x) * 7919ull % n;
  long long t0 = clock64();
  for (int k = 0; k < steps; ++k) idx = __ldcg(a + idx);
  long long t1 = clock64();
  if (threadIdx.x == 0) cycles[blockIdx.x] = t1 - t0;
  out[blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x] = idx;
}

int main() {
  int sms = 0; cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
  const size_t sizes_mb[] = {32, 256, 1024, 4096, 16384};
  const int warps_per_sm[] = {1, 8, 32};
  for (size_t mb : sizes_mb) {
    unsigned long long n = mb * 1024ull * 1024ull / 8ull;
    unsigned long long* a = nullptr;
    if (cudaMalloc(&a, n * 8) != cudaSuccess) { printf("alloc %zu MB failed\n", mb); return 1; }
    // large odd multiplier, coprime with n (n is a power of two here)
    init_perm<<<sms * 8, 256>>>(a, n, 2654435761ull);
    cudaDeviceSynchronize();
    for (int w : warps_per_sm) {
      int blocks = sms * (w >= 8 ? w / 8 : 1), threads = w >= 8 ? 256 : 32;
      unsigned long long total = (unsigned long long)blocks * threads;
      unsigned long long* out; long long* cyc;
      cudaMalloc(&out, total * 8); cudaMalloc(&cyc, blocks * 8);
      const int steps = 200;
      chase<<<blocks, threads>>>(a, n, steps, out, cyc);
      cudaEvent_t e0, e1; cudaEventCreate(&e0); cudaEventCreate(&e1);
      cudaEventRecord(e0);
      chase<<<blocks, threads>>>(a, n, steps, out, cyc);
      cudaEventRecord(e1); cudaEventSynchronize(e1);
      float ms = 0; cudaEventElapsedTime(&ms, e0, e1);
      std::vector<long long> c(blocks); cudaMemcpy(c.data(), cyc, blocks * 8, cudaMemcpyDeviceToHost);
      double avg = 0; for (auto x : c) avg += x; avg /= blocks;
      printf("footprint %6zu MB  warps/SM %2d  latency %7.1f cycles (%.2f us)  throughput %.2f G loads/s\n", mb, w,
             avg / steps, avg / steps / 1965.0, total * (double)steps / (ms * 1e6));
      cudaFree(out); cudaFree(cyc);
    }
    cudaFree(a);
  }
  cudaError_t e = cudaGetLastError();
  printf("status %s\n", cudaGetErrorString(e));
  return e == cudaSuccess ? 0 : 1;
}
