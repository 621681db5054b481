// hvm64_atomic_peak -- the L2 atomic rate that bounds the reducer next to HBM
// bandwidth: 64-bit atomicExch and atomicCAS on random words of a large
// array (the reducer's heap accesses are 8-byte atomics at data-dependent
// addresses).  Prints one JSON line: operations per second for each.
//
//   hvm64_atomic_peak [GiB (default 4)] [iterations per thread (default 256)]
#include <cuda_runtime.h>
#include <stdio.h>
#include <stdlib.h>

#define CK(x)                                                                  \
  do {                                                                         \
    cudaError_t e_ = (x);                                                      \
    if (e_ != cudaSuccess) {                                                   \
      fprintf(stderr, "%s: %s\n", #x, cudaGetErrorString(e_));                 \
      return 1;                                                                \
    }                                                                          \
  } while (0)

__global__ void exch_kernel(unsigned long long* a, unsigned long long n, unsigned iters, unsigned long long* sink) {
  unsigned long long x = 0x9E3779B97F4A7C15ull ^ (blockIdx.x * 1024ull + threadIdx.x);
  unsigned long long acc = 0;
  for (unsigned i = 0; i < iters; i++) {
    x ^= x << 13;
    x ^= x >> 7;
    x ^= x << 17;
    acc += atomicExch(a + (x % n), x);
  }
  if (acc == 42) *sink = acc;  // keeps the results live
}

__global__ void cas_kernel(unsigned long long* a, unsigned long long n, unsigned iters, unsigned long long* sink) {
  unsigned long long x = 0xD1B54A32D192ED03ull ^ (blockIdx.x * 1024ull + threadIdx.x);
  unsigned long long acc = 0;
  for (unsigned i = 0; i < iters; i++) {
    x ^= x << 13;
    x ^= x >> 7;
    x ^= x << 17;
    unsigned long long* p = a + (x % n);
    acc += atomicCAS(p, acc, x);
  }
  if (acc == 42) *sink = acc;
}

int main(int argc, char** argv) {
  double gib = argc > 1 ? atof(argv[1]) : 4.0;
  unsigned iters = argc > 2 ? unsigned(atoi(argv[2])) : 256;
  if (gib <= 0 || gib > 64 || iters == 0 || iters > 65536) {
    fprintf(stderr, "usage: hvm64_atomic_peak [GiB 0..64] [iterations 1..65536]\n");
    return 2;
  }
  unsigned long long n = (unsigned long long)(gib * (1ull << 30)) / 8;
  unsigned long long *a = nullptr, *sink = nullptr;
  CK(cudaMalloc(&a, n * 8));
  CK(cudaMalloc(&sink, 8));
  CK(cudaMemset(a, 0, n * 8));
  int sms = 0;
  CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0));
  unsigned blocks = unsigned(sms) * 8, threads = 256;
  double ops = double(blocks) * threads * iters;
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  float best[2] = {1e30f, 1e30f};
  for (int rep = 0; rep < 4; rep++) {
    for (int k = 0; k < 2; k++) {
      CK(cudaEventRecord(e0));
      if (k == 0) exch_kernel<<<blocks, threads>>>(a, n, iters, sink);
      else cas_kernel<<<blocks, threads>>>(a, n, iters, sink);
      CK(cudaGetLastError());
      CK(cudaEventRecord(e1));
      CK(cudaEventSynchronize(e1));
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, e0, e1));
      if (rep > 0 && ms < best[k]) best[k] = ms;  // the first round warms up
    }
  }
  printf("{\"array_gib\": %.2f, \"ops_per_launch\": %.0f, \"atomic_exch_gops\": %.3f, \"atomic_cas_gops\": %.3f}\n",
         gib, ops, ops / (best[0] / 1e3) / 1e9, ops / (best[1] / 1e3) / 1e9);
  cudaFree(a);
  cudaFree(sink);
  return 0;
}
