// Accuracy check of the library's Newton-refined FP64 reciprocal and square
// root (nr_rcp, nr_sqrt in cgli_dev.cuh) against CUDA's IEEE-rounded
// division and sqrt: for n log-uniform operands in [lo, hi) the largest
// difference in units in the last place, per function.  Built and loaded by
// tests/test_fp64_recip.py.
#include <cuda_runtime.h>
#include <stdint.h>

#include "cgli_dev.cuh"

namespace {

__device__ __forceinline__ long long ulp_diff(double a, double b) {
  const long long ia = __double_as_longlong(a), ib = __double_as_longlong(b);
  const long long d = ia > ib ? ia - ib : ib - ia;
  return (ia ^ ib) < 0 ? 0x7fffffffffffffffLL : d;   // sign mismatch: unbounded
}

// splitmix64 -> uniform [0, 1)
__device__ __forceinline__ double uniform(unsigned long long s) {
  s += 0x9E3779B97F4A7C15ull;
  s = (s ^ (s >> 30)) * 0xBF58476D1CE4E5B9ull;
  s = (s ^ (s >> 27)) * 0x94D049BB133111EBull;
  s ^= s >> 31;
  return (double)(s >> 11) * (1.0 / 9007199254740992.0);
}

__global__ void k_check(long long n, unsigned long long seed, double llo, double lhi, unsigned long long *worst) {
  long long rcp = 0, sq = 0;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    const double x = exp(llo + (lhi - llo) * uniform(seed + (unsigned long long)t));
    const long long a = ulp_diff(cgli::nr_rcp(x), 1.0 / x), b = ulp_diff(cgli::nr_sqrt(x), sqrt(x));
    rcp = a > rcp ? a : rcp;
    sq = b > sq ? b : sq;
  }
  atomicMax(worst, (unsigned long long)rcp);
  atomicMax(worst + 1, (unsigned long long)sq);
}

}  // namespace

extern "C" int fp64_recip_check(long long n, unsigned long long seed, double lo, double hi, long long out[2]) {
  unsigned long long *w = nullptr;
  if (cudaMalloc(&w, 2 * sizeof(unsigned long long)) != cudaSuccess) return 1;
  cudaMemset(w, 0, 2 * sizeof(unsigned long long));
  k_check<<<592, 256>>>(n, seed, log(lo), log(hi), w);
  unsigned long long h[2] = {0, 0};
  const cudaError_t e = cudaMemcpy(h, w, sizeof h, cudaMemcpyDeviceToHost);
  cudaFree(w);
  out[0] = (long long)h[0];
  out[1] = (long long)h[1];
  return e == cudaSuccess ? 0 : 2;
}
