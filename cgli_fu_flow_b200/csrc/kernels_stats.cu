// Running statistics of Statistic.cpp:120-160: per (i, j) sums over k of
// U, V, W, T, UU, VV, WW, TT, UV, UT, VT of the current U_, accumulated once
// per call (once per physical step), and the instantaneous U and T of cell
// k = 150 (:155-158; kept only when the row has that cell).  One CTA per
// (i, j) row, a fixed-order reduction over k, so repeated runs give
// identical sums.
#include "cgli_dev.cuh"
#include "cgli_launch.h"

namespace cgli {
namespace {

constexpr int NSTAT = 11;   // accumulated quantities; two sampled ones follow
constexpr int KSAMPLE = 150;  // reference k index of the instantaneous sample

__global__ void k_statistics(Dev d, double *sums) {
  const int jl = blockIdx.x, il = blockIdx.y;     // interior row (0-based)
  const int i = il + 3, j = jl + 2;
  double a[NSTAT];
#pragma unroll
  for (int q = 0; q < NSTAT; q++) a[q] = 0.0;
  for (int kl = threadIdx.x; kl < d.nz; kl += blockDim.x) {
    const long long c = ix(d, i, j, kl + 2);
    const double rho = d.U_[0][c];
    const double U = d.U_[1][c] / rho, V = d.U_[2][c] / rho, W = d.U_[3][c] / rho;
    const double VV = U * U + V * V + W * W;
    const double P = (d.U_[4][c] - 0.5 * rho * VV) * (KG - 1) * d.J[c];
    const double T = P / (rho * RG) / d.J[c];
    a[0] += U; a[1] += V; a[2] += W; a[3] += T;
    a[4] += U * U; a[5] += V * V; a[6] += W * W; a[7] += T * T;
    a[8] += U * V; a[9] += U * T; a[10] += V * T;
    if (kl + 2 == KSAMPLE) {
      sums[((long long)NSTAT * d.nx + il) * d.ny + jl] = U;
      sums[((long long)(NSTAT + 1) * d.nx + il) * d.ny + jl] = T;
    }
  }
  __shared__ double red[NSTAT][128];
#pragma unroll
  for (int q = 0; q < NSTAT; q++) red[q][threadIdx.x] = a[q];
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s)
#pragma unroll
      for (int q = 0; q < NSTAT; q++) red[q][threadIdx.x] += red[q][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x < NSTAT) {
    const long long o = ((long long)threadIdx.x * d.nx + il) * d.ny + jl;
    sums[o] += red[threadIdx.x][0];
  }
}

}  // namespace

void launch_statistics(const Dev &d, cudaStream_t s, double *sums) {
  k_statistics<<<dim3(d.ny, d.nx), 128, 0, s>>>(d, sums);
}

}  // namespace cgli
