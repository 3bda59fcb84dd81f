// Update and residual norms without any device allocation.
//
// Some callers cannot call cudaMalloc at the moment they need this step: a
// host code that owns every device buffer through its own pool and forbids
// allocations from libraries, a time loop that must not pay the device-wide
// synchronisation an allocation can imply, or a process that has already
// committed the whole GPU memory to its own arrays.  For them this file holds
// one entry point that works on caller-owned device arrays only: the primitive
// update of Dual_time_stepping.cpp:1702-1743 and the five norms of
// :1761-1782, the same arithmetic as the context path (kernels_ref.cu,
// k_update + k_norms), whose per-row partial sums live in context memory.
// Here the partial sums live in one file-scope device array of fixed size,
// whose device address every call looks up with cudaGetSymbolAddress (no
// allocation) on the current device.
#include <cuda_runtime.h>

#include <cmath>
#include <string>

#include "../../include/cgli_fu_flow.h"
#include "cgli_dev.cuh"
#include "cgli_launch.h"

namespace {

// Per-row partial sums (5 doubles per (i, j) row of the slab) followed by the
// five reduced norms.  Every GPU that loads the library holds this array
// (5 MiB) until the process exits.
__device__ __align__(256) double g_noalloc_scratch[5 * CGLI_NOALLOC_MAX_ROWS + 8];

struct Ptr5 {
  double *p[5];
};
struct CPtr5 {
  const double *p[5];
};

// k_update of kernels_ref.cu with the partial sums written to `partial`;
// one block per (i, j) row, row r = (i - 3) * Ny + (j - 2) on a 1-D grid
__global__ void k_update_noalloc(int ny, int nz, long long di, long long dj, Ptr5 q, const double *J, CPtr5 nr,
                                 double *partial) {
  const int i = 3 + blockIdx.x / ny, j = 2 + blockIdx.x % ny;
  double acc[5] = {0, 0, 0, 0, 0};
  for (int k = 2 + threadIdx.x; k <= nz + 1; k += blockDim.x) {
    const long long c = (long long)i * di + (long long)j * dj + k;
    const double Jc = J[c];
    double q1 = q.p[0][c];
    double rhoold = q1 * Jc;
    double Uold = q.p[1][c] / q1, Vold = q.p[2][c] / q1, Wold = q.p[3][c] / q1;
    double VVold = Uold * Uold + Vold * Vold + Wold * Wold;
    double Pold = (q.p[4][c] * Jc - 0.5 * rhoold * VVold) * (cgli::KG - 1);
    double Told = Pold / rhoold;
    double P = Pold + nr.p[0][c] * Jc;
    double U = Uold + nr.p[1][c] * Jc;
    double V = Vold + nr.p[2][c] * Jc;
    double W = Wold + nr.p[3][c] * Jc;
    double T = Told + nr.p[4][c] * Jc;
    double rho = P / T;
    q.p[0][c] = rho / Jc;
    q.p[1][c] = rho * U / Jc;
    q.p[2][c] = rho * V / Jc;
    q.p[3][c] = rho * W / Jc;
    q.p[4][c] = (P / (cgli::KG - 1) + 0.5 * rho * (U * U + V * V + W * W)) / Jc;
    acc[0] += (rho - rhoold) * (rho - rhoold);
    acc[1] += (U - Uold) * (U - Uold);
    acc[2] += (V - Vold) * (V - Vold);
    acc[3] += (W - Wold) * (W - Wold);
    acc[4] += (T - Told) * (T - Told);
  }
  // every row writes its own five sums, so no part of the scratch has to
  // start at zero; only the rows of this call are read back
  cgli::block_sum5(acc, partial + 5 * (long long)blockIdx.x);
}

// k_norms of kernels_ref.cu
__global__ void k_norms_noalloc(const double *partial, int nrows, double scale, double *out) {
  double acc[5] = {0, 0, 0, 0, 0};
  for (int b = threadIdx.x; b < nrows; b += blockDim.x)
    for (int v = 0; v < 5; v++) acc[v] += partial[5 * (long long)b + v];
  __shared__ double tot[5];
  cgli::block_sum5(acc, tot);
  __syncthreads();
  if (threadIdx.x < 5) out[threadIdx.x] = sqrt(tot[threadIdx.x]) * scale;
}

int fail(int code, const std::string &m) {
  cgli::set_last_error(m);   // reported by cgli_last_error()
  return code;
}

}  // namespace

extern "C" {

int cgli_update_norms_noalloc(int nx, int ny, int nz, double *const U_[5], const double *J,
                              const double *const NR[5], double er[5], void *stream) {
  if (nx < 1 || ny < 1 || nz < 1 || !U_ || !J || !NR || !er) return fail(CGLI_EINVAL, "bad argument");
  if ((long long)nx * ny > CGLI_NOALLOC_MAX_ROWS)
    return fail(CGLI_EINVAL, "Nx*Ny = " + std::to_string((long long)nx * ny) +
                                 " rows exceeds the fixed scratch of CGLI_NOALLOC_MAX_ROWS = " +
                                 std::to_string(CGLI_NOALLOC_MAX_ROWS) + " rows");
  Ptr5 q;
  CPtr5 n;
  for (int v = 0; v < 5; v++) {
    if (!U_[v] || !NR[v]) return fail(CGLI_EINVAL, "null array");
    q.p[v] = U_[v];
    n.p[v] = NR[v];
  }
  // The device address of the static array on the current device.  The
  // array's host-side name is only a stand-in for it; the address belongs to
  // the device's current context and changes if that context is torn down
  // and created again (cudaDeviceReset), so it is looked up on every call
  // (a table lookup in the runtime: nothing is allocated).
  void *p = nullptr;
  cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p)
    return fail(CGLI_ECUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  double *scratch = (double *)p;
  cudaStream_t s = (cudaStream_t)stream;
  const long long dj = nz + 4, di = (long long)(ny + 4) * (nz + 4);
  const int nrows = nx * ny;
  double *norms = scratch + 5 * (long long)CGLI_NOALLOC_MAX_ROWS;
  k_update_noalloc<<<nrows, 128, 0, s>>>(ny, nz, di, dj, q, J, n, scratch);
  k_norms_noalloc<<<1, 1024, 0, s>>>(scratch, nrows, 1.0 / ((double)nx * ny * nz), norms);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(CGLI_ECUDA, std::string("launch: ") + cudaGetErrorString(e));
  e = cudaMemcpyAsync(er, norms, 5 * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail(CGLI_ECUDA, std::string("norm read-back: ") + cudaGetErrorString(e));
  return CGLI_OK;
}

}  // extern "C"
