// DP-LUR inner solver (DPLUSGS.cpp): four Jacobi relaxations of the
// split-Jacobian operator of the LU-SGS sweeps, then the primitive-variable
// update with the pressure increment as the first norm.
//
// A relaxation is a 7-point stencil with no ordering between cells, so it is
// a plain data-parallel kernel.  Each CTA owns a (j, k) tile of TJ rows x 30
// columns and marches through a chunk of x planes.  Every cell forms its own
// split Jacobians once per plane and applies them to its own previous
// iterate: the "lower" product A+ NL (used by the neighbour above it) and the
// "upper" product A* NL (used by the neighbour below it) in each direction.
// Neighbours exchange those products instead of re-forming each other's
// Jacobians: along k by warp shuffles (one warp per j row, lanes 0 and 31
// the halo columns), along j through shared memory (two extra halo rows),
// along x in registers (the march).  A cell outside the interior contributes
// nothing, which is the reference's zero NL ghost rows (DPLUSGS.cpp:190-318).
#include "cgli_dev.cuh"
#include "cgli_launch.h"

namespace cgli {

namespace {

constexpr int RELAX_TK = 30;     // interior columns per warp (lanes 1..30)

// split Jacobian of one cell in one direction applied to the cell's own
// iterate n: lower (A+ n, the parenthesised LL terms of DPLUSGS.cpp:728-787)
// and upper (A- diagonal / A+ off-diagonal mixture, the UU terms of
// :1004-1063) products; returns the spectral radius used by the diagonal
__device__ __forceinline__ double dir_products(const CPrim<double> &q, double mx, double my, double mz,
                                               const double n[5], double lo[5], double up[5]) {
  const double K = KG, beta = q.beta, U = mx * q.u + my * q.v + mz * q.w;
  const double S = sqrt(U * U * (beta - 1) * (beta - 1) + 4 * beta * q.C * (mx * mx + my * my + mz * mz));
  const double lam = ((beta + 1) * fabs(U) + S) / 2;
  Split<double> s;
  const double pk = 0.5 * q.P * K * beta, hr = 0.5 / q.rho, bt = 0.5 * beta * q.Tt * (K - 1);
  s.p11 = 0.5 * (beta * U + lam);
  s.p12 = pk * mx; s.p13 = pk * my; s.p14 = pk * mz;
  s.p21 = mx * hr; s.p31 = my * hr; s.p41 = mz * hr;
  s.p22 = 0.5 * (U + lam);
  s.p51 = 0.5 * U * (K - 1) * (beta - 1) / q.rho / K;
  s.p52 = bt * mx; s.p53 = bt * my; s.p54 = bt * mz;
  s.m11 = 0.5 * (beta * U - lam);
  s.m22 = 0.5 * (U - lam);
  lower_terms<double>(s, n, lo);
  upper_terms<double>(s, n, up);
  return lam;
}

}  // namespace

struct RelaxPtrs {
  const double *src[5];
  double *dst[5];
};

// One Jacobi relaxation, DPLUSGS.cpp:488-1141: dst = D^-1 (MR - LL(src) -
// UU(src)) on planes [ilo, ihi] of this CTA's chunk; src on planes 2 and
// ie+1 is read at its periodic images ie and 3 (the self-copy exchange of
// :510-531).  The diagonal is that of DPLUSGS.cpp:1068-1107 (inviscid).
template <int TJ>
__global__ void __launch_bounds__((TJ + 2) * 32, TJ <= 6 ? 2 : 1) k_dplur_relax(Dev d, RelaxPtrs a, int chunk) {
  extern __shared__ double ysm[];   // [2 buffers][TJ+2 rows][10 values][32 lanes]
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int j = 1 + blockIdx.y * TJ + w;
  const int k = 1 + blockIdx.x * RELAX_TK + lane;
  const int ie = d.nx + 2, jn = d.ny + 1, kn = d.nz + 1;
  const int ilo = 3 + blockIdx.z * chunk;
  const int ihi = min(ie, ilo + chunk - 1);
  const bool active = j >= 2 && j <= jn && k >= 2 && k <= kn;
  const bool row = w >= 1 && w <= TJ;                       // an interior row of the tile
  const bool out = active && row && lane >= 1 && lane <= RELAX_TK;
  const double idx = 1.0 / d.dxi, idy = 1.0 / d.det, idz = 1.0 / d.dzt;
  const double dt = d.dt;
  double lxp[5] = {0, 0, 0, 0, 0};   // lower x product of plane p-1
  double part[5] = {0, 0, 0, 0, 0};  // MR - LL - UU(y, z) of plane p-1
  double d11 = 0, d22 = 0, d51 = 0;  // diagonal of plane p-1
  for (int p = ilo - 1; p <= ihi + 1; p++) {
    const bool edge = p < ilo || p > ihi;     // only the x products are needed
    double lx[5] = {0, 0, 0, 0, 0}, ux[5] = {0, 0, 0, 0, 0};
    double ly[5] = {0, 0, 0, 0, 0}, uy[5] = {0, 0, 0, 0, 0};
    double lz[5] = {0, 0, 0, 0, 0}, uz[5] = {0, 0, 0, 0, 0};
    double mr[5] = {0, 0, 0, 0, 0};
    double lam = 0, beta = 0, rho = 0;
    if (active && (row || !edge)) {
      const long long c = ix(d, p, j, k);
      const int pn = p == 2 ? ie : (p == ie + 1 ? 3 : p);
      const long long cn = ix(d, pn, j, k);
      const CPrim<double> q =
          cprim<double>(d.U_[0][c], d.U_[1][c], d.U_[2][c], d.U_[3][c], d.U_[4][c], d.J[c], d.e);
      double n[5];
#pragma unroll
      for (int v = 0; v < 5; v++) n[v] = a.src[v][cn];
      beta = q.beta; rho = q.rho;
      if (row) {
        double lamx = dir_products(q, d.m[0][c], d.m[1][c], d.m[2][c], n, lx, ux);
        lam = lamx * idx;
      }
      if (!edge) {
        double lamy = dir_products(q, d.m[3][c], d.m[4][c], d.m[5][c], n, ly, uy);
        lam += lamy * idy;
        if (row) {
          double lamz = dir_products(q, d.m[6][c], d.m[7][c], d.m[8][c], n, lz, uz);
          lam += lamz * idz;
        }
        if (out) {
#pragma unroll
          for (int v = 0; v < 5; v++) mr[v] = d.MR[v][c];
        }
      }
    }
    // finish plane p-1 with the upper x product of plane p
    if (out && p - 1 >= ilo) {
      const long long c = ix(d, p - 1, j, k);
      double r[5];
#pragma unroll
      for (int v = 0; v < 5; v++) r[v] = part[v] - ux[v] * idx;
      a.dst[0][c] = d11 * r[0];
      a.dst[1][c] = d22 * r[1];
      a.dst[2][c] = d22 * r[2];
      a.dst[3][c] = d22 * r[3];
      a.dst[4][c] = d51 * r[0] + d22 * r[4];
    }
    if (edge) {
#pragma unroll
      for (int v = 0; v < 5; v++) lxp[v] = lx[v];
      continue;   // p is the same for every thread of the CTA
    }
    // k neighbours by shuffles: lower product of k-1, upper product of k+1
    double lzm[5], uzp[5];
#pragma unroll
    for (int v = 0; v < 5; v++) {
      lzm[v] = __shfl_up_sync(0xffffffffu, lz[v], 1);
      uzp[v] = __shfl_down_sync(0xffffffffu, uz[v], 1);
    }
    // j neighbours through shared memory
    double *buf = ysm + (size_t)(p & 1) * (TJ + 2) * 10 * 32;
#pragma unroll
    for (int v = 0; v < 5; v++) {
      buf[(w * 10 + v) * 32 + lane] = ly[v];
      buf[(w * 10 + 5 + v) * 32 + lane] = uy[v];
    }
    __syncthreads();
    if (out) {
      double lym[5], uyp[5];
#pragma unroll
      for (int v = 0; v < 5; v++) {
        lym[v] = buf[((w - 1) * 10 + v) * 32 + lane];
        uyp[v] = buf[((w + 1) * 10 + 5 + v) * 32 + lane];
      }
#pragma unroll
      for (int v = 0; v < 5; v++) {
        const double LL = lxp[v] * idx + lym[v] * idy + lzm[v] * idz;
        const double UUyz = uyp[v] * idy + uzp[v] * idz;
        part[v] = mr[v] - LL - UUyz;
      }
      // DPLUSGS.cpp:1091-1107
      const double t3 = 3 + 2 * lam * dt, t3b = 3 * beta + 2 * lam * dt;
      d11 = 2 * dt / t3b;
      d22 = 2 * dt / t3;
      d51 = -(6 * (KG - 1) * (beta - 1) * dt) / (KG * t3 * t3b * rho);
    }
#pragma unroll
    for (int v = 0; v < 5; v++) lxp[v] = lx[v];
  }
}

// Update of DPLUSGS.cpp:1152-1196 from the last relaxation's result, with
// per-block partial sums of the squared squared increments (:1203-1215);
// one block per (j, i) row of k
__global__ void k_dplur_update(Dev d, RelaxPtrs a) {
  int k = 2 + threadIdx.x;
  int j = 2 + blockIdx.x;
  int i = 3 + blockIdx.y;
  const double *const *nr = a.src;
  double acc[5] = {0, 0, 0, 0, 0};
  for (int kk = k; kk <= d.nz + 1; kk += blockDim.x) {
    long long c = ix(d, i, j, kk);
    const double J = d.J[c];
    double q1 = d.U_[0][c];
    double rhoold = q1 * J;
    double Uold = d.U_[1][c] / q1, Vold = d.U_[2][c] / q1, Wold = d.U_[3][c] / q1;
    double VVold = Uold * Uold + Vold * Vold + Wold * Wold;
    double Pold = (d.U_[4][c] * J - 0.5 * rhoold * VVold) * (KG - 1);
    double Told = Pold / rhoold;
    double P = Pold + nr[0][c] * J;
    double U = Uold + nr[1][c] * J;
    double V = Vold + nr[2][c] * J;
    double W = Wold + nr[3][c] * J;
    double T = Told + nr[4][c] * J;
    double rho = P / T;
    d.U_[0][c] = rho / J;
    d.U_[1][c] = rho * U / J;
    d.U_[2][c] = rho * V / J;
    d.U_[3][c] = rho * W / J;
    d.U_[4][c] = (P / (KG - 1) + 0.5 * rho * (U * U + V * V + W * W)) / J;
    double r[5] = {(P - Pold) * (P - Pold), (U - Uold) * (U - Uold), (V - Vold) * (V - Vold),
                   (W - Wold) * (W - Wold), (T - Told) * (T - Told)};
#pragma unroll
    for (int v = 0; v < 5; v++) acc[v] += r[v] * r[v];
  }
  block_sum5(acc, d.partial + 5 * ((long long)blockIdx.y * gridDim.x + blockIdx.x));
}

namespace {

template <int TJ>
void relax(const Dev &d, const RelaxPtrs &a, cudaStream_t s, int chunk) {
  const size_t smem = sizeof(double) * 2 * (TJ + 2) * 10 * 32;
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(k_dplur_relax<TJ>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  dim3 g((d.nz + RELAX_TK - 1) / RELAX_TK, (d.ny + TJ - 1) / TJ, (d.nx + chunk - 1) / chunk);
  k_dplur_relax<TJ><<<g, (TJ + 2) * 32, smem, s>>>(d, a, chunk);
}

RelaxPtrs ptrs(double *const *src, double *const *dst) {
  RelaxPtrs a;
  for (int v = 0; v < 5; v++) { a.src[v] = src[v]; a.dst[v] = dst[v]; }
  return a;
}

}  // namespace

int dplur_tile_rows = 6;   // TJ of the relaxation tiles (6 or 14)
int dplur_chunk = 32;      // x planes per CTA

void launch_dplur_relax(const Dev &d, cudaStream_t s, bool from_nr) {
  RelaxPtrs a = from_nr ? ptrs(d.NR, d.NL) : ptrs(d.NL, d.NR);
  if (dplur_tile_rows == 14) relax<14>(d, a, s, dplur_chunk);
  else relax<6>(d, a, s, dplur_chunk);
}

// residual (NL = NR = D^-1 MR), four relaxations NR->NL->NR->NL->NR, update
void launch_dplur(const Dev &d, cudaStream_t s) {
  launch_dts_residual(d, s);
  for (int sweep = 0; sweep < 4; sweep++) launch_dplur_relax(d, s, sweep % 2 == 0);
  RelaxPtrs a = ptrs(d.NR, d.NL);
  k_dplur_update<<<dim3(d.ny, d.nx), 128, 0, s>>>(d, a);
}

void launch_dplur_iteration(const Dev &d, cudaStream_t s) {
  launch_halo_bc(d, s);
  launch_flux_x(d, s);
  launch_flux_y(d, s);
  launch_flux_z(d, s);
  launch_viscous(d, s);
  launch_dplur(d, s);
}

}  // namespace cgli
