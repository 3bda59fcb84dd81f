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

}  // namespace

struct RelaxPtrs {
  const double *src[5];
  double *dst[5];
  const double *Jtab, *etdytab;   // per-j J and etdy of a grid uniform in x and z
};

__device__ __forceinline__ void cp_async8(double *dst, const double *src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

template <int TJ, bool CH>
constexpr size_t relax_smem() {
  return sizeof(double) * (2 * (TJ + 2) * 10 * 32 + 2 * (CH ? 15 : 25) * (TJ + 2) * 32);
}

// One Jacobi relaxation, DPLUSGS.cpp:488-1141: dst = D^-1 (MR - LL(src) -
// UU(src)) on planes [ilo, ihi] of this CTA's chunk; src on planes 2 and
// ie+1 is read at its periodic images ie and 3 (the self-copy exchange of
// :510-531).  The diagonal is that of DPLUSGS.cpp:1068-1107 (inviscid).
// Each thread copies its cell's inputs of the next plane into shared memory
// with cp.async while it computes the current plane.  CH: the metrics are
// those of a grid uniform in x and z, read per row from Jtab / etdytab.
template <int TJ, bool CH>
__global__ void __launch_bounds__((TJ + 2) * 32, TJ <= 6 ? 2 : 1) k_dplur_relax(Dev d, RelaxPtrs a, int chunk) {
  constexpr int NT = (TJ + 2) * 32;
  constexpr int NV = CH ? 15 : 25;          // staged doubles per cell: U_, src, MR (+ J, 9 metrics)
  extern __shared__ double sm[];
  double *const ysm = sm;                   // [2 buffers][TJ+2 rows][10 values][32 lanes]
  double *const stg = sm + 2 * (TJ + 2) * 10 * 32;   // [2 stages][NV][NT]
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
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
  double Jc = 0, etc = 0;
  if (CH && active) { Jc = a.Jtab[j]; etc = a.etdytab[j]; }

  auto issue = [&](int p) {
    const bool edge = p < ilo || p > ihi;
    if (!active || (!row && edge)) return;
    const long long c = ix(d, p, j, k);
    const int pn = p == 2 ? ie : (p == ie + 1 ? 3 : p);
    const long long cn = ix(d, pn, j, k);
    double *s = stg + (size_t)(p & 1) * NV * NT + tid;
#pragma unroll
    for (int v = 0; v < 5; v++) cp_async8(s + v * NT, d.U_[v] + c);
#pragma unroll
    for (int v = 0; v < 5; v++) cp_async8(s + (5 + v) * NT, a.src[v] + cn);
    if (out && !edge) {
#pragma unroll
      for (int v = 0; v < 5; v++) cp_async8(s + (10 + v) * NT, d.MR[v] + c);
    }
    if (!CH) {
      cp_async8(s + 15 * NT, d.J + c);
#pragma unroll
      for (int v = 0; v < 9; v++) cp_async8(s + (16 + v) * NT, d.m[v] + c);
    }
  };

  double lxp[5] = {0, 0, 0, 0, 0};   // lower x product of plane p-1
  double part[5] = {0, 0, 0, 0, 0};  // MR - LL - UU(y, z) of plane p-1
  double d11 = 0, d22 = 0, d51 = 0;  // diagonal of plane p-1
  issue(ilo - 1);
  cp_async_commit();
  for (int p = ilo - 1; p <= ihi + 1; p++) {
    if (p + 1 <= ihi + 1) issue(p + 1);
    cp_async_commit();
    cp_async_wait1();                        // this thread's copies of plane p have landed
    const bool edge = p < ilo || p > ihi;    // only the x products are needed
    double lx[5] = {0, 0, 0, 0, 0}, ux[5] = {0, 0, 0, 0, 0};
    double ly[5] = {0, 0, 0, 0, 0}, uy[5] = {0, 0, 0, 0, 0};
    double lz[5] = {0, 0, 0, 0, 0}, uz[5] = {0, 0, 0, 0, 0};
    double mr[5] = {0, 0, 0, 0, 0};
    double c11 = 0, c22 = 0, c51 = 0;      // diagonal of plane p
    if (active && (row || !edge)) {
      const double *s = stg + (size_t)(p & 1) * NV * NT + tid;
      double mm[9], J;
      if (CH) {
        J = Jc;
        mm[0] = 1; mm[1] = 0; mm[2] = 0; mm[3] = 0; mm[4] = etc; mm[5] = 0; mm[6] = 0; mm[7] = 0; mm[8] = 1;
      } else {
        J = s[15 * NT];
#pragma unroll
        for (int v = 0; v < 9; v++) mm[v] = s[(16 + v) * NT];
      }
      double n[5];
      // an open slab's end planes hold zero iterates (DPLUSGS.cpp:191-233)
      const bool zero_end = d.x_open && (p == 2 || p == ie + 1);
#pragma unroll
      for (int v = 0; v < 5; v++) n[v] = zero_end ? 0.0 : s[(5 + v) * NT];
      if (row) {
        // the cell's three split Jacobians and its diagonal, each repeated
        // divisor as one reciprocal
        SweepCoef<double> sc;
        sweep_coef<double>(s[0], s[NT], s[2 * NT], s[3 * NT], s[4 * NT], J, mm, d.e, idx, idy, idz, dt, sc);
        lower_terms<double>(sc.A[0], n, lx);
        upper_terms<double>(sc.A[0], n, ux);
        if (!edge) {
          lower_terms<double>(sc.A[1], n, ly);
          upper_terms<double>(sc.A[1], n, uy);
          lower_terms<double>(sc.A[2], n, lz);
          upper_terms<double>(sc.A[2], n, uz);
          c11 = sc.d11; c22 = sc.d22; c51 = sc.d51;
        }
      } else {
        // a halo row: only its y products are used
        const double rq1 = 1 / s[0], rho = s[0] * J;
        const double u = s[NT] * rq1, v = s[2 * NT] * rq1, w = s[3 * NT] * rq1;
        const double VV = u * u + v * v + w * w;
        const double P = (s[4 * NT] * J - 0.5 * rho * VV) * (KG - 1);
        const double rrho = 1 / rho, C = KG * P * rrho, Tt = P * rrho, th = VV / C;
        const double beta = th > d.e ? th : d.e;
        double lam;
        const Split<double> sy = split_fast<double>(beta, C, P, Tt, rrho, u, v, w, mm[3], mm[4], mm[5], false, lam);
        lower_terms<double>(sy, n, ly);
        upper_terms<double>(sy, n, uy);
      }
      if (out && !edge) {
#pragma unroll
        for (int v = 0; v < 5; v++) mr[v] = s[(10 + v) * NT];
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
#pragma unroll
      for (int v = 0; v < 5; v++) {
        const double lym = buf[((w - 1) * 10 + v) * 32 + lane];
        const double uyp = buf[((w + 1) * 10 + 5 + v) * 32 + lane];
        const double LL = lxp[v] * idx + lym * idy + lzm[v] * idz;
        const double UUyz = uyp * idy + uzp[v] * idz;
        part[v] = mr[v] - LL - UUyz;
      }
      d11 = c11; d22 = c22; d51 = c51;   // DPLUSGS.cpp:1091-1107
    }
#pragma unroll
    for (int v = 0; v < 5; v++) lxp[v] = lx[v];
  }
}

// Residual of DPLUSGS.cpp:324-478 (the same values as Dual_time_stepping.cpp:
// 737-908 without its zero sponge terms): MR and the first iterate
// NL = D^-1 MR on the interior cells, with each repeated divisor as one
// reciprocal.  CH as for the relaxation.
template <bool CH>
__global__ void __launch_bounds__(128) k_dplur_residual(Dev d, RelaxPtrs a) {
  int k = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  int j = 2 + blockIdx.y;
  int i = 3 + blockIdx.z;
  if (k > d.nz + 1) return;
  const long long c = ix(d, i, j, k);
  double mm[9], J;
  if (CH) {
    J = a.Jtab[j];
    mm[0] = 1; mm[1] = 0; mm[2] = 0; mm[3] = 0; mm[4] = a.etdytab[j]; mm[5] = 0; mm[6] = 0; mm[7] = 0; mm[8] = 1;
  } else {
    J = d.J[c];
#pragma unroll
    for (int v = 0; v < 9; v++) mm[v] = d.m[v][c];
  }
  const CPrim<double> q = cprim<double>(d.U_[0][c], d.U_[1][c], d.U_[2][c], d.U_[3][c], d.U_[4][c], J, d.e);
  const double rho = q.rho, u = q.u, v = q.v, w = q.w, VV = q.VV, T = q.Tt, H = q.H, beta = q.beta;
  const double irho = 1 / rho, itemp = 1 / (rho * KG);
  const double d11 = -(H * (KG - 1) + VV - KG * (T + VV)) * beta;
  const double d12 = -(KG - 1) * u * beta, d13 = -(KG - 1) * v * beta, d14 = -(KG - 1) * w * beta;
  const double d15 = (KG - 1) * beta;
  const double d51 = (KG - 1) * (VV + KG * T * beta + (KG - 1) * VV * beta + H * (-1 + beta - KG * beta)) * itemp;
  const double g5 = -(KG - 1) * (1 + (KG - 1) * beta) * itemp;
  const long long fx1 = ix(d, i, j - 1, k - 1), f0 = ix(d, i - 1, j - 1, k - 1);
  const long long fy1 = ix(d, i - 1, j, k - 1), fz1 = ix(d, i - 1, j - 1, k);
  const double i2dt = 1 / (2 * d.dt), idx = 1 / d.dxi, idy = 1 / d.det, idz = 1 / d.dzt, iJ = 1 / J;
  const double f = d.scal[0];
  double Rk[5];
#pragma unroll
  for (int n = 0; n < 5; n++) {
    const double Rp = -(3 * d.U_[n][c] - 4 * d.U[n][c] + d.Uq[n][c]) * i2dt;
    const double Rf = -((d.inF[0][n][fx1] - d.inF[0][n][f0]) * idx + (d.inF[1][n][fy1] - d.inF[1][n][f0]) * idy +
                        (d.inF[2][n][fz1] - d.inF[2][n][f0]) * idz);
    Rk[n] = Rp + Rf;
  }
  Rk[1] = Rk[1] + d.vF[0][c] + f * iJ;
  Rk[2] = Rk[2] + d.vF[1][c];
  Rk[3] = Rk[3] + d.vF[2][c];
  Rk[4] = Rk[4] + d.vF[3][c] + f * u * iJ;
  double MR[5];
  MR[0] = d11 * Rk[0] + d12 * Rk[1] + d13 * Rk[2] + d14 * Rk[3] + d15 * Rk[4];
  MR[1] = (Rk[1] - u * Rk[0]) * irho;
  MR[2] = (Rk[2] - v * Rk[0]) * irho;
  MR[3] = (Rk[3] - w * Rk[0]) * irho;
  MR[4] = d51 * Rk[0] + g5 * (u * Rk[1] + v * Rk[2] + w * Rk[3] - Rk[4]);
  const Diag<double> dg = diag<double>(q, mm, d.dxi, d.det, d.dzt, d.dt);
#pragma unroll
  for (int n = 0; n < 5; n++) d.MR[n][c] = MR[n];
  a.dst[0][c] = dg.d11 * MR[0];
  a.dst[1][c] = dg.d22 * MR[1];
  a.dst[2][c] = dg.d22 * MR[2];
  a.dst[3][c] = dg.d22 * MR[3];
  a.dst[4][c] = dg.d51 * MR[0] + dg.d22 * MR[4];
}

// Update of DPLUSGS.cpp:1152-1196 from the last relaxation's result, with
// per-block partial sums of the squared squared increments (:1203-1215);
// one block per (j, i) row of k
__global__ void __launch_bounds__(128, 8) k_dplur_update(Dev d, RelaxPtrs a) {
  int k = 2 + threadIdx.x;
  int j = 2 + blockIdx.x;
  int i = 3 + blockIdx.y;
  const double *const *nr = a.src;
  double acc[5] = {0, 0, 0, 0, 0};
  for (int kk = k; kk <= d.nz + 1; kk += blockDim.x) {
    long long c = ix(d, i, j, kk);
    // the divisions by q1, rho, T and J as reciprocals (1/J from the table)
    const double J = d.J[c], iJ = d.iJ[c];
    double q1 = d.U_[0][c], iq1 = 1 / q1;
    double rhoold = q1 * J;
    double Uold = d.U_[1][c] * iq1, Vold = d.U_[2][c] * iq1, Wold = d.U_[3][c] * iq1;
    double VVold = Uold * Uold + Vold * Vold + Wold * Wold;
    double Pold = (d.U_[4][c] * J - 0.5 * rhoold * VVold) * (KG - 1);
    double Told = Pold / rhoold;
    double P = Pold + nr[0][c] * J;
    double U = Uold + nr[1][c] * J;
    double V = Vold + nr[2][c] * J;
    double W = Wold + nr[3][c] * J;
    double T = Told + nr[4][c] * J;
    double rho = P / T, rJ = rho * iJ;
    d.U_[0][c] = rJ;
    d.U_[1][c] = rJ * U;
    d.U_[2][c] = rJ * V;
    d.U_[3][c] = rJ * W;
    d.U_[4][c] = (P * (1 / (KG - 1)) + 0.5 * rho * (U * U + V * V + W * W)) * iJ;
    double r[5] = {(P - Pold) * (P - Pold), (U - Uold) * (U - Uold), (V - Vold) * (V - Vold),
                   (W - Wold) * (W - Wold), (T - Told) * (T - Told)};
#pragma unroll
    for (int v = 0; v < 5; v++) acc[v] += r[v] * r[v];
  }
  block_sum5(acc, d.partial + 5 * ((long long)blockIdx.y * gridDim.x + blockIdx.x));
}

namespace {

template <int TJ, bool CH>
void relax(const Dev &d, const RelaxPtrs &a, cudaStream_t s, int chunk) {
  constexpr size_t smem = relax_smem<TJ, CH>();
  if (smem > 48 * 1024)
    cudaFuncSetAttribute(k_dplur_relax<TJ, CH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  dim3 g((d.nz + RELAX_TK - 1) / RELAX_TK, (d.ny + TJ - 1) / TJ, (d.nx + chunk - 1) / chunk);
  k_dplur_relax<TJ, CH><<<g, (TJ + 2) * 32, smem, s>>>(d, a, chunk);
}

RelaxPtrs ptrs(double *const *src, double *const *dst, const SweepArgs &sw) {
  RelaxPtrs a;
  for (int v = 0; v < 5; v++) { a.src[v] = src[v]; a.dst[v] = dst[v]; }
  a.Jtab = sw.Jtab;
  a.etdytab = sw.etdytab;
  return a;
}

}  // namespace

// relaxation tiles of 6 j rows marching over 32 x planes, the shape chosen
// by measurement at 256x192x192 (14 rows and other plane counts)
constexpr int kDplurChunk = 32;

void launch_dplur_relax(const Dev &d, const SweepArgs &sw, cudaStream_t s, bool from_nr) {
  RelaxPtrs a = from_nr ? ptrs(d.NR, d.NL, sw) : ptrs(d.NL, d.NR, sw);
  if (sw.channel_metrics) relax<6, true>(d, a, s, kDplurChunk);
  else relax<6, false>(d, a, s, kDplurChunk);
}

// residual (MR, NR = D^-1 MR), four relaxations NR->NL->NR->NL->NR, update
void launch_dplur(const Dev &d, const SweepArgs &sw, cudaStream_t s) {
  RelaxPtrs r = ptrs(d.NL, d.NR, sw);
  dim3 g((d.nz + 127) / 128, d.ny, d.nx);
  if (sw.channel_metrics) k_dplur_residual<true><<<g, 128, 0, s>>>(d, r);
  else k_dplur_residual<false><<<g, 128, 0, s>>>(d, r);
  for (int sweep = 0; sweep < 4; sweep++) launch_dplur_relax(d, sw, s, sweep % 2 == 0);
  RelaxPtrs a = ptrs(d.NR, d.NL, sw);
  k_dplur_update<<<dim3(d.ny, d.nx), 128, 0, s>>>(d, a);
}

void launch_dplur_iteration(const Dev &d, const SweepArgs &sw, cudaStream_t s) {
  launch_halo_bc(d, s);
  launch_flux_x(d, s);
  launch_flux_y(d, s);
  launch_flux_z(d, s);
  launch_viscous(d, s);
  launch_dplur(d, sw, s);
}

}  // namespace cgli
