// Fast path of one inner iteration: halo and boundaries, fluxes, viscous
// terms, residual assembly, four wavefront sweep passes with the update
// fused into the last one.
#include <type_traits>

#include "cgli_dev.cuh"
#include "cgli_launch.h"

// CTAs per SM the residual kernel is compiled for (register cap)
#ifndef CGLI_RESIDUAL_MINBLOCKS
#define CGLI_RESIDUAL_MINBLOCKS 1
#endif

namespace cgli {

// the nine metric terms of cell c (row j): per-row tables on the channel grid
template <bool CH>
__device__ __forceinline__ void cell_metrics(const Dev &d, const SweepArgs &a, int j, long long c, double mm[9]) {
  if (CH) {
    mm[0] = 1; mm[1] = 0; mm[2] = 0; mm[3] = 0; mm[4] = a.etdytab[j]; mm[5] = 0; mm[6] = 0; mm[7] = 0; mm[8] = 1;
  } else {
#pragma unroll
    for (int v2 = 0; v2 < 9; v2++) mm[v2] = d.m[v2][c];
  }
}

// Dual_time_stepping.cpp:737-922 for the fast path: MR of every interior
// cell, and D^-1 MR on planes ie and 3 as the lagged halos of the first sweep
// (the reference initialises NL = NR = D^-1 MR, :897-908, and the sweep
// exchanges planes ie and 3 before its first pass, :942-976).  CH: the grid
// is uniform in x and z (a.channel_metrics), J and etdy come from the per-row
// tables instead of ten 3-D metric arrays.
// (the mixed-precision channel instance is held at six CTAs per SM, the
// occupancy of the other instances: uncapped it takes ten registers more and
// drops to five)
template <bool MIXED, bool CH>
__global__ void __launch_bounds__(64, (MIXED && CH && CGLI_RESIDUAL_MINBLOCKS < 6) ? 6 : CGLI_RESIDUAL_MINBLOCKS)
    k_residual_fast(Dev d, SweepArgs a) {
  int k = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  int j = 2 + blockIdx.y;
  int i = 2 + blockIdx.z;
  if (k > d.nz + 1) return;
  long long c = ix(d, i, j, k);
  const double J = CH ? a.Jtab[j] : d.J[c], deltaT = d.dt;

  const int ie = d.nx + 2;
  const bool halo_plane = (i == 2 || i == ie + 1);
  const long long slot = halo_plane ? 0 : skew_slot<typename std::conditional<MIXED, float, double>::type>(d, i, j, k);
  double r8, r9, r10;   // record words stored together with MR
  {
    // the cell's sweep record; planes 2 and ie+1 (the periodic halo copies)
    // go to the per-(j,k) halo records
    double mm[9], r[REC_N];
    cell_metrics<CH>(d, a, j, c, mm);
    make_record(d.U_[0][c], d.U_[1][c], d.U_[2][c], d.U_[3][c], d.U_[4][c], J, mm, d.e, d.rdxi, d.rdet, d.rdzt,
                deltaT, r);
    const long long h = (long long)j * d.dj + k;
    if (halo_plane) {
      for (int v2 = 0; v2 < REC_N; v2++) {
        if (MIXED) {
          if (i == 2) a.hrecf_f[v2][h] = (float)r[v2];
          else a.hrecf_b[v2][h] = (float)r[v2];
        } else {
          if (i == 2) a.hrec_f[v2][h] = r[v2];
          else a.hrec_b[v2][h] = r[v2];
        }
      }
      return;
    }
    // the record part of the cell's contiguous block; the vectors that the
    // record's last words share with MR go out with MR below
    // (vectors in the rotated order of rec_vec_pos: t = slot % 8, the
    // slot's position in its step block, whose size is a multiple of 8)
    const int t = (int)(slot & 7);
    if (MIXED) {
      float4 *o = reinterpret_cast<float4 *>(a.cellrecf + slot * CR_N);
      o[rec_vec_pos<float>(0, t)] = make_float4((float)r[0], (float)r[1], (float)r[2], (float)r[3]);
      o[rec_vec_pos<float>(1, t)] = make_float4((float)r[4], (float)r[5], (float)r[6], (float)r[7]);
    } else {
      double2 *o = reinterpret_cast<double2 *>(a.cellrec + slot * CR_N);
#pragma unroll
      for (int q = 0; q < 5; q++) o[rec_vec_pos<double>(q, t)] = make_double2(r[2 * q], r[2 * q + 1]);
    }
    r8 = r[8];
    r9 = r[9];
    r10 = r[10];
  }
  CPrim<double> q = cprim<double>(d.U_[0][c], d.U_[1][c], d.U_[2][c], d.U_[3][c], d.U_[4][c], J, d.e);
  double rho = q.rho, u = q.u, v = q.v, w = q.w, VV = q.VV, T = q.Tt, H = q.H, beta = q.beta;
  // Gamma^-1 of Dual_time_stepping.cpp:771-802; divisions by rho and by
  // rho*gamma as one (Newton-refined) reciprocal and products
  const double irho = nr_rcp(rho), itemp = irho * (1.0 / KG);
  double d11 = -(H * (KG - 1) + VV - KG * (T + VV)) * beta;
  double d12 = -(KG - 1) * u * beta, d13 = -(KG - 1) * v * beta, d14 = -(KG - 1) * w * beta;
  double d15 = (KG - 1) * beta;
  double d21 = -u * irho, d22 = irho;
  double d31 = -v * irho;
  double d41 = -w * irho;
  double d51 = (KG - 1) * (VV + KG * T * beta + (KG - 1) * VV * beta + H * (-1 + beta - KG * beta)) * itemp;
  double d52 = -(KG - 1) * u * (1 + (KG - 1) * beta) * itemp;
  double d53 = -(KG - 1) * v * (1 + (KG - 1) * beta) * itemp;
  double d54 = -(KG - 1) * w * (1 + (KG - 1) * beta) * itemp;
  double d55 = (KG - 1) * (1 + (KG - 1) * beta) * itemp;
  long long fx1 = ix(d, i, j - 1, k - 1), fx0 = ix(d, i - 1, j - 1, k - 1);
  long long fy1 = ix(d, i - 1, j, k - 1), fz1 = ix(d, i - 1, j - 1, k);
  double Rk[5], sp[5];
  sponge_terms(d, i, c, sp);
  double f = d.buoyancy ? -(rho - 1.1842) * 9.81 : d.scal[0];
  const double i2dt = nr_rcp(2 * deltaT), idx = d.rdxi, idy = d.rdet, idz = d.rdzt, iJ = nr_rcp(J);
  for (int n = 0; n < 5; n++) {
    double Rp = -(3 * d.U_[n][c] - 4 * d.U[n][c] + d.Uq[n][c]) * i2dt;
    double Rf = -((d.inF[0][n][fx1] - d.inF[0][n][fx0]) * idx + (d.inF[1][n][fy1] - d.inF[1][n][fx0]) * idy +
                  (d.inF[2][n][fz1] - d.inF[2][n][fx0]) * idz);
    Rk[n] = sp[n] * iJ + Rp + Rf;
  }
  Rk[1] = Rk[1] + d.vF[0][c] + f * iJ;
  Rk[2] = Rk[2] + d.vF[1][c];
  Rk[3] = Rk[3] + d.vF[2][c];
  Rk[4] = Rk[4] + d.vF[3][c] + f * u * iJ;
  double MR[5];
  MR[0] = (d11 * Rk[0] + d12 * Rk[1] + d13 * Rk[2] + d14 * Rk[3] + d15 * Rk[4]);
  MR[1] = (d21 * Rk[0] + d22 * Rk[1]);
  MR[2] = (d31 * Rk[0] + d22 * Rk[2]);
  MR[3] = (d41 * Rk[0] + d22 * Rk[3]);
  MR[4] = (d51 * Rk[0] + d52 * Rk[1] + d53 * Rk[2] + d54 * Rk[3] + d55 * Rk[4]);
  // MR after the record in the cell's contiguous block of CR_N = 16 words
  // (record words 0..10, MR 11..15)
  const int t = (int)(slot & 7);
  if (MIXED) {
    float4 *o = reinterpret_cast<float4 *>(a.cellrecf + slot * CR_N);
    o[rec_vec_pos<float>(2, t)] = make_float4((float)r8, (float)r9, (float)r10, (float)MR[0]);
    o[rec_vec_pos<float>(3, t)] = make_float4((float)MR[1], (float)MR[2], (float)MR[3], (float)MR[4]);
  } else {
    double2 *o = reinterpret_cast<double2 *>(a.cellrec + slot * CR_N);
    (void)r8;
    (void)r9;
    o[rec_vec_pos<double>(5, t)] = make_double2(r10, MR[0]);
    o[rec_vec_pos<double>(6, t)] = make_double2(MR[1], MR[2]);
    o[rec_vec_pos<double>(7, t)] = make_double2(MR[3], MR[4]);
  }
  // the lagged halos of the first sweep; an open slab's stay zero
  if (!d.x_open && (i == ie || i == 3)) {
    double mm[9];
    cell_metrics<CH>(d, a, j, c, mm);
    Diag<double> dd = diag<double>(q, mm, d.dxi, d.det, d.dzt, deltaT);
    double n5[5] = {dd.d11 * MR[0], dd.d22 * MR[1], dd.d22 * MR[2], dd.d22 * MR[3], dd.d51 * MR[0] + dd.d22 * MR[4]};
    long long h = (long long)j * d.dj + k;
    for (int n = 0; n < 5; n++) {
      if (MIXED) {
        if (i == ie) a.halo_ff[n][h] = (float)n5[n];
        if (i == 3) a.halo_bf[n][h] = (float)n5[n];
      } else {
        if (i == ie) a.halo_f[n][h] = n5[n];
        if (i == 3) a.halo_b[n][h] = n5[n];
      }
    }
  }
}

void launch_residual_fast(const Dev &d, const SweepArgs &a, cudaStream_t s, bool mixed) {
  dim3 g((d.nz + 63) / 64, d.ny, d.nx + 2);
  if (a.channel_metrics) {
    if (mixed) k_residual_fast<true, true><<<g, 64, 0, s>>>(d, a);
    else k_residual_fast<false, true><<<g, 64, 0, s>>>(d, a);
  } else {
    if (mixed) k_residual_fast<true, false><<<g, 64, 0, s>>>(d, a);
    else k_residual_fast<false, false><<<g, 64, 0, s>>>(d, a);
  }
}

void launch_fused_residual(const Dev &d, const SweepArgs &a, cudaStream_t s, int precision) {
  launch_halo_bc(d, s);
  launch_flux_x(d, s);
  launch_flux_y(d, s);
  launch_flux_z(d, s);
  launch_viscous(d, s);
  launch_target_u(d, s);
  launch_residual_fast(d, a, s, precision == 1);
}

}  // namespace cgli
