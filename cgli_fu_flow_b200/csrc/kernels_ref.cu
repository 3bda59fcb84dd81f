// Reference-granularity kernels: one kernel (or a short sequence) per
// reference routine, reading and writing the same arrays in the same layout
// as the reference, so every entry point of include/cgli_fu_flow.h can be
// checked against its counterpart on its own.  The fused fast path of
// cgli_inner_iteration lives in kernels_fused.cu.
#include "cgli_dev.cuh"
#include "cgli_launch.h"
#include "viscous_face.cuh"

// CTAs of 64 threads per SM the inviscid flux and the viscous face kernels
// are compiled for (register caps: 12 CTAs leave the fluxes 80 registers, a
// few spilled, 18 % faster than the uncapped 116 at 256x192x192; 8 CTAs
// leave the viscous faces 128, 3 % faster than 154, 10 CTAs are slower)
#ifndef CGLI_FLUX_MINBLOCKS
#define CGLI_FLUX_MINBLOCKS 12
#endif
#ifndef CGLI_VISCOUS_MINBLOCKS
#define CGLI_VISCOUS_MINBLOCKS 8
#endif

namespace cgli {

// ---------------------------------------------------------------- halos
// main.cpp:167-200: U_[ie+1..ie+3] <- U_[3..5], U_[0..2] <- U_[ie-2..ie]
__global__ void k_halo_x(Dev d) {
  long long plane = d.di;
  long long n = 3 * plane;
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n) return;
  int v = blockIdx.y;
  int ie = d.nx + 2;
  double *q = d.U_[v];
  q[(long long)(ie + 1) * plane + t] = q[3 * plane + t];
  q[t] = q[(long long)(ie - 2) * plane + t];
}

// Y_boundary_condition.cpp:94-182 for interior planes i = 3..ie: the
// zero-gradient copy of :100-112, replaced inside the heated section
// (planes nx_inlet+3 .. Nx-nx_outlet+2, :114) by the isothermal no-slip
// reflection
__global__ void k_bc_y(Dev d) {
  int k = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  int i = 3 + blockIdx.y;
  int side = blockIdx.z;
  int jn = d.ny + 1, kn = d.nz + 1;
  if (k > kn) return;
  int js = side ? jn : 2, jg = side ? jn + 1 : 1;
  long long c = ix(d, i, js, k), g = ix(d, i, jg, k);
  if (!(i > d.nx_inlet + 2 && i < d.nx - d.nx_outlet + 3)) {
    for (int v = 0; v < 5; v++) d.U_[v][g] = d.U_[v][c];
    return;
  }
  double q1 = d.U_[0][c], q2 = d.U_[1][c], q3 = d.U_[2][c], q4 = d.U_[3][c], q5 = d.U_[4][c];
  double Jc = d.J[c], Jg = d.J[g];
  double rho = q1 * Jc;
  double U = q2 / q1, V = q3 / q1, W = q4 / q1;
  double VV = U * U + V * V + W * W;
  double P = (q5 * Jc - 0.5 * rho * VV) * (KG - 1);
  double T = side ? d.twh : d.twl;
  rho = P / RG / T;
  d.U_[0][g] = rho / Jg;
  d.U_[1][g] = -rho * U / Jg;
  d.U_[2][g] = -rho * V / Jg;
  d.U_[3][g] = -rho * W / Jg;
  d.U_[4][g] = (P / (KG - 1) + 0.5 * rho * VV) / Jg;
}

// Z_boundary_condition.cpp:39-66: all rows 0..nyyy of planes 0..ie+3
// (planes 2..ie+1 on an open slab, :40-44)
__global__ void k_bc_z(Dev d) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  long long n = (long long)d.X * d.Y;
  if (t >= n) return;
  if (d.x_open) {
    const int i = (int)(t / d.Y);
    if (i < 2 || i > d.nx + 3) return;
  }
  int v = blockIdx.y;
  long long row = t * d.dj;
  int kn = d.nz + 1;
  double *q = d.U_[v];
  q[row + 1] = q[row + kn];
  q[row + kn + 1] = q[row + 2];
}

// X_boundary_condition.cpp:73-338 on an open slab: one pseudo-time step of
// dtau = dt/200 on the ghost cell of each interior row, with
// M (Gamma + 3 dtau/(2 dt) M)^-1 applied to the characteristic amplitudes
// (the outgoing ones from one-sided x differences against the interior
// neighbour, the incoming ones zero) plus the BDF2 time derivative.
// blockIdx.z: 0 inlet (plane 2 against 3), 1 outlet (plane ie+1 against ie).
__global__ void k_bc_x(Dev d) {
  const int k = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y;
  const int side = blockIdx.z;
  if (k > d.nz + 1) return;
  const int ie = d.nx + 2;
  const long long c = ix(d, side ? ie : 3, j, k), g = ix(d, side ? ie + 1 : 2, j, k);
  const double K = KG, deltaT = d.dt, deltaTau = deltaT / 200., rdx = 1 / d.dxi;
  double q[5], qi[5];
#pragma unroll
  for (int v = 0; v < 5; v++) { q[v] = d.U_[v][g]; qi[v] = d.U_[v][c]; }
  // interior neighbour
  const double Jc = d.J[c], iq1 = 1 / qi[0];
  const double rho_ = qi[0] * Jc, U_ = qi[1] * iq1, V_ = qi[2] * iq1, W_ = qi[3] * iq1;
  const double P_ = (qi[4] * Jc - 0.5 * rho_ * (U_ * U_ + V_ * V_ + W_ * W_)) * (K - 1);
  const double T_ = P_ / rho_;
  // ghost cell
  const double Jg = d.J[g], ig1 = 1 / q[0];
  const double rho = q[0] * Jg, U = q[1] * ig1, V = q[2] * ig1, W = q[3] * ig1;
  const double VV = U * U + V * V + W * W;
  const double P = (q[4] * Jg - 0.5 * rho * VV) * (K - 1);
  const double C2 = K * P / rho, C = sqrt(C2);
  const double T = P / rho;
  const double H = 0.5 * VV + C * C / (K - 1);
  const double th = VV / C / C, beta = th > d.e ? th : d.e;
  // M (Gamma + 3 dtau/(2 dt) M)^-1, :98-147
  const double itemp = 1 / (K * T * (2 * deltaT + 3 * deltaTau) * (2 * deltaT + 3 * beta * deltaTau));
  const double temp2 = (K - 1) * (beta - 1) * deltaT * deltaT;
  const double temp3 = H - H * K - VV + K * (T + VV);
  const double a4 = -4 * temp2 * itemp, t3 = 4 * temp3 * (beta - 1) * deltaT * deltaT * itemp;
  const double vel[3] = {U, V, W};
  double dm[5][5];
  dm[0][0] = (2 * deltaT * (-2 * (-(K - 1) * (H - VV) - temp3 * beta) * deltaT + 3 * K * T * beta * deltaTau)) * itemp;
  dm[0][4] = -a4;
  dm[4][0] = H * t3;
  dm[4][4] = (2 * deltaT * (2 * H * (K - 1) * (beta - 1) * deltaT + K * T * (2 * deltaT + 3 * beta * deltaTau))) * itemp;
#pragma unroll
  for (int a = 0; a < 3; a++) {
    dm[0][1 + a] = vel[a] * a4;
    dm[1 + a][0] = vel[a] * t3;
    dm[1 + a][4] = -vel[a] * a4;
    dm[4][1 + a] = H * vel[a] * a4;
#pragma unroll
    for (int b = 0; b < 3; b++)
      dm[1 + a][1 + b] = a == b ? (2 * deltaT * (2 * K * (T - vel[a] * vel[a] * (beta - 1)) * deltaT +
                                                 2 * vel[a] * vel[a] * (beta - 1) * deltaT + 3 * K * T * beta * deltaTau)) * itemp
                                : vel[a] * vel[b] * a4;
  }
  const double U_p = 0.5 * (beta + 1) * U;
  const double C_p = 0.5 * sqrt(U * U * (beta - 1) * (beta - 1) + 4 * beta * C * C);
  double L1 = 0, L2 = 0, L3 = 0, L4, L5;
  if (!side) {
    // inlet, :151-187: L5 from the interior, L4 from it, L1..L3 only for backflow
    const double dp = (P_ - P) * rdx, du = (U_ - U) * rdx, dv = (V_ - V) * rdx, dw = (W_ - W) * rdx, dT = (T_ - T) * rdx;
    L5 = (U_p - C_p) * (dp - rho * (U_p + C_p - U) * du);
    L4 = L5 * (U_p - C_p - U) / (U_p + C_p - U);
    if (U <= 0) { L1 = U * (dT + 1.0 / rho * dp * (1 - K) / K); L2 = U * dw; L3 = -U * dv; }
  } else {
    // outlet, :292-327
    const double dp = (P - P_) * rdx, du = (U - U_) * rdx, dv = (V - V_) * rdx, dw = (W - W_) * rdx, dT = (T - T_) * rdx;
    L4 = (U_p + C_p) * (dp - rho * (U_p - C_p - U) * du);
    L5 = L4 * (U_p + C_p - U) / (U_p - C_p - U);
    if (U > 0) { L1 = U * (dT + 1.0 / rho * dp * (1 - K) / K); L2 = U * dw; L3 = -U * dv; }
  }
  double KAL[5];
  KAL[0] = 0.5 / C_p * (L4 * (U_p + C_p - U) - L5 * (U_p - C_p - U));
  KAL[1] = 0.5 / (rho * C_p) * (L4 - L5);
  KAL[2] = -L3;
  KAL[3] = L2;
  KAL[4] = L1 + 1. / rho * (K - 1) / K * KAL[0];
  const double iJg = 1 / Jg, i2dt = 1 / (2 * deltaT);
#pragma unroll
  for (int v = 0; v < 5; v++) KAL[v] = KAL[v] * iJg + (3 * q[v] - 4 * d.U[v][g] + d.Uq[v][g]) * i2dt;
#pragma unroll
  for (int v = 0; v < 5; v++)
    d.U_[v][g] = q[v] - deltaTau * (dm[v][0] * KAL[0] + dm[v][1] * KAL[1] + dm[v][2] * KAL[2] + dm[v][3] * KAL[3] +
                                    dm[v][4] * KAL[4]);
}

// Clears *ok if some face of set `set` in the ranges the face generator
// fills (x: i 2..ie, rows 1..jn-1, k 1..kn-1; y: i 2..ie-1, rows 1..jn,
// k 1..kn-1; z: i 2..ie-1, rows 1..jn-1, k 1..kn) is not of the channel's
// form with the etdy and J of its row's face (2, row, 1)
__global__ void k_check_face_set(Dev d, int set, int i1, int j1, int k1, int *ok) {
  const int k = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y, i = 2 + blockIdx.z;
  if (k > k1 || j > j1 || i > i1) return;
  const long long f = ix(d, i, j, k), r = ix(d, 2, j, 1);
  const double *const *m = d.mf[set];
  const bool good = m[0][f] == 1.0 && m[1][f] == 0.0 && m[2][f] == 0.0 && m[3][f] == 0.0 && m[5][f] == 0.0 &&
                    m[6][f] == 0.0 && m[7][f] == 0.0 && m[8][f] == 1.0 && m[4][f] == m[4][r] &&
                    d.Jf[set][f] == d.Jf[set][r];
  if (!good) atomicExch(ok, 0);
}
__global__ void k_fill_face_tables(Dev d) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= d.Y) return;
  for (int set = 0; set < 3; set++) {
    const long long r = ix(d, 2, j, 1);
    double *t = d.ftab + ((long long)set * d.Y + j) * 4;
    t[0] = d.mf[set][4][r];
    t[1] = d.Jf[set][r];
    t[2] = 1.0 / t[1];
    t[3] = 1.0 / fabs(t[0]);
  }
}

// outlet sponge target velocity, Dual_time_stepping.cpp:510-532: the sum
// over plane 3, rows j = 2..Ny+2, k = 2..Nz+2, of u deltaET / etdy deltaZT,
// over high deltaZT Nz; one block, into d.scal[1]
__global__ void k_target_u(Dev d) {
  const int nj = d.ny + 1, nk = d.nz + 1;
  double acc[5] = {0, 0, 0, 0, 0};
  for (int t = threadIdx.x; t < nj * nk; t += blockDim.x) {
    const int j = 2 + t / nk, k = 2 + t % nk;
    const long long c = ix(d, 3, j, k);
    acc[0] += d.U_[1][c] / d.U_[0][c] * d.det / d.m[4][c] * d.dzt;
  }
  __shared__ double tot[5];
  block_sum5(acc, tot);
  __syncthreads();
  if (threadIdx.x == 0) d.scal[1] = tot[0] * (1. / (d.high * d.dzt * d.nz));
}

// ---------------------------------------------------------------- fluxes
// x faces i = 2..ie, tangential j = 1..jn-1, k = 1..kn-1 (Flux_X.cpp:96-357)
__global__ void __launch_bounds__(64, CGLI_FLUX_MINBLOCKS) k_flux_x(Dev d) {
  int k = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  int j = 1 + blockIdx.y;
  int i = 2 + blockIdx.z;
  if (k > d.nz) return;
  long long f = ix(d, i, j, k);
  // left state ML[i] from cells i-2..i+2, right state MR[i] from i-1..i+3
  long long c = ix(d, i, j + 1, k + 1);
  double L[5], R[5], F[5], fav3, pp;
  const int ie = d.nx + 2;
  const long long di = d.di;
  if (d.x_open && (i <= 3 || i >= ie - 1)) {
    // the first and last rank's reduced stencils, Flux_X.cpp:139-216
    if (i == 2) side2(d, c, c + di, L);
    else if (i == 3 || i == ie) side3L(d, c - di, di, L);
    else side5L(d, c - 2 * di, di, L);
    if (i == 2 || i == ie - 1) side3R(d, c, di, R);
    else if (i == ie) side2(d, c, c + di, R);
    else side5R(d, c - di, di, R);
  } else {
    side5L(d, c - 2 * di, di, L);
    side5R(d, c - di, di, R);
  }
  double mm[9], Jf, iJf, sq, insqr;
  face_metrics(d, 0, f, j, mm, Jf, iJf);
  face_norm(d, 0, j, mm[0], mm[1], mm[2], sq, insqr);
  roe_face(L, R, mm[0], mm[1], mm[2], sq, insqr, iJf, d.e, F, fav3, pp);
  for (int v = 0; v < 5; v++) d.inF[0][v][f] = F[v];
}

// left / right MUSCL states of all five variables at y face j+1/2 of column
// (i,k), with the reduced stencils of Flux_Y.cpp:135-250 (valid for Ny >= 6)
__device__ __forceinline__ void muscl_y(const Dev &d, int i, int j, int k, double L[5], double R[5]) {
  const int jn = d.ny + 1;
  const long long dj = d.dj;
  const long long c = ix(d, i, j, k);
  if (j == 1 || j == 2) side2(d, c, c + dj, L);
  else if (j == 3 || j == jn - 1) side3L(d, c - dj, dj, L);
  else if (j == jn) side2(d, c, c - dj, L);
  else side5L(d, c - 2 * dj, dj, L);
  const long long r = c + dj;  // cell j+1
  if (j == 1) side2(d, r, r + dj, R);
  else if (j == 2 || j == jn - 2) side3R(d, r - dj, dj, R);
  else if (j == jn - 1) side2(d, r, r - dj, R);
  else if (j == jn) side2(d, c, c + dj, R);
  else side5R(d, r - 2 * dj, dj, R);
}

// y faces j = 1..jn, i = 2..ie-1, k = 1..kn-1 (Flux_Y.cpp:94-413)
__global__ void __launch_bounds__(64, CGLI_FLUX_MINBLOCKS) k_flux_y(Dev d) {
  int k = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  int j = 1 + blockIdx.y;
  int i = 2 + blockIdx.z;
  if (k > d.nz) return;
  int jn = d.ny + 1;
  long long f = ix(d, i, j, k);
  double L[5], R[5], F[5], fav3, pp;
  muscl_y(d, i + 1, j, k + 1, L, R);
  double mm[9], Jf, iJf, sq, insqr;
  face_metrics(d, 1, f, j, mm, Jf, iJf);
  const double ety = mm[4];
  face_norm(d, 1, j, mm[3], ety, mm[5], sq, insqr);
  roe_face(L, R, mm[3], ety, mm[5], sq, insqr, iJf, d.e, F, fav3, pp);
  if (j == 1 || j == jn) {
    F[0] = 0; F[1] = 0; F[3] = 0; F[4] = 0;
    F[2] = 0.5 * (ety * pp - 1. * fav3) * iJf;
    if (d.curved_walls) {
      // a curved wall also carries the x and z pressure force
      F[1] = 0.5 * (mm[3] * pp) * iJf;
      F[3] = 0.5 * (mm[5] * pp) * iJf;
    }
  }
  for (int v = 0; v < 5; v++) d.inF[1][v][f] = F[v];
}

// left / right states of all five variables at z face k+1/2
// (Flux_Z.cpp:105-216, valid for Nz >= 4)
__device__ __forceinline__ void muscl_z(const Dev &d, int i, int j, int k, double L[5], double R[5]) {
  const int kn = d.nz + 1;
  const long long c = ix(d, i, j, k);
  if (k == 1) side2(d, c, c + 1, L);
  else if (k == 2 || k == kn) side3L(d, c - 1, 1, L);
  else side5L(d, c - 2, 1, L);
  const long long r = c + 1;
  if (k == 1 || k == kn - 1) side3R(d, r - 1, 1, R);
  else if (k == kn) side2(d, c, c + 1, R);
  else side5R(d, r - 2, 1, R);
}

// z faces k = 1..kn, i = 2..ie-1, j = 1..jn-1 (Flux_Z.cpp:91-359)
__global__ void __launch_bounds__(64, CGLI_FLUX_MINBLOCKS) k_flux_z(Dev d) {
  int k = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  int j = 1 + blockIdx.y;
  int i = 2 + blockIdx.z;
  if (k > d.nz + 1) return;
  long long f = ix(d, i, j, k);
  double L[5], R[5], F[5], fav3, pp;
  muscl_z(d, i + 1, j + 1, k, L, R);
  double mm[9], Jf, iJf, sq, insqr;
  face_metrics(d, 2, f, j, mm, Jf, iJf);
  face_norm(d, 2, j, mm[6], mm[7], mm[8], sq, insqr);
  roe_face(L, R, mm[6], mm[7], mm[8], sq, insqr, iJf, d.e, F, fav3, pp);
  for (int v = 0; v < 5; v++) d.inF[2][v][f] = F[v];
}

// ---------------------------------------------------------------- viscous
// velocity and temperature of every cell the viscous face fluxes read
// (Viscous_terms.cpp:260-394): planes 2..ie+1, rows 1..nyy, k 1..nzz
__global__ void k_vprim(Dev d) {
  int k = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  int j = 1 + blockIdx.y;
  int i = 2 + blockIdx.z;
  if (k > d.nz + 2) return;
  long long c = ix(d, i, j, k);
  // the divisions by rho, rho R and J as Newton-refined reciprocals
  double rho = d.U_[0][c], irho = nr_rcp(rho);
  double U = d.U_[1][c] * irho, V = d.U_[2][c] * irho, W = d.U_[3][c] * irho;
  double P = (d.U_[4][c] - 0.5 * rho * (U * U + V * V + W * W)) * (KG - 1) * d.J[c];
  double T = P * (irho * (1.0 / RG)) * nr_rcp(d.J[c]);
  d.vprim[0][c] = U; d.vprim[1][c] = V; d.vprim[2][c] = W; d.vprim[3][c] = T;
}

struct VP { double U, V, W, T; };
__device__ __forceinline__ VP vp(const Dev &d, long long c) {
  VP r; r.U = d.vprim[0][c]; r.V = d.vprim[1][c]; r.W = d.vprim[2][c]; r.T = d.vprim[3][c]; return r;
}

// face viscous fluxes of cell (i,j,k): x face i-1/2 for j<=jn, k<=kn; y face
// j-1/2 for i<=ie, k<=kn; z face k-1/2 for i<=ie, j<=jn (the faces the
// divergence of Viscous_terms.cpp:875-904 reads).  CH: the face metrics have
// the channel's form (d.face_tables), so the per-row tables give eta_y and
// 1/J and the channel forms of the face fluxes apply.
// (the channel form fits 64 registers without spills: held at 16 CTAs per
// SM, 32 warps to hide its stencil loads)
template <bool CH>
__global__ void __launch_bounds__(64, (CH && CGLI_VISCOUS_MINBLOCKS < 16) ? 16 : CGLI_VISCOUS_MINBLOCKS)
    k_viscous_faces(Dev d) {
  int k = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  int j = 2 + blockIdx.y;
  int i = 3 + blockIdx.z;
  int ie = d.nx + 2, jn = d.ny + 1, kn = d.nz + 1;
  if (k > kn + 1) return;
  long long c = ix(d, i, j, k);
  long long f = ix(d, i - 1, j - 1, k - 1);
  const long long di = d.di, dj = d.dj;
  VP o = vp(d, c);
  if (j <= jn && k <= kn) {
    double out[4];
    if (CH) {
      const double *t = d.ftab + (0LL * d.Y + (j - 1)) * 4;
      visc_face_x_channel(d.rdxi, d.rdet, d.rdzt, d.mu, d.rpr, t[0], o, vp(d, c - di), vp(d, c + dj),
                          vp(d, c - di + dj), vp(d, c - dj), vp(d, c - di - dj), vp(d, c + 1), vp(d, c - di + 1),
                          vp(d, c - 1), vp(d, c - di - 1), t[2], out);
    } else {
      double mm[9], Jf, iJf;
      face_metrics(d, 0, f, j - 1, mm, Jf, iJf);
      visc_face_x(d.rdxi, d.rdet, d.rdzt, d.mu, d.rpr, o, vp(d, c - di), vp(d, c + dj), vp(d, c - di + dj), vp(d, c - dj),
                  vp(d, c - di - dj), vp(d, c + 1), vp(d, c - di + 1), vp(d, c - 1), vp(d, c - di - 1), mm, iJf, out);
    }
    for (int v = 0; v < 4; v++) d.vflux[0][v][c] = out[v];
  }
  if (i <= ie && k <= kn) {
    double out[4];
    if (CH) {
      const double *t = d.ftab + (1LL * d.Y + (j - 1)) * 4;
      visc_face_y_channel(d.rdxi, d.rdet, d.rdzt, d.mu, d.rpr, t[0], o, vp(d, c - dj), vp(d, c + di),
                          vp(d, c + di - dj), vp(d, c - di), vp(d, c - di - dj), vp(d, c + 1), vp(d, c - dj + 1),
                          vp(d, c - 1), vp(d, c - dj - 1), t[2], out);
    } else {
      double mm[9], Jf, iJf;
      face_metrics(d, 1, f, j - 1, mm, Jf, iJf);
      visc_face_y(d.rdxi, d.rdet, d.rdzt, d.mu, d.rpr, o, vp(d, c - dj), vp(d, c + di), vp(d, c + di - dj), vp(d, c - di),
                  vp(d, c - di - dj), vp(d, c + 1), vp(d, c - dj + 1), vp(d, c - 1), vp(d, c - dj - 1), mm, iJf, out);
    }
    for (int v = 0; v < 4; v++) d.vflux[1][v][c] = out[v];
  }
  if (i <= ie && j <= jn) {
    double out[4];
    if (CH) {
      const double *t = d.ftab + (2LL * d.Y + (j - 1)) * 4;
      visc_face_z_channel(d.rdxi, d.rdet, d.rdzt, d.mu, d.rpr, t[0], o, vp(d, c - 1), vp(d, c + di),
                          vp(d, c + di - 1), vp(d, c - di), vp(d, c - di - 1), vp(d, c + dj), vp(d, c + dj - 1),
                          vp(d, c - dj), vp(d, c - dj - 1), t[2], out);
    } else {
      double mm[9], Jf, iJf;
      face_metrics(d, 2, f, j - 1, mm, Jf, iJf);
      visc_face_z(d.rdxi, d.rdet, d.rdzt, d.mu, d.rpr, o, vp(d, c - 1), vp(d, c + di), vp(d, c + di - 1), vp(d, c - di),
                  vp(d, c - di - 1), vp(d, c + dj), vp(d, c + dj - 1), vp(d, c - dj), vp(d, c - dj - 1),
                  vp(d, c - di + dj), mm, iJf, out);
    }
    for (int v = 0; v < 4; v++) d.vflux[2][v][c] = out[v];
  }
}

// Viscous_terms.cpp:875-904
__global__ void k_viscous_div(Dev d) {
  int k = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  int j = 2 + blockIdx.y;
  int i = 3 + blockIdx.z;
  if (k > d.nz + 1) return;
  long long c = ix(d, i, j, k);
  const double invXI = d.rdxi, invET = d.rdet, invZT = d.rdzt;
  for (int v = 0; v < 4; v++)
    d.vF[v][c] = (d.vflux[0][v][c + d.di] - d.vflux[0][v][c]) * invXI +
                 (d.vflux[1][v][c + d.dj] - d.vflux[1][v][c]) * invET +
                 (d.vflux[2][v][c + 1] - d.vflux[2][v][c]) * invZT;
}

// ---------------------------------------------------- dual-time residual
// Dual_time_stepping.cpp:737-922 (the sponge Residual terms are zero for a
// domain without inlet / outlet layers and are left out)
__global__ void k_dts_residual(Dev d) {
  int k = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  int j = 2 + blockIdx.y;
  int i = 3 + blockIdx.z;
  if (k > d.nz + 1) return;
  long long c = ix(d, i, j, k);
  const double J = d.J[c], deltaT = d.dt;
  CPrim<double> q = cprim<double>(d.U_[0][c], d.U_[1][c], d.U_[2][c], d.U_[3][c], d.U_[4][c], J, d.e);
  double rho = q.rho, u = q.u, v = q.v, w = q.w, VV = q.VV, T = q.Tt, H = q.H, beta = q.beta;
  double temp = rho * KG;
  double d11 = -(H * (KG - 1) + VV - KG * (T + VV)) * beta;
  double d12 = -(KG - 1) * u * beta, d13 = -(KG - 1) * v * beta, d14 = -(KG - 1) * w * beta;
  double d15 = (KG - 1) * beta;
  double d21 = -u / rho, d22 = 1 / rho;
  double d31 = -v / rho;
  double d41 = -w / rho;
  double d51 = (KG - 1) * (VV + KG * T * beta + (KG - 1) * VV * beta + H * (-1 + beta - KG * beta)) / temp;
  double d52 = -(KG - 1) * u * (1 + (KG - 1) * beta) / temp;
  double d53 = -(KG - 1) * v * (1 + (KG - 1) * beta) / temp;
  double d54 = -(KG - 1) * w * (1 + (KG - 1) * beta) / temp;
  double d55 = (KG - 1) * (1 + (KG - 1) * beta) / temp;
  long long fx1 = ix(d, i, j - 1, k - 1), fx0 = ix(d, i - 1, j - 1, k - 1);
  long long fy1 = ix(d, i - 1, j, k - 1), fz1 = ix(d, i - 1, j - 1, k);
  double Rk[5], sp[5];
  sponge_terms(d, i, c, sp);
  double f = d.buoyancy ? -(rho - 1.1842) * 9.81 : d.scal[0];
  for (int n = 0; n < 5; n++) {
    double Rp = -(3 * d.U_[n][c] - 4 * d.U[n][c] + d.Uq[n][c]) / (2 * deltaT);
    double Rf = -((d.inF[0][n][fx1] - d.inF[0][n][fx0]) / d.dxi + (d.inF[1][n][fy1] - d.inF[1][n][fx0]) / d.det +
                  (d.inF[2][n][fz1] - d.inF[2][n][fx0]) / d.dzt);
    Rk[n] = sp[n] / J + Rp + Rf;
  }
  Rk[1] = Rk[1] + d.vF[0][c] + f / J;
  Rk[2] = Rk[2] + d.vF[1][c];
  Rk[3] = Rk[3] + d.vF[2][c];
  Rk[4] = Rk[4] + d.vF[3][c] + f * u / J;
  double MR1 = (d11 * Rk[0] + d12 * Rk[1] + d13 * Rk[2] + d14 * Rk[3] + d15 * Rk[4]);
  double MR2 = (d21 * Rk[0] + d22 * Rk[1]);
  double MR3 = (d31 * Rk[0] + d22 * Rk[2]);
  double MR4 = (d41 * Rk[0] + d22 * Rk[3]);
  double MR5 = (d51 * Rk[0] + d52 * Rk[1] + d53 * Rk[2] + d54 * Rk[3] + d55 * Rk[4]);
  d.MR[0][c] = MR1; d.MR[1][c] = MR2; d.MR[2][c] = MR3; d.MR[3][c] = MR4; d.MR[4][c] = MR5;
  double mm[9];
  for (int v2 = 0; v2 < 9; v2++) mm[v2] = d.m[v2][c];
  Diag<double> dd = diag<double>(q, mm, d.dxi, d.det, d.dzt, deltaT);
  double n1 = dd.d11 * MR1, n2 = dd.d22 * MR2, n3 = dd.d22 * MR3, n4 = dd.d22 * MR4;
  double n5 = dd.d51 * MR1 + dd.d22 * MR5;
  d.NL[0][c] = n1; d.NL[1][c] = n2; d.NL[2][c] = n3; d.NL[3][c] = n4; d.NL[4][c] = n5;
  d.NR[0][c] = n1; d.NR[1][c] = n2; d.NR[2][c] = n3; d.NR[3][c] = n4; d.NR[4][c] = n5;
}

// ------------------------------------------------------------- sweeps
// lagged periodic halo planes of the sweep, Dual_time_stepping.cpp:942-976:
// NL[2] <- NL[ie], NR[ie+1] <- NR[3]; zero on an open slab (:204-246, and
// the exchange with absent neighbours leaves them so)
__global__ void k_sweep_halo(Dev d) {
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= d.di) return;
  int v = blockIdx.y;
  int ie = d.nx + 2;
  d.NL[v][2 * d.di + t] = d.x_open ? 0.0 : d.NL[v][(long long)ie * d.di + t];
  d.NR[v][(long long)(ie + 1) * d.di + t] = d.x_open ? 0.0 : d.NR[v][3 * d.di + t];
}

__device__ __forceinline__ CPrim<double> cp_at(const Dev &d, long long c) {
  return cprim<double>(d.U_[0][c], d.U_[1][c], d.U_[2][c], d.U_[3][c], d.U_[4][c], d.J[c], d.e);
}
__device__ __forceinline__ Split<double> split_at(const Dev &d, long long c, int dir) {
  CPrim<double> q = cp_at(d, c);
  return split<double>(q, d.m[3 * dir][c], d.m[3 * dir + 1][c], d.m[3 * dir + 2][c], dir == 0);
}

// forward sweep on hyperplane m = i+j+k, Dual_time_stepping.cpp:983-1300
__global__ void k_forward_plane(Dev d, int m, int ilo, int jcount) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int i = ilo + t / jcount, j = 2 + t % jcount;
  int k = m - i - j;
  int ie = d.nx + 2, kn = d.nz + 1;
  if (i > ie || k < 2 || k > kn) return;
  long long c = ix(d, i, j, k), ci = c - d.di, cj = c - d.dj, ck = c - 1;
  double a[5], b[5], e3[5], n[5];
  for (int v = 0; v < 5; v++) n[v] = d.NL[v][ci];
  lower_terms<double>(split_at(d, ci, 0), n, a);
  for (int v = 0; v < 5; v++) n[v] = d.NL[v][cj];
  lower_terms<double>(split_at(d, cj, 1), n, b);
  for (int v = 0; v < 5; v++) n[v] = d.NL[v][ck];
  lower_terms<double>(split_at(d, ck, 2), n, e3);
  double LL[5];
  for (int v = 0; v < 5; v++) LL[v] = a[v] / d.dxi + b[v] / d.det + e3[v] / d.dzt;
  CPrim<double> q = cp_at(d, c);
  double mm[9];
  for (int v = 0; v < 9; v++) mm[v] = d.m[v][c];
  Diag<double> dg = diag<double>(q, mm, d.dxi, d.det, d.dzt, d.dt);
  double r1 = d.MR[0][c] - LL[0];
  d.NL[0][c] = dg.d11 * r1;
  d.NL[1][c] = dg.d22 * (d.MR[1][c] - LL[1]);
  d.NL[2][c] = dg.d22 * (d.MR[2][c] - LL[2]);
  d.NL[3][c] = dg.d22 * (d.MR[3][c] - LL[3]);
  d.NL[4][c] = dg.d51 * r1 + dg.d22 * (d.MR[4][c] - LL[4]);
}

// backward sweep on hyperplane m, Dual_time_stepping.cpp:1312-1664
__global__ void k_backward_plane(Dev d, int m, int ilo, int jcount) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  int i = ilo + t / jcount, j = 2 + t % jcount;
  int k = m - i - j;
  int ie = d.nx + 2, kn = d.nz + 1;
  if (i > ie || k < 2 || k > kn) return;
  long long c = ix(d, i, j, k), ci = c + d.di, cj = c + d.dj, ck = c + 1;
  double a[5], b[5], e3[5], n[5];
  for (int v = 0; v < 5; v++) n[v] = d.NR[v][ci];
  upper_terms<double>(split_at(d, ci, 0), n, a);
  for (int v = 0; v < 5; v++) n[v] = d.NR[v][cj];
  upper_terms<double>(split_at(d, cj, 1), n, b);
  for (int v = 0; v < 5; v++) n[v] = d.NR[v][ck];
  upper_terms<double>(split_at(d, ck, 2), n, e3);
  double UU[5];
  for (int v = 0; v < 5; v++) UU[v] = a[v] / d.dxi + b[v] / d.det + e3[v] / d.dzt;
  CPrim<double> q = cp_at(d, c);
  double mm[9];
  for (int v = 0; v < 9; v++) mm[v] = d.m[v][c];
  Diag<double> dg = diag<double>(q, mm, d.dxi, d.det, d.dzt, d.dt);
  d.NR[0][c] = d.NL[0][c] - dg.d11 * UU[0];
  d.NR[1][c] = d.NL[1][c] - dg.d22 * UU[1];
  d.NR[2][c] = d.NL[2][c] - dg.d22 * UU[2];
  d.NR[3][c] = d.NL[3][c] - dg.d22 * UU[3];
  d.NR[4][c] = d.NL[4][c] - (dg.d51 * UU[0] + dg.d22 * UU[4]);
}

// NL <- NR on interior cells, Dual_time_stepping.cpp:1675-1689
__global__ void k_copy_nr_nl(Dev d) {
  int k = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  int j = 2 + blockIdx.y;
  int i = 3 + blockIdx.z;
  if (k > d.nz + 1) return;
  long long c = ix(d, i, j, k);
  for (int v = 0; v < 5; v++) d.NL[v][c] = d.NR[v][c];
}

// --------------------------------------------------------------- update
// Dual_time_stepping.cpp:1702-1743 plus per-block partial sums of the
// squared increments (:1761-1776); one block per (j,i) row pair of k
__global__ void k_update(Dev d) {
  int k = 2 + threadIdx.x;
  int j = 2 + blockIdx.x;
  int i = 3 + blockIdx.y;
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
    double P = Pold + d.NR[0][c] * J;
    double U = Uold + d.NR[1][c] * J;
    double V = Vold + d.NR[2][c] * J;
    double W = Wold + d.NR[3][c] * J;
    double T = Told + d.NR[4][c] * J;
    double rho = P / T;
    d.U_[0][c] = rho / J;
    d.U_[1][c] = rho * U / J;
    d.U_[2][c] = rho * V / J;
    d.U_[3][c] = rho * W / J;
    d.U_[4][c] = (P / (KG - 1) + 0.5 * rho * (U * U + V * V + W * W)) / J;
    acc[0] += (rho - rhoold) * (rho - rhoold);
    acc[1] += (U - Uold) * (U - Uold);
    acc[2] += (V - Vold) * (V - Vold);
    acc[3] += (W - Wold) * (W - Wold);
    acc[4] += (T - Told) * (T - Told);
  }
  block_sum5(acc, d.partial + 5 * ((long long)blockIdx.y * gridDim.x + blockIdx.x));
}

// ------------------------------------------------------------ launchers
static dim3 cellgrid(int nk, int nj, int ni, int bx) { return dim3((nk + bx - 1) / bx, nj, ni); }

// main.cpp:167-210: halo exchange, then Y, X, Z boundaries
void launch_halo_bc(const Dev &d, cudaStream_t s) {
  launch_halo_x(d, s);
  k_bc_y<<<dim3((d.nz + 127) / 128, d.nx, 2), 128, 0, s>>>(d);
  launch_bc_x(d, s);
  long long rows = (long long)d.X * d.Y;
  k_bc_z<<<dim3((unsigned)((rows + 255) / 256), 5), 256, 0, s>>>(d);
}
void launch_halo_x(const Dev &d, cudaStream_t s) {
  if (d.x_open) return;   // both neighbours absent
  long long n = 3 * d.di;
  k_halo_x<<<dim3((unsigned)((n + 255) / 256), 5), 256, 0, s>>>(d);
}
void launch_bc_x(const Dev &d, cudaStream_t s) {
  if (!d.x_open) return;   // interior rank: no-op
  k_bc_x<<<dim3((d.nz + 63) / 64, d.ny, 2), 64, 0, s>>>(d);
}
bool check_face_tables(const Dev &d, int *dflag, cudaStream_t s) {
  const int ie = d.nx + 2, jn = d.ny + 1, kn = d.nz + 1;
  const int one = 1;
  if (cudaMemcpyAsync(dflag, &one, sizeof(int), cudaMemcpyHostToDevice, s) != cudaSuccess) return false;
  const int rng[3][3] = {{ie, jn - 1, kn - 1}, {ie - 1, jn, kn - 1}, {ie - 1, jn - 1, kn}};
  for (int set = 0; set < 3; set++)
    k_check_face_set<<<dim3((rng[set][2] + 127) / 128, rng[set][1], rng[set][0] - 1), 128, 0, s>>>(
        d, set, rng[set][0], rng[set][1], rng[set][2], dflag);
  int ok = 0;
  if (cudaMemcpyAsync(&ok, dflag, sizeof(int), cudaMemcpyDeviceToHost, s) != cudaSuccess) return false;
  if (cudaStreamSynchronize(s) != cudaSuccess) return false;
  if (ok) k_fill_face_tables<<<(d.Y + 127) / 128, 128, 0, s>>>(d);
  return ok != 0;
}

void launch_target_u(const Dev &d, cudaStream_t s) {
  if (!d.x_open || d.nx_outlet == 0) return;
  k_target_u<<<1, 256, 0, s>>>(d);
}
void launch_bc_y(const Dev &d, cudaStream_t s) {
  k_bc_y<<<dim3((d.nz + 127) / 128, d.nx, 2), 128, 0, s>>>(d);
}
void launch_bc_z(const Dev &d, cudaStream_t s) {
  long long rows = (long long)d.X * d.Y;
  k_bc_z<<<dim3((unsigned)((rows + 255) / 256), 5), 256, 0, s>>>(d);
}
void launch_flux_x(const Dev &d, cudaStream_t s) {
  k_flux_x<<<cellgrid(d.nz, d.ny, d.nx + 1, 64), 64, 0, s>>>(d);
}
void launch_flux_y(const Dev &d, cudaStream_t s) {
  k_flux_y<<<cellgrid(d.nz, d.ny + 1, d.nx, 64), 64, 0, s>>>(d);
}
void launch_flux_z(const Dev &d, cudaStream_t s) {
  k_flux_z<<<cellgrid(d.nz + 1, d.ny, d.nx, 64), 64, 0, s>>>(d);
}
void launch_viscous(const Dev &d, cudaStream_t s) {
  k_vprim<<<cellgrid(d.nz + 2, d.ny + 2, d.nx + 2, 64), 64, 0, s>>>(d);
  if (d.face_tables) k_viscous_faces<true><<<cellgrid(d.nz + 1, d.ny + 1, d.nx + 1, 64), 64, 0, s>>>(d);
  else k_viscous_faces<false><<<cellgrid(d.nz + 1, d.ny + 1, d.nx + 1, 64), 64, 0, s>>>(d);
  k_viscous_div<<<cellgrid(d.nz, d.ny, d.nx, 64), 64, 0, s>>>(d);
}
void launch_dts_residual(const Dev &d, cudaStream_t s) {
  k_dts_residual<<<cellgrid(d.nz, d.ny, d.nx, 64), 64, 0, s>>>(d);
}

void launch_dts(const Dev &d, cudaStream_t s, int update_blocks_x) {
  launch_target_u(d, s);
  k_dts_residual<<<cellgrid(d.nz, d.ny, d.nx, 64), 64, 0, s>>>(d);
  int ie = d.nx + 2, jn = d.ny + 1, kn = d.nz + 1;
  for (int sweep = 1; sweep <= 2; sweep++) {
    k_sweep_halo<<<dim3((unsigned)((d.di + 255) / 256), 5), 256, 0, s>>>(d);
    for (int m = 7; m <= ie + jn + kn; m++) {
      int ilo = m - jn - kn > 3 ? m - jn - kn : 3;
      int ihi = m - 4 < ie ? m - 4 : ie;
      int n = (ihi - ilo + 1) * d.ny;
      k_forward_plane<<<(n + 127) / 128, 128, 0, s>>>(d, m, ilo, d.ny);
    }
    for (int m = ie + jn + kn; m >= 7; m--) {
      int ilo = m - jn - kn > 3 ? m - jn - kn : 3;
      int ihi = m - 4 < ie ? m - 4 : ie;
      int n = (ihi - ilo + 1) * d.ny;
      k_backward_plane<<<(n + 127) / 128, 128, 0, s>>>(d, m, ilo, d.ny);
    }
    k_copy_nr_nl<<<cellgrid(d.nz, d.ny, d.nx, 64), 64, 0, s>>>(d);
  }
  (void)update_blocks_x;
  k_update<<<dim3(d.ny, d.nx), 128, 0, s>>>(d);
}

// five norms from the per-block partial sums, in a fixed order
__global__ void k_norms(const double *partial, int nblocks, double scale, double *out) {
  double acc[5] = {0, 0, 0, 0, 0};
  for (int b = threadIdx.x; b < nblocks; b += blockDim.x)
    for (int v = 0; v < 5; v++) acc[v] += partial[5 * (long long)b + v];
  __shared__ double tot[5];
  block_sum5(acc, tot);
  __syncthreads();
  if (threadIdx.x < 5) out[threadIdx.x] = sqrt(tot[threadIdx.x]) * scale;
}

// bulk mass flux, Driven_force.cpp:38-62: sum over interior cells of
// (U2_*J)/J / Jsum with Jsum the column volume sum at (i,k) = (3,3)
// bulk mass flux of Driven_force.cpp:38-62: sum over the interior of
// (rho u / J... as written) / Jsum, divided by Nx Nz; a grid-wide two-stage
// reduction in a fixed order (per-block partials, then one block)
__global__ void k_bulk_partial(Dev d, double *part) {
  double acc[5] = {0, 0, 0, 0, 0};
  const long long n = (long long)d.nx * d.ny * d.nz;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < n; t += (long long)gridDim.x * blockDim.x) {
    int k = (int)(t % d.nz), j = (int)((t / d.nz) % d.ny), i = (int)(t / ((long long)d.nz * d.ny));
    long long c = ix(d, i + 3, j + 2, k + 2);
    acc[0] += (d.U_[1][c] * d.J[c]) * 1. / d.J[c];
  }
  __shared__ double tot[5];
  block_sum5(acc, tot);
  __syncthreads();
  if (threadIdx.x == 0) part[blockIdx.x] = tot[0];
}
__global__ void k_bulk_final(Dev d, const double *part, int nblk, double *out) {
  double acc[5] = {0, 0, 0, 0, 0};
  for (int b = threadIdx.x; b < nblk; b += blockDim.x) acc[0] += part[b];
  __shared__ double tot[5];
  block_sum5(acc, tot);
  __syncthreads();
  if (threadIdx.x == 0) {
    double Jsum = 0;
    for (int j = 2; j <= d.ny + 1; j++) Jsum = Jsum + 1. / d.J[ix(d, 3, j, 3)];
    out[0] = tot[0] / Jsum / d.nx / d.nz;
  }
}

// main.cpp:364-386 over planes 2..ie+1, all rows; Q^(n-2) is kept as well
__global__ void k_end_step(Dev d) {
  long long n = (long long)(d.nx + 2) * d.di;
  long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= n) return;
  int v = blockIdx.y;
  long long c = 2 * d.di + t;
  d.Uqq[v][c] = d.Uq[v][c];
  d.Uq[v][c] = d.U[v][c];
  d.U[v][c] = d.U_[v][c];
}

// initial guess of the inner iteration on the interior cells: order 1 gives
// 2Q^n - Q^(n-1), order 2 gives 3Q^n - 3Q^(n-1) + Q^(n-2) (of Q/J; the grid
// is fixed in time, so extrapolating Q/J is extrapolating Q)
__global__ void k_predict(Dev d, int order) {
  int k = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  int j = 2 + blockIdx.y;
  int i = 3 + blockIdx.z;
  if (k > d.nz + 1) return;
  long long c = ix(d, i, j, k);
  for (int v = 0; v < 5; v++) {
    double q = d.U[v][c], q1 = d.Uq[v][c];
    d.U_[v][c] = order >= 2 ? 3 * q - 3 * q1 + d.Uqq[v][c] : 2 * q - q1;
  }
}

void launch_predict(const Dev &d, cudaStream_t s, int order) {
  k_predict<<<dim3((d.nz + 63) / 64, d.ny, d.nx), 64, 0, s>>>(d, order);
}

void launch_norms(const Dev &d, cudaStream_t s, int nblocks, double scale, double *out) {
  k_norms<<<1, 1024, 0, s>>>(d.partial, nblocks, scale, out);
}
__global__ void k_inverse_j(Dev d, long long n) {
  const long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (c < n) d.iJ[c] = d.J[c] != 0.0 ? 1.0 / d.J[c] : 0.0;
}
void launch_inverse_j(const Dev &d, cudaStream_t s) {
  const long long n = (long long)d.X * d.Y * d.Z;
  k_inverse_j<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(d, n);
}
void launch_bulk_flux(const Dev &d, cudaStream_t s, double *out) {
  // the per-block partials go to out[8 ..]: the caller's scratch holds 8 + 296 doubles
  constexpr int kBlocks = 296;
  k_bulk_partial<<<kBlocks, 256, 0, s>>>(d, out + 8);
  k_bulk_final<<<1, 256, 0, s>>>(d, out + 8, kBlocks, out);
}
void launch_end_step(const Dev &d, cudaStream_t s) {
  long long n = (long long)(d.nx + 2) * d.di;
  k_end_step<<<dim3((unsigned)((n + 255) / 256), 5), 256, 0, s>>>(d);
}

}  // namespace cgli
