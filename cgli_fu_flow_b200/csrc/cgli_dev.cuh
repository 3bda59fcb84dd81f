// Device-side state description and the per-cell / per-face arithmetic of
// the hot path, shared by every kernel translation unit.
//
// All arrays use the reference layout [X_np][Y_m][Z_m], k fastest (see
// include/cgli_fu_flow.h).  The arithmetic helpers restate the reference's
// expressions in the same evaluation order (file:line cited at each); the
// compiler may contract a*b+c into fused multiply-adds, so results agree
// with the CPU reference to rounding, not bit for bit.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace cgli {

constexpr double KG = 1.4;    // gamma, prm.h:7
constexpr double RG = 287.0;  // gas constant, prm.h:8
constexpr double CV = 717.5;  // Viscous_terms.h:3

// Pointers and sizes of one context's device state; passed by value.
struct Dev {
  int nx, ny, nz;         // interior cells
  int X, Y, Z;            // X_np, Y_m, Z_m
  long long di, dj;       // strides of i and j (k stride is 1)
  double dxi, det, dzt, dt, e, mu, pr, twl, twh;
  double rdxi, rdet, rdzt, rpr;   // 1/dxi, 1/det, 1/dzt, 1/pr (formed on the host)
  int curved_walls;       // wall-face pressure force with eta_x, eta_z terms
  int x_open;             // open x ends (single rank 0 of 1), else a periodic slab
  int nx_inlet, nx_outlet;  // sponge layers (open x only)
  int buoyancy;           // f = -(rho - 1.1842) 9.81 instead of scal[0]
  double high;            // channel height parameter (sponge strength)
  double *U_[5], *U[5], *Uq[5];
  double *Uqq[5];         // Q^(n-2)/J for the extrapolated initial guess
  double *J, *m[9];
  double *iJ;             // 1/J per cell (0 where J = 0), formed when the metrics change
  double *Jf[3], *mf[3][9];
  // per-row face metrics [3 sets][Y][etdy, J, 1/J, 1/|etdy|], used when
  // face_tables is set: every face of each set has the channel's form
  // xi = (1,0,0), eta = (0,etdy(row),0), zeta = (0,0,1) with J a function of
  // the row
  double *ftab;
  int face_tables;
  double *inF[3][5], *vF[4];
  double *MR[5], *NL[5], *NR[5];
  double *vflux[3][4];
  double *vprim[4];
  double *scal;           // [0] = driving force, [1] = outlet sponge target velocity
  double *partial;        // per-block partial sums of the update norms
  int *status;            // device status word (0 ok)
  // mixed-precision sweep state
  float *MRf[5], *NLf[5], *NRf[5];
};

__host__ __device__ __forceinline__ long long ix(const Dev &d, int i, int j, int k) {
  return (long long)i * d.di + (long long)j * d.dj + k;
}

// ------------------------------------------ FP64 reciprocal and square root
// The residual side is bound by FP64 arithmetic, and an IEEE-rounded FP64
// division or square root is a long instruction sequence with a special-case
// branch.  These two refine the hardware's approximate seeds (PTX
// rcp.approx.ftz.f64 and rsqrt.approx.ftz.f64, each good to about 20 bits)
// by Newton-Raphson iteration with fused multiply-adds:
//   reciprocal of a:  e = 1 - a y,  y <- y + y e          (twice)
//   square root of x: g = x y, h = y / 2 (g ~ sqrt x, h ~ 1 / (2 sqrt x)),
//                     r = 1/2 - g h,  g <- g + g r,  h <- h + h r   (coupled
//                     Newton step on g and h), then g <- g + h (x - g g)
// (P. Markstein, "Computation of elementary functions on the IBM RISC
// System/6000 processor", IBM J. Res. Dev. 34(1), 1990).  Each step roughly
// squares the relative error, so both results are within one unit in the
// last place of the rounded value for the positive normal operands the
// solver forms (densities, pressures, sound speeds, metric norms, face
// Jacobians); the tests check that bound against CUDA's IEEE results.  Only
// finite positive operands are meant: a zero or non-finite operand returns
// NaN (the reciprocal), and x <= 0 returns 0 for x == 0 or NaN.
__device__ __forceinline__ double nr_rcp(double a) {
  double y;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(a));
  double e = fma(-a, y, 1.0);
  y = fma(y, e, y);
  e = fma(-a, y, 1.0);
  return fma(y, e, y);
}
__device__ __forceinline__ double nr_sqrt(double x) {
  double y;
  asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
  double g = x * y, h = 0.5 * y;
  const double r = fma(-g, h, 0.5);
  g = fma(g, r, g);
  h = fma(h, r, h);
  g = fma(fma(-g, g, x), h, g);
  return x > 0.0 ? g : (x == 0.0 ? 0.0 : __longlong_as_double(0x7ff8000000000000LL));
}

// the nine metric terms, J and 1/J of face set `set` (0 x, 1 y, 2 z faces)
// at face index f, whose row index is jj: from the per-row tables when the
// face metrics have the channel's form, else from the 3-D face arrays
__device__ __forceinline__ void face_metrics(const Dev &d, int set, long long f, int jj, double mm[9], double &Jf,
                                             double &iJf) {
  if (d.face_tables) {
    const double *t = d.ftab + ((long long)set * d.Y + jj) * 4;
    mm[0] = 1; mm[1] = 0; mm[2] = 0; mm[3] = 0; mm[4] = t[0]; mm[5] = 0; mm[6] = 0; mm[7] = 0; mm[8] = 1;
    Jf = t[1];
    iJf = t[2];
  } else {
#pragma unroll
    for (int v = 0; v < 9; v++) mm[v] = d.mf[set][v][f];
    Jf = d.Jf[set][f];
    iJf = nr_rcp(Jf);
  }
}

// |n| and 1/|n| of the face normal of direction `set` (the metric vector of
// that direction): from the per-row table on the channel grid (1 for the x
// and z faces, |etdy| for the y faces), else formed from the metric terms
__device__ __forceinline__ void face_norm(const Dev &d, int set, int jj, double mx, double my, double mz, double &sq,
                                          double &insqr) {
  if (d.face_tables) {
    if (set == 1) {
      sq = fabs(my);
      insqr = d.ftab[((long long)set * d.Y + jj) * 4 + 3];
    } else {
      sq = 1.0;
      insqr = 1.0;
    }
  } else {
    sq = nr_sqrt(mx * mx + my * my + mz * mz);
    insqr = nr_rcp(sq);
  }
}

// ---------------------------------------------------------------- MUSCL
// 1/J-weighted upwind-biased interpolation of Q/J (Flux_X.cpp:112-126 and
// the reduced stencils of Flux_X.cpp:138-216, Flux_Y.cpp:135-250,
// Flux_Z.cpp:135-216).
__device__ __forceinline__ double m5L(const double *u, const double *J, long long a, long long b,
                                      long long c, long long dd, long long e) {
  double t = 1. / (2 / J[a] - 13 / J[b] + 47 / J[c] + 27 / J[dd] - 3 / J[e]);
  return t * (2 * u[a] - 13 * u[b] + 47 * u[c] + 27 * u[dd] - 3 * u[e]);
}
__device__ __forceinline__ double m5R(const double *u, const double *J, long long a, long long b,
                                      long long c, long long dd, long long e) {
  double t = 1. / (-3 / J[a] + 27 / J[b] + 47 / J[c] - 13 / J[dd] + 2 / J[e]);
  return t * (-3 * u[a] + 27 * u[b] + 47 * u[c] - 13 * u[dd] + 2 * u[e]);
}
__device__ __forceinline__ double m3L(const double *u, const double *J, long long a, long long b, long long c) {
  double t = 1. / (-1 / J[a] + 5 / J[b] + 2 / J[c]);
  return t * (-u[a] + 5 * u[b] + 2 * u[c]);
}
__device__ __forceinline__ double m3R(const double *u, const double *J, long long a, long long b, long long c) {
  double t = 1. / (2 / J[a] + 5 / J[b] - 1 / J[c]);
  return t * (2 * u[a] + 5 * u[b] - u[c]);
}
__device__ __forceinline__ double m2(const double *u, const double *J, long long a, long long b) {
  double t = 1. / (1 / J[a] + 1 / J[b]);
  return t * (u[a] + u[b]);
}

// One side of a face for all five variables: the weight
// t = 1 / sum(c_p / J_p) (c_p / J_p as c_p times the cell's stored 1/J) is
// computed once and applied to each variable's sum(c_p u_p) (the reference's
// m5L/m5R/m3L/m3R/m2 expressions, same evaluation order).
template <int N>
__device__ __forceinline__ void muscl_side(const Dev &d, const long long (&o)[N], const double (&c)[N], double out[5]) {
  double s = c[0] * d.iJ[o[0]];
#pragma unroll
  for (int p = 1; p < N; p++) s += c[p] * d.iJ[o[p]];
  const double t = nr_rcp(s);
#pragma unroll
  for (int v = 0; v < 5; v++) {
    const double *u = d.U_[v];
    double a = c[0] * u[o[0]];
#pragma unroll
    for (int p = 1; p < N; p++) a += c[p] * u[o[p]];
    out[v] = t * a;
  }
}
// stencil kinds: 5L, 5R on (a..e); 3L, 3R on (a, b, c); 2 on (a, b)
__device__ __forceinline__ void side5L(const Dev &d, long long a, long long st, double out[5]) {
  const long long o[5] = {a, a + st, a + 2 * st, a + 3 * st, a + 4 * st};
  const double c[5] = {2, -13, 47, 27, -3};
  muscl_side<5>(d, o, c, out);
}
__device__ __forceinline__ void side5R(const Dev &d, long long a, long long st, double out[5]) {
  const long long o[5] = {a, a + st, a + 2 * st, a + 3 * st, a + 4 * st};
  const double c[5] = {-3, 27, 47, -13, 2};
  muscl_side<5>(d, o, c, out);
}
__device__ __forceinline__ void side3L(const Dev &d, long long a, long long st, double out[5]) {
  const long long o[3] = {a, a + st, a + 2 * st};
  const double c[3] = {-1, 5, 2};
  muscl_side<3>(d, o, c, out);
}
__device__ __forceinline__ void side3R(const Dev &d, long long a, long long st, double out[5]) {
  const long long o[3] = {a, a + st, a + 2 * st};
  const double c[3] = {2, 5, -1};
  muscl_side<3>(d, o, c, out);
}
__device__ __forceinline__ void side2(const Dev &d, long long a, long long b, double out[5]) {
  const long long o[2] = {a, b};
  const double c[2] = {1, 1};
  muscl_side<2>(d, o, c, out);
}

// ------------------------------------------------------------- Roe flux
// Preconditioned Roe flux through one face, Flux_X.cpp:229-350 (same
// statements in Flux_Y.cpp:291-396 and Flux_Z.cpp:250-354; the pressure-jump
// term uses the face's own unit normal).  L, R: MUSCL states; (mx,my,mz)
// face metric, sq its norm and insqr = 1/sq; iJf the reciprocal of the face
// Jacobian.  Also returns Fav3 and iP+P_ for the wall faces of
// Flux_Y.cpp:400-408.
__device__ __forceinline__ void roe_face(const double L[5], const double R[5], double mx, double my,
                                         double mz, double sq, double insqr, double iJf, double e, double F[5],
                                         double &Fav3o, double &ppo) {
  // The reference's statements in its order; each group of divisions by one
  // denominator is one reciprocal and products, the divisions by the
  // constant gamma - 1 are products with its reciprocal, the Roe-averaged
  // density sqrt(rho_L rho_R) is the product of the two square roots the
  // averages use anyway, and the reciprocals and square roots are the
  // Newton-refined ones (results differ from the reference's in the last
  // bits only).
  constexpr double rkg = 1.0 / (KG - 1);
  const double NX = mx * insqr, NY = my * insqr, NZ = mz * insqr;
  const double _rho = L[0], irl = nr_rcp(_rho);
  const double _u = L[1] * irl, _v = L[2] * irl, _w = L[3] * irl;
  const double iU = mx * _u + my * _v + mz * _w;
  const double _VV = _u * _u + _v * _v + _w * _w;
  const double iP = (L[4] - 0.5 * _rho * _VV) * (KG - 1);
  const double iC = KG * iP * irl;
  const double _H = 0.5 * _VV + iC * rkg;
  const double rho_ = R[0], irr = nr_rcp(rho_);
  const double u_ = R[1] * irr, v_ = R[2] * irr, w_ = R[3] * irr;
  const double U_ = mx * u_ + my * v_ + mz * w_;
  const double VV_ = u_ * u_ + v_ * v_ + w_ * w_;
  const double P_ = (R[4] - 0.5 * rho_ * VV_) * (KG - 1);
  const double C_ = KG * P_ * irr;
  const double H_ = 0.5 * VV_ + C_ * rkg;
  const double temp5 = nr_sqrt(_rho), temp6 = nr_sqrt(rho_);
  const double i4 = nr_rcp(temp5 + temp6);
  const double rho = temp5 * temp6;
  const double u = (temp5 * _u + temp6 * u_) * i4;
  const double v = (temp5 * _v + temp6 * v_) * i4;
  const double w = (temp5 * _w + temp6 * w_) * i4;
  const double U = (temp5 * iU + temp6 * U_) * i4;
  const double VV = u * u + v * v + w * w;
  const double H = (temp5 * _H + temp6 * H_) * i4;
  const double C = (H - 0.5 * VV) * (KG - 1);
  const double iCc = nr_rcp(C);
  const double dU1 = rho_ - _rho;
  const double dU2 = rho_ * u_ - _rho * _u;
  const double dU3 = rho_ * v_ - _rho * _v;
  const double dU4 = rho_ * w_ - _rho * _w;
  const double dU5 = (P_ * rkg + 0.5 * rho_ * VV_) - (iP * rkg + 0.5 * _rho * _VV);
  const double theda_p = VV * iCc;
  const double beta = theda_p > e ? theda_p : e;   // max() macro semantics
  const double Un = U * insqr;
  const double temp = 0.5 * (1 + beta) * Un;
  const double S = 0.5 * nr_sqrt(4 * beta * C + Un * Un * (1 - beta) * (1 - beta));
  const double iS = nr_rcp(S);
  const double U_p = 0.5 * (1 + theda_p) * Un;
  const double C_p = 0.5 * nr_sqrt(4 * C * theda_p + Un * Un * (1 - theda_p) * (1 - theda_p));
  const double dP = P_ - iP, dUn = (U_ - iU) * insqr;
  const double temp1 = dP * iCc * nr_rcp(rho * beta);
  const double temp2 = U_p * iS * dUn;
  const double temp3 = 0.5 * (1 - beta) * Un * temp * iS;
  const double temp4 = 0.5 * (1 - theda_p) * Un * U_p * iS;
  const double deltaU = (S - temp3 - beta * fabs(U) * insqr) * temp1 + temp2;
  const double deltaP = U_p * iS * dP + (C_p - fabs(U) * insqr + temp4) * rho * dUn;
  const double aU = fabs(Un);
  const double Fav1 = aU * dU1 + deltaU * rho;
  const double Fav2 = aU * dU2 + deltaU * rho * u + deltaP * NX;
  const double Fav3 = aU * dU3 + deltaU * rho * v + deltaP * NY;
  const double Fav4 = aU * dU4 + deltaU * rho * w + deltaP * NZ;
  const double Fav5 = aU * dU5 + deltaU * rho * H + deltaP * Un;
  const double h = 0.5 * iJf;
  F[0] = ((_rho * iU + rho_ * U_) - Fav1 * sq) * h;
  F[1] = ((_rho * _u * iU + rho_ * u_ * U_ + mx * (iP + P_)) - Fav2 * sq) * h;
  F[2] = ((_rho * _v * iU + rho_ * v_ * U_ + my * (iP + P_)) - Fav3 * sq) * h;
  F[3] = ((_rho * _w * iU + rho_ * w_ * U_ + mz * (iP + P_)) - Fav4 * sq) * h;
  F[4] = ((iU * (3.5 * iP + 0.5 * _rho * _VV) + U_ * (3.5 * P_ + 0.5 * rho_ * VV_)) - Fav5 * sq) * h;
  Fav3o = Fav3;
  ppo = iP + P_;
}

// ------------------------------------------------ dual-time primitives
// Primitive state of one cell as Dual_time_stepping.cpp:759-769 forms it.
template <typename T>
struct CPrim {
  T rho, u, v, w, VV, P, C, Tt, H, beta;
};

// reciprocal in the arithmetic type: the Newton-refined one in FP64
template <typename T>
__device__ __forceinline__ T recip(T a);
template <>
__device__ __forceinline__ double recip<double>(double a) { return nr_rcp(a); }
template <>
__device__ __forceinline__ float recip<float>(float a) { return 1.0f / a; }

template <typename T>
__device__ __forceinline__ CPrim<T> cprim(T q1, T q2, T q3, T q4, T q5, T J, T e) {
  CPrim<T> r;
  const T K = (T)KG;
  // divisions by one denominator as one reciprocal and products
  const T iq1 = recip<T>(q1);
  r.rho = q1 * J;
  r.u = q2 * iq1;
  r.v = q3 * iq1;
  r.w = q4 * iq1;
  r.VV = r.u * r.u + r.v * r.v + r.w * r.w;
  r.P = (q5 * J - (T)0.5 * r.rho * r.VV) * (K - 1);
  const T irho = recip<T>(r.rho);
  r.C = K * r.P * irho;
  r.Tt = r.P * irho;
  r.H = (T)0.5 * r.VV + r.C * (T)(1.0 / (KG - 1));
  const T th = r.VV * recip<T>(r.C);
  r.beta = th > e ? th : e;
  return r;
}

// Own LU-SGS diagonal of one cell, Dual_time_stepping.cpp:853-895.
template <typename T>
struct Diag {
  T d11, d22, d51;
};

template <typename T>
__device__ __forceinline__ Diag<T> diag(const CPrim<T> &q, const T mm[9], T dxi, T det, T dzt, T deltaT) {
  const T K = (T)KG;
  T beta = q.beta, C = q.C;
  T U = mm[0] * q.u + mm[1] * q.v + mm[2] * q.w;
  T V = mm[3] * q.u + mm[4] * q.v + mm[5] * q.w;
  T W = mm[6] * q.u + mm[7] * q.v + mm[8] * q.w;
  T Sx = sqrt(U * U * (beta - 1) * (beta - 1) + 4 * beta * C * (mm[0] * mm[0] + mm[1] * mm[1] + mm[2] * mm[2]));
  T Sy = sqrt(V * V * (beta - 1) * (beta - 1) + 4 * beta * C * (mm[3] * mm[3] + mm[4] * mm[4] + mm[5] * mm[5]));
  T Sz = sqrt(W * W * (beta - 1) * (beta - 1) + 4 * beta * C * (mm[6] * mm[6] + mm[7] * mm[7] + mm[8] * mm[8]));
  T lambdaX = ((beta + 1) * fabs(U) + Sx) / 2;
  T lambdaY = ((beta + 1) * fabs(V) + Sy) / 2;
  T lambdaZ = ((beta + 1) * fabs(W) + Sz) / 2;
  T lambda = lambdaX / dxi + lambdaY / det + lambdaZ / dzt;
  Diag<T> d;
  d.d11 = 2 * deltaT / (3 * beta + 2 * lambda * deltaT);
  d.d22 = 2 * deltaT / (3 + 2 * lambda * deltaT);
  T temp1 = 6 * (K - 1) * (beta - 1) * deltaT;
  T temp2 = K * (3 + 2 * lambda * deltaT) * (3 * beta + 2 * lambda * deltaT) * q.rho;
  d.d51 = -temp1 / temp2;
  return d;
}

// Split Jacobian of a neighbour in one direction: A+ entries of
// Dual_time_stepping.cpp:1054-1072 (B+ :1103-1121, C+ :1152-1170) and the
// A- diagonals of :1405-1409.  `xdir` selects the x product order of row 5.
template <typename T>
struct Split {
  T p11, p12, p13, p14, p21, p22, p31, p41, p51, p52, p53, p54, m11, m22;
};

template <typename T>
__device__ __forceinline__ Split<T> split(const CPrim<T> &q, T mx, T my, T mz, bool xdir) {
  const T K = (T)KG;
  T beta = q.beta, U = mx * q.u + my * q.v + mz * q.w;
  T Sx = sqrt(U * U * (beta - 1) * (beta - 1) + 4 * beta * q.C * (mx * mx + my * my + mz * mz));
  T lambdaX = ((beta + 1) * fabs(U) + Sx) / 2;
  T dd = fabs(lambdaX);
  Split<T> a;
  a.p11 = (T)0.5 * (beta * U + dd);
  a.p12 = (T)0.5 * q.P * K * beta * mx;
  a.p13 = (T)0.5 * q.P * K * beta * my;
  a.p14 = (T)0.5 * q.P * K * beta * mz;
  a.p21 = (T)0.5 * mx / q.rho;
  a.p22 = (T)0.5 * (U + dd);
  a.p31 = (T)0.5 * my / q.rho;
  a.p41 = (T)0.5 * mz / q.rho;
  a.p51 = (T)0.5 * U * (K - 1) * (beta - 1) / q.rho / K;
  if (xdir) {
    a.p52 = (T)0.5 * mx * beta * q.Tt * (K - 1);
    a.p53 = (T)0.5 * my * beta * q.Tt * (K - 1);
    a.p54 = (T)0.5 * mz * beta * q.Tt * (K - 1);
  } else {
    a.p52 = (T)0.5 * beta * q.Tt * (K - 1) * mx;
    a.p53 = (T)0.5 * beta * q.Tt * (K - 1) * my;
    a.p54 = (T)0.5 * beta * q.Tt * (K - 1) * mz;
  }
  a.m11 = (T)0.5 * (beta * U - dd);
  a.m22 = (T)0.5 * (U - dd);
  return a;
}

// Lower-triangular contribution of one upwind neighbour to LL1..LL5,
// the parenthesised terms of Dual_time_stepping.cpp:1172-1232.
template <typename T>
__device__ __forceinline__ void lower_terms(const Split<T> &A, const T n[5], T o[5]) {
  o[0] = -A.p11 * n[0] - A.p12 * n[1] - A.p13 * n[2] - A.p14 * n[3];
  o[1] = -A.p21 * n[0] - A.p22 * n[1];
  o[2] = -A.p31 * n[0] - A.p22 * n[2];
  o[3] = -A.p41 * n[0] - A.p22 * n[3];
  o[4] = -A.p51 * n[0] - A.p52 * n[1] - A.p53 * n[2] - A.p54 * n[3] - A.p22 * n[4];
}
// Upper-triangular contribution, Dual_time_stepping.cpp:1529-1590.
template <typename T>
__device__ __forceinline__ void upper_terms(const Split<T> &A, const T n[5], T o[5]) {
  o[0] = +A.m11 * n[0] + A.p12 * n[1] + A.p13 * n[2] + A.p14 * n[3];
  o[1] = +A.p21 * n[0] + A.m22 * n[1];
  o[2] = +A.p31 * n[0] + A.m22 * n[2];
  o[3] = +A.p41 * n[0] + A.m22 * n[3];
  o[4] = +A.p51 * n[0] + A.p52 * n[1] + A.p53 * n[2] + A.p54 * n[3] + A.m22 * n[4];
}

// Sponge terms of Dual_time_stepping.cpp:554-664 at interior cell c (plane i)
// of an open slab, the reference's Residual1..5: zero outside the inlet
// layer (planes 3..nx_inlet+2) and the outlet layer (planes
// max(3, Nx-nx_outlet+2)..Nx+2; the outlet wins where they overlap).  The
// inlet profile uses the slab's first global index (:586), the outlet one the
// plane's (:644); the outlet target velocity targetU is d.scal[1].
__device__ __forceinline__ void sponge_terms(const Dev &d, int i, long long c, double out[5]) {
#pragma unroll
  for (int v = 0; v < 5; v++) out[v] = 0.0;
  if (!d.x_open) return;
  const int nxin = d.nx_inlet, nxout = d.nx_outlet;
  const bool outlet = nxout > 0 && i >= max(3, d.nx - nxout + 2);
  const bool inlet = !outlet && nxin > 0 && i <= nxin + 2;
  if (!inlet && !outlet) return;
  const double J = d.J[c], q1 = d.U_[0][c];
  const double rho = q1 * J, u = d.U_[1][c] / q1, v = d.U_[2][c] / q1, w = d.U_[3][c] / q1;
  const double VV = u * u + v * v + w * w;
  const double P = (d.U_[4][c] * J - 0.5 * rho * VV) * (KG - 1);
  const double C = KG * P / rho;
  const double th = VV / C, beta = th > d.e ? th : d.e;
  const double C_plan = 0.5 * sqrt(u * u * (beta - 1) * (beta - 1) + 4 * beta * C);
  double Us, Sig, t2 = 0, t5 = 0;
  if (inlet) {
    Us = pow((nxin - 0.5) / nxin, 3.0) * C_plan;
    Sig = 0.035 * Us / d.high;
  } else {
    Us = pow((i - 0.5 - ((d.nx + 1) - nxout)) / nxout, 3.0) * C_plan;
    Sig = 1.25 * Us / d.high;
    const double tU = d.scal[1];
    t2 = 1.1842 * tU;
    t5 = 0.5 * 1.1842 * tU * tU;
  }
  const long long b = c - d.di;
  const double Jb = d.J[b], idx = 1 / d.dxi;
  const double rhs[5] = {rho - 1.1842, rho * u - t2, rho * v, rho * w, d.U_[4][c] * J - 253250.0 - t5};
#pragma unroll
  for (int n = 0; n < 5; n++) out[n] = -Us * (d.U_[n][c] * J - d.U_[n][b] * Jb) * idx - Sig * rhs[n];
}

// Deterministic block reduction of five partial sums (warp shuffles, then
// one warp over the per-warp results); thread 0 writes out[0..4].  Requires
// blockDim.x a multiple of 32 and at most 1024.
__device__ __forceinline__ void block_sum5(double acc[5], double *out) {
  __shared__ double red[32][5];
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int v = 0; v < 5; v++)
    for (int o = 16; o > 0; o >>= 1) acc[v] += __shfl_down_sync(0xffffffffu, acc[v], o);
  if (lane == 0)
    for (int v = 0; v < 5; v++) red[warp][v] = acc[v];
  __syncthreads();
  if (warp == 0) {
    double a[5];
    for (int v = 0; v < 5; v++) a[v] = lane < nw ? red[lane][v] : 0.0;
    for (int v = 0; v < 5; v++)
      for (int o = 16; o > 0; o >>= 1) a[v] += __shfl_down_sync(0xffffffffu, a[v], o);
    if (lane == 0)
      for (int v = 0; v < 5; v++) out[v] = a[v];
  }
}

// ---------------------------------------------------------------------------
// Coefficients of the LU-SGS sweeps with each division by a repeated divisor
// replaced by one reciprocal and multiplications (the reference divides every
// time; results differ from it by rounding only).  Used by the wavefront
// sweeps, where these quantities are formed once per cell and pass.
template <typename T>
struct SweepCoef {
  T d11, d22, d51;           // own diagonal, Dual_time_stepping.cpp:887-895
  Split<T> A[3];             // split Jacobians in x, y, z (A+ entries and A- diagonals)
  T rho, u, v, w, P, Tt;     // primitive state (for the update)
};

template <typename T>
__device__ __forceinline__ Split<T> split_fast(T beta, T C, T P, T Tt, T rrho, T u, T v, T w, T mx, T my, T mz,
                                               bool xdir, T &lam) {
  const T K = (T)KG;
  Split<T> a;
  T U = mx * u + my * v + mz * w;
  T S = sqrt(U * U * (beta - 1) * (beta - 1) + 4 * beta * C * (mx * mx + my * my + mz * mz));
  T lambdaX = ((beta + 1) * fabs(U) + S) * (T)0.5;
  lam = lambdaX;
  T dd = fabs(lambdaX);
  T hPKb = (T)0.5 * P * K * beta;
  a.p11 = (T)0.5 * (beta * U + dd);
  a.p12 = hPKb * mx;
  a.p13 = hPKb * my;
  a.p14 = hPKb * mz;
  T hr = (T)0.5 * rrho;
  a.p21 = hr * mx;
  a.p22 = (T)0.5 * (U + dd);
  a.p31 = hr * my;
  a.p41 = hr * mz;
  a.p51 = (T)0.5 * U * (K - 1) * (beta - 1) * rrho * (T)(1.0 / KG);
  T hbT = xdir ? (T)0.5 * beta * Tt * (K - 1) : (T)0.5 * beta * Tt * (K - 1);
  a.p52 = hbT * mx;
  a.p53 = hbT * my;
  a.p54 = hbT * mz;
  a.m11 = (T)0.5 * (beta * U - dd);
  a.m22 = (T)0.5 * (U - dd);
  return a;
}

// q1..q5 = Q/J of the cell, J its Jacobian, mm its nine metric terms;
// rdx = 1/deltaXI etc.
template <typename T>
__device__ __forceinline__ void sweep_coef(T q1, T q2, T q3, T q4, T q5, T J, const T mm[9], T e, T rdx, T rdy,
                                           T rdz, T dt, SweepCoef<T> &c) {
  const T K = (T)KG;
  T rq1 = (T)1 / q1;
  T rho = q1 * J;
  T u = q2 * rq1, v = q3 * rq1, w = q4 * rq1;
  T VV = u * u + v * v + w * w;
  T P = (q5 * J - (T)0.5 * rho * VV) * (K - 1);
  T rrho = (T)1 / rho;
  T C = K * P * rrho;
  T Tt = P * rrho;
  T th = VV / C;
  T beta = th > e ? th : e;
  T lx, ly, lz;
  c.A[0] = split_fast<T>(beta, C, P, Tt, rrho, u, v, w, mm[0], mm[1], mm[2], true, lx);
  c.A[1] = split_fast<T>(beta, C, P, Tt, rrho, u, v, w, mm[3], mm[4], mm[5], false, ly);
  c.A[2] = split_fast<T>(beta, C, P, Tt, rrho, u, v, w, mm[6], mm[7], mm[8], false, lz);
  T lambda = lx * rdx + ly * rdy + lz * rdz;
  T ld = 2 * lambda * dt;
  T a1 = (T)1 / (3 * beta + ld);
  T a2 = (T)1 / (3 + ld);
  c.d11 = 2 * dt * a1;
  c.d22 = 2 * dt * a2;
  c.d51 = -(6 * (K - 1) * (beta - 1) * dt) * (a1 * a2) * rrho * (T)(1.0 / KG);
  c.rho = rho; c.u = u; c.v = v; c.w = w; c.P = P; c.Tt = Tt;
}

// ---------------------------------------------------------------------------
// Compact per-cell record of everything the sweeps need, formed once per inner
// iteration by the residual kernel (the coefficients are the same in all four
// passes).  With the face metric (mx, my, mz) of a direction the split
// Jacobian entries are
//   p11 = (beta U + lam)/2    p12..14 = h (mx, my, mz)    p21,31,41 = hr (mx, my, mz)
//   p22 = (U + lam)/2         p51 = g U                   p52..54 = hbT (mx, my, mz)
//   m11 = (beta U - lam)/2    m22 = (U - lam)/2
// with U = mx u + my v + mz w the contravariant velocity, lam its spectral
// radius (Dual_time_stepping.cpp:1040-1072 and :1384-1409), h = P K beta / 2,
// hr = 1 / (2 rho), hbT = beta T (K-1) / 2, g = (K-1)(beta-1) / (2 rho K); the
// own diagonal d11, d22, d51 of :887-895.  The record keeps beta, h, hr, the
// three U and lam, d11 and d22 (11 words); hbT = 2 h hr (K-1)/K,
// g = (beta-1) hr (K-1)/K and d51 = -3 g d11 d22 / dt are formed from them
// where they are used (a few products, off the wavefront's dependency
// chain), so that a cell's record and MR are 16 words.
constexpr int REC_N = 11;
enum { R_BETA = 0, R_H, R_HR, R_UX, R_UY, R_UZ, R_LX, R_LY, R_LZ, R_D11, R_D22 };

template <typename T>
__device__ __forceinline__ T rec_hbt(const T r[REC_N]) {
  return r[R_H] * r[R_HR] * (T)(2.0 * (KG - 1) / KG);
}
template <typename T>
__device__ __forceinline__ T rec_g(const T r[REC_N]) {
  return (r[R_BETA] - 1) * r[R_HR] * (T)((KG - 1) / KG);
}
// rdt = 1 / dt
template <typename T>
__device__ __forceinline__ T rec_d51(const T r[REC_N], T rdt) {
  return (T)-3 * rec_g<T>(r) * r[R_D11] * r[R_D22] * rdt;
}

__device__ __forceinline__ void make_record(double q1, double q2, double q3, double q4, double q5, double J,
                                            const double mm[9], double e, double rdx, double rdy, double rdz,
                                            double dt, double r[REC_N]) {
  const double K = KG;
  double rq1 = nr_rcp(q1);
  double rho = q1 * J;
  double u = q2 * rq1, v = q3 * rq1, w = q4 * rq1;
  double VV = u * u + v * v + w * w;
  double P = (q5 * J - 0.5 * rho * VV) * (K - 1);
  double rrho = nr_rcp(rho);
  double C = K * P * rrho;
  double th = VV * nr_rcp(C);
  double beta = th > e ? th : e;
  double lam[3], U[3];
#pragma unroll
  for (int dd = 0; dd < 3; dd++) {
    double mx = mm[3 * dd], my = mm[3 * dd + 1], mz = mm[3 * dd + 2];
    U[dd] = mx * u + my * v + mz * w;
    double S = nr_sqrt(U[dd] * U[dd] * (beta - 1) * (beta - 1) + 4 * beta * C * (mx * mx + my * my + mz * mz));
    lam[dd] = ((beta + 1) * fabs(U[dd]) + S) * 0.5;
  }
  double lambda = lam[0] * rdx + lam[1] * rdy + lam[2] * rdz;
  double ld = 2 * lambda * dt;
  double a1 = nr_rcp(3 * beta + ld);
  double a2 = nr_rcp(3 + ld);
  r[R_BETA] = beta;
  r[R_H] = 0.5 * P * K * beta;
  r[R_HR] = 0.5 * rrho;
  r[R_UX] = U[0]; r[R_UY] = U[1]; r[R_UZ] = U[2];
  r[R_LX] = lam[0]; r[R_LY] = lam[1]; r[R_LZ] = lam[2];
  r[R_D11] = 2 * dt * a1;
  r[R_D22] = 2 * dt * a2;
}

// split Jacobian entries of one direction from a record
template <typename T>
__device__ __forceinline__ Split<T> split_from_record(const T r[REC_N], int dir, T mx, T my, T mz) {
  const T U = r[R_UX + dir], lam = r[R_LX + dir], beta = r[R_BETA];
  Split<T> a;
  a.p11 = (T)0.5 * (beta * U + lam);
  a.p12 = r[R_H] * mx;
  a.p13 = r[R_H] * my;
  a.p14 = r[R_H] * mz;
  a.p21 = r[R_HR] * mx;
  a.p31 = r[R_HR] * my;
  a.p41 = r[R_HR] * mz;
  a.p22 = (T)0.5 * (U + lam);
  const T hbt = rec_hbt<T>(r);
  a.p51 = rec_g<T>(r) * U;
  a.p52 = hbt * mx;
  a.p53 = hbt * my;
  a.p54 = hbt * mz;
  a.m11 = (T)0.5 * (beta * U - lam);
  a.m22 = (T)0.5 * (U - lam);
  return a;
}

}  // namespace cgli
