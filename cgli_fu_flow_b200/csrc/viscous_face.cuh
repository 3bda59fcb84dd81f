// Viscous face fluxes (x-momentum, y-momentum, z-momentum, energy) of one
// face, Viscous_terms.cpp:397-861.  Included by the kernel translation units
// after the definition of a primitive type `VP` {U, V, W, T} (velocity and
// temperature of one cell, Viscous_terms.cpp:260-394).  The arguments name
// the stencil cells relative to the cell (i,j,k) that owns the face at its
// lower side: im = (i-1,j,k), jp = (i,j+1,k), iJ = (i-1,j+1,k), and so on.
#pragma once

namespace cgli {

struct MetricProducts {
  double a1, a2, a3, a4, a5, a6, a7, b1, b2, b3, b4, b5, b6, b7, c1, c2, c3, c4, c5, c6, c7;
  double d1, d2, d3, d4, d5, d6, d7, d8, d9, d10, e1, e2, e3, e4, e5, e6, e7, e8, e9, e10;
  double f1, f2, f3, f4, f5, f6, f7, f8, f9, f10;
};

// a1..f10 of Viscous_terms.cpp:464-519 from one face's nine metric terms
__device__ __forceinline__ MetricProducts metric_products(const double x[9]) {
  const double xix = x[0], xiy = x[1], xiz = x[2], etx = x[3], ety = x[4], etz = x[5], ztx = x[6], zty = x[7], ztz = x[8];
  MetricProducts q;
  q.a1 = (4. / 3) * xix * xix + xiy * xiy + xiz * xiz;
  q.a2 = xix * xix + (4. / 3) * xiy * xiy + xiz * xiz;
  q.a3 = xix * xix + xiy * xiy + (4. / 3) * xiz * xiz;
  q.a4 = xix * xix + xiy * xiy + xiz * xiz;
  q.a5 = (1. / 3) * xix * xiy;
  q.a6 = (1. / 3) * xiy * xiz;
  q.a7 = (1. / 3) * xix * xiz;
  q.b1 = (4. / 3) * etx * etx + ety * ety + etz * etz;
  q.b2 = etx * etx + (4. / 3) * ety * ety + etz * etz;
  q.b3 = etx * etx + ety * ety + (4. / 3) * etz * etz;
  q.b4 = etx * etx + ety * ety + etz * etz;
  q.b5 = (1. / 3) * etx * ety;
  q.b6 = (1. / 3) * ety * etz;
  q.b7 = (1. / 3) * etx * etz;
  q.c1 = (4. / 3) * ztx * ztx + zty * zty + ztz * ztz;
  q.c2 = ztx * ztx + (4. / 3) * zty * zty + ztz * ztz;
  q.c3 = ztx * ztx + zty * zty + (4. / 3) * ztz * ztz;
  q.c4 = ztx * ztx + zty * zty + ztz * ztz;
  q.c5 = (1. / 3) * ztx * zty;
  q.c6 = (1. / 3) * zty * ztz;
  q.c7 = (1. / 3) * ztx * ztz;
  q.d1 = (4. / 3) * xix * etx + xiy * ety + xiz * etz;
  q.d2 = xix * etx + (4. / 3) * xiy * ety + xiz * etz;
  q.d3 = xix * etx + xiy * ety + (4. / 3) * xiz * etz;
  q.d4 = xix * etx + xiy * ety + xiz * etz;
  q.d5 = xix * ety - (2. / 3) * xiy * etx;
  q.d6 = xix * etz - (2. / 3) * xiz * etx;
  q.d7 = xiy * etx - (2. / 3) * xix * ety;
  q.d8 = xiy * etz - (2. / 3) * xiz * ety;
  q.d9 = xiz * etx - (2. / 3) * xix * etz;
  q.d10 = xiz * ety - (2. / 3) * xiy * etz;
  q.e1 = (4. / 3) * xix * ztx + xiy * zty + xiz * ztz;
  q.e2 = xix * ztx + (4. / 3) * xiy * zty + xiz * ztz;
  q.e3 = xix * ztx + xiy * zty + (4. / 3) * xiz * ztz;
  q.e4 = xix * ztx + xiy * zty + xiz * ztz;
  q.e5 = xix * zty - (2. / 3) * xiy * ztx;
  q.e6 = xix * ztz - (2. / 3) * xiz * ztx;
  q.e7 = xiy * ztx - (2. / 3) * xix * zty;
  q.e8 = xiy * ztz - (2. / 3) * xiz * zty;
  q.e9 = xiz * ztx - (2. / 3) * xix * ztz;
  q.e10 = xiz * zty - (2. / 3) * xiy * ztz;
  q.f1 = (4. / 3) * etx * ztx + ety * zty + etz * ztz;
  q.f2 = etx * ztx + (4. / 3) * ety * zty + etz * ztz;
  q.f3 = etx * ztx + ety * zty + (4. / 3) * etz * ztz;
  q.f4 = etx * ztx + ety * zty + etz * ztz;
  q.f5 = etx * zty - (2. / 3) * ety * ztx;
  q.f6 = etx * ztz - (2. / 3) * etz * ztx;
  q.f7 = ety * ztx - (2. / 3) * etx * zty;
  q.f8 = ety * ztz - (2. / 3) * etz * zty;
  q.f9 = etz * ztx - (2. / 3) * etx * ztz;
  q.f10 = etz * zty - (2. / 3) * ety * ztz;
  return q;
}

// Sutherland's law as Viscous_terms.cpp:527 writes it, with (T/Tref)^1.5
// evaluated as x*sqrt(x) (the same value to rounding, without pow) and the
// Newton-refined square root and reciprocal
__device__ __forceinline__ double sutherland_mu(double mu, double T) {
  const double x = T * (1.0 / 298.0592);
  return mu * (x * nr_sqrt(x)) * (298.0592 + 110.) * nr_rcp(T + 110.);
}

// x face i-1/2, Viscous_terms.cpp:399-546
template <typename P>
__device__ __forceinline__ void visc_face_x(double rdxi, double rdet, double rdzt, double mu, double ipr,
                                            const P &o, const P &im, const P &jp, const P &iJ, const P &jm,
                                            const P &ijm, const P &kp, const P &iK, const P &km, const P &ikm,
                                            const double mm[9], double iJf, double out[4]) {
  const double invXI = rdxi, inv4ET = 0.25 * rdet, inv4ZT = 0.25 * rdzt;
  const double CvK = CV * KG;
  double U = o.U, V = o.V, W = o.W, T = o.T;
  double du_dx = (U - im.U) * invXI, dv_dx = (V - im.V) * invXI, dw_dx = (W - im.W) * invXI;
  double du2_dx = (U * U - im.U * im.U) * invXI, dv2_dx = (V * V - im.V * im.V) * invXI,
         dw2_dx = (W * W - im.W * im.W) * invXI;
  double duv_dx = (U * V - im.U * im.V) * invXI, dvw_dx = (V * W - im.V * im.W) * invXI,
         duw_dx = (U * W - im.U * im.W) * invXI;
  double dT_dx = (T - im.T) * invXI;
  double du_dy = (jp.U + iJ.U - jm.U - ijm.U) * inv4ET, dv_dy = (jp.V + iJ.V - jm.V - ijm.V) * inv4ET,
         dw_dy = (jp.W + iJ.W - jm.W - ijm.W) * inv4ET;
  double du2_dy = (jp.U * jp.U + iJ.U * iJ.U - jm.U * jm.U - ijm.U * ijm.U) * inv4ET;
  double dv2_dy = (jp.V * jp.V + iJ.V * iJ.V - jm.V * jm.V - ijm.V * ijm.V) * inv4ET;
  double dw2_dy = (jp.W * jp.W + iJ.W * iJ.W - jm.W * jm.W - ijm.W * ijm.W) * inv4ET;
  double dT_dy = (jp.T + iJ.T - jm.T - ijm.T) * inv4ET;
  double du_dz = (kp.U + iK.U - km.U - ikm.U) * inv4ZT, dv_dz = (kp.V + iK.V - km.V - ikm.V) * inv4ZT,
         dw_dz = (kp.W + iK.W - km.W - ikm.W) * inv4ZT;
  double du2_dz = (kp.U * kp.U + iK.U * iK.U - km.U * km.U - ikm.U * ikm.U) * inv4ZT;
  double dv2_dz = (kp.V * kp.V + iK.V * iK.V - km.V * km.V - ikm.V * ikm.V) * inv4ZT;
  double dw2_dz = (kp.W * kp.W + iK.W * iK.W - km.W * km.W - ikm.W * ikm.W) * inv4ZT;
  double dT_dz = (kp.T + iK.T - km.T - ikm.T) * inv4ZT;
  MetricProducts q = metric_products(mm);
  double Ux = 0.5 * (U + im.U), Vx = 0.5 * (V + im.V), Wx = 0.5 * (W + im.W), Tx = 0.5 * (T + im.T);
  double mu_E = sutherland_mu(mu, Tx);
  out[0] = mu_E * (q.a1 * du_dx + q.a5 * dv_dx + q.a7 * dw_dx + q.d1 * du_dy + q.d7 * dv_dy + q.d9 * dw_dy +
                   q.e1 * du_dz + q.e7 * dv_dz + q.e9 * dw_dz) * iJf;
  out[1] = mu_E * (q.a5 * du_dx + q.a2 * dv_dx + q.a6 * dw_dx + q.d5 * du_dy + q.d2 * dv_dy + q.d10 * dw_dy +
                   q.e5 * du_dz + q.e2 * dv_dz + q.e10 * dw_dz) * iJf;
  out[2] = mu_E * (q.a7 * du_dx + q.a6 * dv_dx + q.a3 * dw_dx + q.d6 * du_dy + q.d8 * dv_dy + q.d3 * dw_dy +
                   q.e6 * du_dz + q.e8 * dv_dz + q.e3 * dw_dz) * iJf;
  out[3] = mu_E * (0.5 * q.a1 * du2_dx + 0.5 * q.a2 * dv2_dx + 0.5 * q.a3 * dw2_dx + q.a5 * duv_dx + q.a6 * dvw_dx +
                   q.a7 * duw_dx + CvK * q.a4 * dT_dx * ipr + 0.5 * q.d1 * du2_dy + 0.5 * q.d2 * dv2_dy +
                   0.5 * q.d3 * dw2_dy + q.d5 * Vx * du_dy + q.d6 * Wx * du_dy + q.d7 * Ux * dv_dy +
                   q.d8 * Wx * dv_dy + q.d9 * Ux * dw_dy + q.d10 * Vx * dw_dy + CvK * q.d4 * dT_dy * ipr +
                   0.5 * q.e1 * du2_dz + 0.5 * q.e2 * dv2_dz + 0.5 * q.e3 * dw2_dz + q.e5 * Vx * du_dz +
                   q.e6 * Wx * du_dz + q.e7 * Ux * dv_dz + q.e8 * Wx * dv_dz + q.e9 * Ux * dw_dz +
                   q.e10 * Vx * dw_dz + CvK * q.e4 * dT_dz * ipr) * iJf;
}

// y face j-1/2, Viscous_terms.cpp:549-700
template <typename P>
__device__ __forceinline__ void visc_face_y(double rdxi, double rdet, double rdzt, double mu, double ipr,
                                            const P &o, const P &jm, const P &ip, const P &jI, const P &im,
                                            const P &ijm, const P &kp, const P &jK, const P &km, const P &jkm,
                                            const double mm[9], double iJf, double out[4]) {
  const double inv4XI = 0.25 * rdxi, invET = rdet, inv4ZT = 0.25 * rdzt;
  const double CvK = CV * KG;
  double U = o.U, V = o.V, W = o.W, T = o.T;
  double du_dx = (ip.U + jI.U - im.U - ijm.U) * inv4XI, dv_dx = (ip.V + jI.V - im.V - ijm.V) * inv4XI,
         dw_dx = (ip.W + jI.W - im.W - ijm.W) * inv4XI;
  double du2_dx = (ip.U * ip.U + jI.U * jI.U - im.U * im.U - ijm.U * ijm.U) * inv4XI;
  double dv2_dx = (ip.V * ip.V + jI.V * jI.V - im.V * im.V - ijm.V * ijm.V) * inv4XI;
  double dw2_dx = (ip.W * ip.W + jI.W * jI.W - im.W * im.W - ijm.W * ijm.W) * inv4XI;
  double dT_dx = (ip.T + jI.T - im.T - ijm.T) * inv4XI;
  double du_dy = (U - jm.U) * invET, dv_dy = (V - jm.V) * invET, dw_dy = (W - jm.W) * invET;
  double du2_dy = (U * U - jm.U * jm.U) * invET, dv2_dy = (V * V - jm.V * jm.V) * invET,
         dw2_dy = (W * W - jm.W * jm.W) * invET;
  double duv_dy = (U * V - jm.U * jm.V) * invET, dvw_dy = (V * W - jm.V * jm.W) * invET,
         duw_dy = (U * W - jm.U * jm.W) * invET;
  double dT_dy = (T - jm.T) * invET;
  double du_dz = (kp.U + jK.U - km.U - jkm.U) * inv4ZT, dv_dz = (kp.V + jK.V - km.V - jkm.V) * inv4ZT,
         dw_dz = (kp.W + jK.W - km.W - jkm.W) * inv4ZT;
  double du2_dz = (kp.U * kp.U + jK.U * jK.U - km.U * km.U - jkm.U * jkm.U) * inv4ZT;
  double dv2_dz = (kp.V * kp.V + jK.V * jK.V - km.V * km.V - jkm.V * jkm.V) * inv4ZT;
  double dw2_dz = (kp.W * kp.W + jK.W * jK.W - km.W * km.W - jkm.W * jkm.W) * inv4ZT;
  double dT_dz = (kp.T + jK.T - km.T - jkm.T) * inv4ZT;
  MetricProducts q = metric_products(mm);
  double Uy = 0.5 * (U + jm.U), Vy = 0.5 * (V + jm.V), Wy = 0.5 * (W + jm.W), Ty = 0.5 * (T + jm.T);
  double mu_E = sutherland_mu(mu, Ty);
  out[0] = mu_E * (q.d1 * du_dx + q.d5 * dv_dx + q.d6 * dw_dx + q.b1 * du_dy + q.b5 * dv_dy + q.b7 * dw_dy +
                   q.f1 * du_dz + q.f7 * dv_dz + q.f9 * dw_dz) * iJf;
  out[1] = mu_E * (q.d7 * du_dx + q.d2 * dv_dx + q.d8 * dw_dx + q.b5 * du_dy + q.b2 * dv_dy + q.b6 * dw_dy +
                   q.f5 * du_dz + q.f2 * dv_dz + q.f10 * dw_dz) * iJf;
  out[2] = mu_E * (q.d9 * du_dx + q.d10 * dv_dx + q.d3 * dw_dx + q.b7 * du_dy + q.b6 * dv_dy + q.b3 * dw_dy +
                   q.f6 * du_dz + q.f8 * dv_dz + q.f3 * dw_dz) * iJf;
  out[3] = mu_E * (0.5 * q.b1 * du2_dy + 0.5 * q.b2 * dv2_dy + 0.5 * q.b3 * dw2_dy + q.b5 * duv_dy + q.b6 * dvw_dy +
                   q.b7 * duw_dy + CvK * q.b4 * dT_dy * ipr + 0.5 * q.d1 * du2_dx + 0.5 * q.d2 * dv2_dx +
                   0.5 * q.d3 * dw2_dx + q.d5 * Uy * dv_dx + q.d6 * Uy * dw_dx + q.d7 * Vy * du_dx +
                   q.d8 * Vy * dw_dx + q.d9 * Wy * du_dx + q.d10 * Wy * dv_dx + CvK * q.d4 * dT_dx * ipr +
                   0.5 * q.f1 * du2_dz + 0.5 * q.f2 * dv2_dz + 0.5 * q.f3 * dw2_dz + q.f5 * Vy * du_dz +
                   q.f6 * Wy * du_dz + q.f7 * Uy * dv_dz + q.f8 * Wy * dv_dz + q.f9 * Uy * dw_dz +
                   q.f10 * Vy * dw_dz + CvK * q.f4 * dT_dz * ipr) * iJf;
}

// z face k-1/2, Viscous_terms.cpp:714-861, with the typo of :744-746 that
// pairs u at (i,j+1,k-1) with v, w at (i-1,j+1,k) (argument iJ)
template <typename P>
__device__ __forceinline__ void visc_face_z(double rdxi, double rdet, double rdzt, double mu, double ipr,
                                            const P &o, const P &km, const P &ip, const P &kI, const P &im,
                                            const P &ikm, const P &jp, const P &kJ, const P &jm, const P &jkm,
                                            const P &iJ, const double mm[9], double iJf, double out[4]) {
  const double inv4XI = 0.25 * rdxi, inv4ET = 0.25 * rdet, invZT = rdzt;
  const double CvK = CV * KG;
  double U = o.U, V = o.V, W = o.W, T = o.T;
  double du_dx = (ip.U + kI.U - im.U - ikm.U) * inv4XI, dv_dx = (ip.V + kI.V - im.V - ikm.V) * inv4XI,
         dw_dx = (ip.W + kI.W - im.W - ikm.W) * inv4XI;
  double du2_dx = (ip.U * ip.U + kI.U * kI.U - im.U * im.U - ikm.U * ikm.U) * inv4XI;
  double dv2_dx = (ip.V * ip.V + kI.V * kI.V - im.V * im.V - ikm.V * ikm.V) * inv4XI;
  double dw2_dx = (ip.W * ip.W + kI.W * kI.W - im.W * im.W - ikm.W * ikm.W) * inv4XI;
  double dT_dx = (ip.T + kI.T - im.T - ikm.T) * inv4XI;
  double du_dy = (jp.U + kJ.U - jm.U - jkm.U) * inv4ET, dv_dy = (jp.V + kJ.V - jm.V - jkm.V) * inv4ET,
         dw_dy = (jp.W + kJ.W - jm.W - jkm.W) * inv4ET;
  double du2_dy = (jp.U * jp.U + kJ.U * kJ.U - jm.U * jm.U - jkm.U * jkm.U) * inv4ET;
  double dv2_dy = (jp.V * jp.V + kJ.V * kJ.V - jm.V * jm.V - jkm.V * jkm.V) * inv4ET;
  double dw2_dy = (jp.W * jp.W + kJ.W * kJ.W - jm.W * jm.W - jkm.W * jkm.W) * inv4ET;
  double dT_dy = (jp.T + kJ.T - jm.T - jkm.T) * inv4ET;
  double du_dz = (U - km.U) * invZT, dv_dz = (V - km.V) * invZT, dw_dz = (W - km.W) * invZT;
  double du2_dz = (U * U - km.U * km.U) * invZT, dv2_dz = (V * V - km.V * km.V) * invZT,
         dw2_dz = (W * W - km.W * km.W) * invZT;
  double duv_dz = (U * V - km.U * km.V) * invZT, dvw_dz = (V * W - km.V * km.W) * invZT,
         duw_dz = (U * W - km.U * km.W) * invZT;
  double dT_dz = (T - km.T) * invZT;
  (void)iJ;
  MetricProducts q = metric_products(mm);
  double Uz = 0.5 * (U + km.U), Vz = 0.5 * (V + km.V), Wz = 0.5 * (W + km.W), Tz = 0.5 * (T + km.T);
  double mu_E = sutherland_mu(mu, Tz);
  out[0] = mu_E * (q.e1 * du_dx + q.e5 * dv_dx + q.e6 * dw_dx + q.f1 * du_dy + q.f5 * dv_dy + q.f6 * dw_dy +
                   q.c1 * du_dz + q.c5 * dv_dz + q.c7 * dw_dz) * iJf;
  out[1] = mu_E * (q.e7 * du_dx + q.e2 * dv_dx + q.e8 * dw_dx + q.f7 * du_dy + q.f2 * dv_dy + q.f8 * dw_dy +
                   q.c5 * du_dz + q.c2 * dv_dz + q.c6 * dw_dz) * iJf;
  out[2] = mu_E * (q.e9 * du_dx + q.e10 * dv_dx + q.e3 * dw_dx + q.f9 * du_dy + q.f10 * dv_dy + q.f3 * dw_dy +
                   q.c7 * du_dz + q.c6 * dv_dz + q.c3 * dw_dz) * iJf;
  out[3] = mu_E * (0.5 * q.c1 * du2_dz + 0.5 * q.c2 * dv2_dz + 0.5 * q.c3 * dw2_dz + q.c5 * duv_dz + q.c6 * dvw_dz +
                   q.c7 * duw_dz + CvK * q.c4 * dT_dz * ipr + 0.5 * q.e1 * du2_dx + 0.5 * q.e2 * dv2_dx +
                   0.5 * q.e3 * dw2_dx + q.e5 * Uz * dv_dx + q.e6 * Uz * dw_dx + q.e7 * Vz * du_dx +
                   q.e8 * Vz * dw_dx + q.e9 * Wz * du_dx + q.e10 * Wz * dv_dx + CvK * q.e4 * dT_dx * ipr +
                   0.5 * q.f1 * du2_dy + 0.5 * q.f2 * dv2_dy + 0.5 * q.f3 * dw2_dy + q.f5 * Uz * dv_dy +
                   q.f6 * Uz * dw_dy + q.f7 * Vz * du_dy + q.f8 * Vz * dw_dy + q.f9 * Wz * du_dy +
                   q.f10 * Wz * dv_dy + CvK * q.f4 * dT_dy * ipr) * iJf;
}

// ----------------------------------------------------------------------------
// The same three face fluxes on a face whose metrics have the channel's form
// xi = (1,0,0), eta = (0,e,0), zeta = (0,0,1) (checked on the device over
// every face before these are used).  Then a1..f10 are a1 = 4/3, a2 = a3 =
// a4 = 1; b1 = b3 = b4 = e^2, b2 = 4/3 e^2; c1 = c2 = c4 = 1, c3 = 4/3;
// d5 = e, d7 = -2/3 e; e6 = 1, e9 = -2/3; f8 = e, f10 = -2/3 e; and every
// other product is exactly zero, so each flux keeps only its nonzero terms
// (the reference's sums with the zero terms dropped: the same value to
// rounding) and only the differences those terms use are formed.

// x face i-1/2 (Viscous_terms.cpp:399-546 with the channel's metrics)
template <typename P>
__device__ __forceinline__ void visc_face_x_channel(double rdxi, double rdet, double rdzt, double mu, double ipr,
                                                    double e, const P &o, const P &im, const P &jp, const P &iJ,
                                                    const P &jm, const P &ijm, const P &kp, const P &iK, const P &km,
                                                    const P &ikm, double iJf, double out[4]) {
  const double invXI = rdxi, inv4ET = 0.25 * rdet, inv4ZT = 0.25 * rdzt;
  const double CvK = CV * KG;
  const double U = o.U, V = o.V, W = o.W, T = o.T;
  const double du_dx = (U - im.U) * invXI, dv_dx = (V - im.V) * invXI, dw_dx = (W - im.W) * invXI;
  const double du2_dx = (U * U - im.U * im.U) * invXI, dv2_dx = (V * V - im.V * im.V) * invXI,
               dw2_dx = (W * W - im.W * im.W) * invXI;
  const double dT_dx = (T - im.T) * invXI;
  const double du_dy = (jp.U + iJ.U - jm.U - ijm.U) * inv4ET, dv_dy = (jp.V + iJ.V - jm.V - ijm.V) * inv4ET;
  const double du_dz = (kp.U + iK.U - km.U - ikm.U) * inv4ZT, dw_dz = (kp.W + iK.W - km.W - ikm.W) * inv4ZT;
  const double Ux = 0.5 * (U + im.U), Vx = 0.5 * (V + im.V), Wx = 0.5 * (W + im.W), Tx = 0.5 * (T + im.T);
  const double m = sutherland_mu(mu, Tx) * iJf;
  out[0] = m * ((4. / 3) * du_dx - (2. / 3) * e * dv_dy - (2. / 3) * dw_dz);
  out[1] = m * (dv_dx + e * du_dy);
  out[2] = m * (dw_dx + du_dz);
  out[3] = m * ((2. / 3) * du2_dx + 0.5 * dv2_dx + 0.5 * dw2_dx + CvK * dT_dx * ipr + e * Vx * du_dy -
                (2. / 3) * e * Ux * dv_dy + Wx * du_dz - (2. / 3) * Ux * dw_dz);
}

// y face j-1/2 (Viscous_terms.cpp:549-700 with the channel's metrics)
template <typename P>
__device__ __forceinline__ void visc_face_y_channel(double rdxi, double rdet, double rdzt, double mu, double ipr,
                                                    double e, const P &o, const P &jm, const P &ip, const P &jI,
                                                    const P &im, const P &ijm, const P &kp, const P &jK, const P &km,
                                                    const P &jkm, double iJf, double out[4]) {
  const double inv4XI = 0.25 * rdxi, invET = rdet, inv4ZT = 0.25 * rdzt;
  const double CvK = CV * KG;
  const double U = o.U, V = o.V, W = o.W, T = o.T;
  const double du_dx = (ip.U + jI.U - im.U - ijm.U) * inv4XI, dv_dx = (ip.V + jI.V - im.V - ijm.V) * inv4XI;
  const double du_dy = (U - jm.U) * invET, dv_dy = (V - jm.V) * invET, dw_dy = (W - jm.W) * invET;
  const double du2_dy = (U * U - jm.U * jm.U) * invET, dv2_dy = (V * V - jm.V * jm.V) * invET,
               dw2_dy = (W * W - jm.W * jm.W) * invET;
  const double dT_dy = (T - jm.T) * invET;
  const double dv_dz = (kp.V + jK.V - km.V - jkm.V) * inv4ZT, dw_dz = (kp.W + jK.W - km.W - jkm.W) * inv4ZT;
  const double Uy = 0.5 * (U + jm.U), Vy = 0.5 * (V + jm.V), Wy = 0.5 * (W + jm.W), Ty = 0.5 * (T + jm.T);
  const double m = sutherland_mu(mu, Ty) * iJf, e2 = e * e;
  out[0] = m * (e * dv_dx + e2 * du_dy);
  out[1] = m * (-(2. / 3) * e * du_dx + (4. / 3) * e2 * dv_dy - (2. / 3) * e * dw_dz);
  out[2] = m * (e2 * dw_dy + e * dv_dz);
  out[3] = m * (0.5 * e2 * du2_dy + (2. / 3) * e2 * dv2_dy + 0.5 * e2 * dw2_dy + CvK * e2 * dT_dy * ipr +
                e * Uy * dv_dx - (2. / 3) * e * Vy * du_dx + e * Wy * dv_dz - (2. / 3) * e * Vy * dw_dz);
}

// z face k-1/2 (Viscous_terms.cpp:714-861 with the channel's metrics; the
// typo of :744-746 only feeds terms whose products are zero here)
template <typename P>
__device__ __forceinline__ void visc_face_z_channel(double rdxi, double rdet, double rdzt, double mu, double ipr,
                                                    double e, const P &o, const P &km, const P &ip, const P &kI,
                                                    const P &im, const P &ikm, const P &jp, const P &kJ, const P &jm,
                                                    const P &jkm, double iJf, double out[4]) {
  const double inv4XI = 0.25 * rdxi, inv4ET = 0.25 * rdet, invZT = rdzt;
  const double CvK = CV * KG;
  const double U = o.U, V = o.V, W = o.W, T = o.T;
  const double du_dx = (ip.U + kI.U - im.U - ikm.U) * inv4XI, dw_dx = (ip.W + kI.W - im.W - ikm.W) * inv4XI;
  const double dv_dy = (jp.V + kJ.V - jm.V - jkm.V) * inv4ET, dw_dy = (jp.W + kJ.W - jm.W - jkm.W) * inv4ET;
  const double du_dz = (U - km.U) * invZT, dv_dz = (V - km.V) * invZT, dw_dz = (W - km.W) * invZT;
  const double du2_dz = (U * U - km.U * km.U) * invZT, dv2_dz = (V * V - km.V * km.V) * invZT,
               dw2_dz = (W * W - km.W * km.W) * invZT;
  const double dT_dz = (T - km.T) * invZT;
  const double Uz = 0.5 * (U + km.U), Vz = 0.5 * (V + km.V), Wz = 0.5 * (W + km.W), Tz = 0.5 * (T + km.T);
  const double m = sutherland_mu(mu, Tz) * iJf;
  out[0] = m * (dw_dx + du_dz);
  out[1] = m * (e * dw_dy + dv_dz);
  out[2] = m * (-(2. / 3) * du_dx - (2. / 3) * e * dv_dy + (4. / 3) * dw_dz);
  out[3] = m * (0.5 * du2_dz + 0.5 * dv2_dz + (2. / 3) * dw2_dz + CvK * dT_dz * ipr + Uz * dw_dx -
                (2. / 3) * Wz * du_dx + e * Vz * dw_dy - (2. / 3) * e * Wz * dv_dy);
}

}  // namespace cgli
