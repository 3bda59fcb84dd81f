// Host-side set-up of the hot path: the analytic channel metrics and the
// hyperplane enumeration.  Both are computed once per run on the host.
#include <cmath>
#include <cstddef>
#include <vector>

#include "host_setup.h"

namespace cgli {

// The tanh wall-clustering mapping of Jacobian.cpp:76-90 evaluated at
// eta = (j - off) * det: d(eta)/dy and dy/d(eta), in the reference's
// statement order (1/cosh and 1./cosh of the face routines are the same value).
static inline void stretch(double high, double g, double det, int j, double off, double &etdy, double &ydet) {
  double temp = (0.5 * high) * (1 - 1. / tanh(g) * tanh(g * (1 - 2 * (j - off) * det)));
  double temp1 = (1 - temp / (0.5 * high)) * tanh(g);
  double temp2 = 1. / cosh(g * (1 - 2 * (j - off) * det));
  etdy = tanh(g) / (2 * (0.5 * high) * g * (1 - temp1 * temp1));
  ydet = high * g * 1. / tanh(g) * temp2 * temp2;
}

// Jacobian.cpp:61-243, Jacobian_u.cpp:59-101, Jacobian_v.cpp:79-151,
// Jacobian_w.cpp:61-106 for an interior slab (planes 0..Nx+5), or with
// x_open for a slab that is the first and the last rank (cell metrics on
// planes 3..Nx+2, then the end planes 2 and Nx+3 as copies of their
// neighbours over j, k = 1..Ny+2 / Nz+2, Jacobian.cpp:110-157, whose ztdx is
// copied three times so that ztdy, ztdz of the end planes stay zero; ghost
// rows on planes 2..Nx+3).  Unset entries stay zero.  The ghost-row copy
// statements of Jacobian.cpp:181-182, :193-194 and :224-237 assign ztdx of
// the neighbour to ztdy and ztdz; they are kept, so ghost rows carry
// ztdy = ztdz = 0.
void channel_metrics(int nx, int ny, int nz, double det, double high, double g, MetricSet &M, bool x_open) {
  const int X = nx + 6, Y = ny + 4, Z = nz + 4;
  const size_t n = (size_t)X * Y * Z;
  auto id = [&](int i, int j, int k) { return ((size_t)i * Y + j) * Z + k; };
  M.J.assign(n, 0.0);
  for (int v = 0; v < 9; v++) M.m[v].assign(n, 0.0);
  for (int d = 0; d < 3; d++) {
    M.Jf[d].assign(n, 0.0);
    for (int v = 0; v < 9; v++) M.mf[d][v].assign(n, 0.0);
  }
  const int ie = nx + 2, jn = ny + 1, kn = nz + 1, nyy = jn + 1, nzz = kn + 1;
  for (int j = 2; j <= jn; j++) {
    double etdy, ydet;
    stretch(high, g, det, j, 1.5, etdy, ydet);
    double J = 1. / (1 * ydet * 1);
    for (int i = x_open ? 3 : 0; i <= (x_open ? ie : ie + 3); i++)
      for (int k = 2; k <= kn; k++) {
        size_t c = id(i, j, k);
        M.m[0][c] = 1; M.m[4][c] = etdy; M.m[8][c] = 1;
        M.J[c] = J;
      }
  }
  if (x_open)
    for (int side = 0; side < 2; side++) {
      const int ig = side ? ie + 1 : 2, is = side ? ie : 3;
      for (int j = 1; j <= nyy; j++)
        for (int k = 1; k <= nzz; k++) {
          size_t gidx = id(ig, j, k), c = id(is, j, k);
          for (int v = 0; v < 7; v++) M.m[v][gidx] = M.m[v][c];
          M.J[gidx] = M.J[c];
        }
    }
  const int ig0 = x_open ? 2 : 0, ig1 = x_open ? ie + 1 : ie + 3;
  for (int i = ig0; i <= ig1; i++)
    for (int k = 2; k <= kn; k++)
      for (int side = 0; side < 2; side++) {
        size_t gidx = id(i, side ? nyy : 1, k), c = id(i, side ? jn : 2, k);
        for (int v = 0; v < 7; v++) M.m[v][gidx] = M.m[v][c];
        M.m[7][gidx] = M.m[6][c];
        M.m[8][gidx] = M.m[6][c];
        M.J[gidx] = M.J[c];
      }
  for (int i = ig0; i <= ig1; i++)
    for (int j = 1; j <= nyy; j++)
      for (int side = 0; side < 2; side++) {
        size_t gidx = id(i, j, side ? nzz : 1), c = id(i, j, side ? kn : 2);
        for (int v = 0; v < 7; v++) M.m[v][gidx] = M.m[v][c];
        M.m[7][gidx] = M.m[6][c];
        M.m[8][gidx] = M.m[6][c];
        M.J[gidx] = M.J[c];
      }
  struct { int i1, j1, k1; double off; } fr[3] = {{ie, jn - 1, kn - 1, 0.5}, {ie - 1, jn, kn - 1, 1.0}, {ie - 1, jn - 1, kn, 0.5}};
  for (int d = 0; d < 3; d++)
    for (int j = 1; j <= fr[d].j1; j++) {
      double etdy, ydet;
      stretch(high, g, det, j, fr[d].off, etdy, ydet);
      double J = 1. / (1 * ydet * 1);
      for (int i = 2; i <= fr[d].i1; i++)
        for (int k = 1; k <= fr[d].k1; k++) {
          size_t c = id(i, j, k);
          M.mf[d][0][c] = 1; M.mf[d][4][c] = etdy; M.mf[d][8][c] = 1;
          M.Jf[d][c] = J;
        }
    }
  // Jacobian_v.cpp:134-151: the wall faces take the ghost-cell metric
  for (int i = 2; i <= ie - 1; i++)
    for (int k = 1; k < kn; k++) {
      size_t f1 = id(i, 1, k), fn = id(i, jn, k), g1 = id(i, 1, k), gn = id(i, nyy, k);
      for (int v = 3; v < 6; v++) { M.mf[1][v][f1] = M.m[v][g1]; M.mf[1][v][fn] = M.m[v][gn]; }
      M.Jf[1][fn] = M.J[gn];
      M.Jf[1][f1] = M.J[g1];
    }
}

// Wavy lower wall, flat upper wall (no reference code): the mapping
// x = xi, z = zeta, y = yw(x) + (high - yw(x)) Y0(eta) / high with the
// channel's tanh clustering Y0 (Jacobian.cpp:76-90) and
// yw(x) = amp sin(4 pi x / Lx), Lx = Nx dxi.  J = 1 / y_eta and the metric
// terms are the analytic inverse: xidx = ztdz = 1, etdx = -y_xi / y_eta,
// etdy = 1 / y_eta, the rest zero; evaluated at the positions and with the
// ghost-row / wall-face rules of channel_metrics, cell i at
// x = (i - 2.5) dxi.
void wavy_metrics(int nx, int ny, int nz, double dxi, double det, double high, double g, double amp, MetricSet &M) {
  const int X = nx + 6, Y = ny + 4, Z = nz + 4;
  const size_t n = (size_t)X * Y * Z;
  auto id = [&](int i, int j, int k) { return ((size_t)i * Y + j) * Z + k; };
  M.J.assign(n, 0.0);
  for (int v = 0; v < 9; v++) M.m[v].assign(n, 0.0);
  for (int d = 0; d < 3; d++) {
    M.Jf[d].assign(n, 0.0);
    for (int v = 0; v < 9; v++) M.mf[d][v].assign(n, 0.0);
  }
  const double kx = 4 * M_PI / (nx * dxi);
  auto point = [&](double x, double eta, double &J, double &etdx, double &etdy) {
    const double Y0 = 0.5 * high * (1 - tanh(g * (1 - 2 * eta)) / tanh(g));
    const double sech = 1. / cosh(g * (1 - 2 * eta));
    const double Y0p = high * g / tanh(g) * sech * sech;
    const double yw = amp * sin(kx * x), ywp = amp * kx * cos(kx * x);
    const double y_eta = (high - yw) * Y0p / high;
    const double y_xi = ywp * (1 - Y0 / high);
    J = 1. / y_eta;
    etdy = 1. / y_eta;
    etdx = -y_xi / y_eta;
  };
  const int ie = nx + 2, jn = ny + 1, kn = nz + 1, nyy = jn + 1, nzz = kn + 1;
  for (int i = 0; i <= ie + 3; i++)
    for (int j = 2; j <= jn; j++) {
      double J, etdx, etdy;
      point((i - 2.5) * dxi, (j - 1.5) * det, J, etdx, etdy);
      for (int k = 2; k <= kn; k++) {
        size_t c = id(i, j, k);
        M.m[0][c] = 1; M.m[3][c] = etdx; M.m[4][c] = etdy; M.m[8][c] = 1;
        M.J[c] = J;
      }
    }
  for (int i = 0; i <= ie + 3; i++)
    for (int k = 2; k <= kn; k++)
      for (int side = 0; side < 2; side++) {
        size_t gidx = id(i, side ? nyy : 1, k), c = id(i, side ? jn : 2, k);
        for (int v = 0; v < 7; v++) M.m[v][gidx] = M.m[v][c];
        M.m[7][gidx] = M.m[6][c];
        M.m[8][gidx] = M.m[6][c];
        M.J[gidx] = M.J[c];
      }
  for (int i = 0; i <= ie + 3; i++)
    for (int j = 1; j <= nyy; j++)
      for (int side = 0; side < 2; side++) {
        size_t gidx = id(i, j, side ? nzz : 1), c = id(i, j, side ? kn : 2);
        for (int v = 0; v < 7; v++) M.m[v][gidx] = M.m[v][c];
        M.m[7][gidx] = M.m[6][c];
        M.m[8][gidx] = M.m[6][c];
        M.J[gidx] = M.J[c];
      }
  // faces: x-face array (i, j, k) <-> face i+1/2 of cell (i, j+1, k+1);
  // y-face (i, j, k) <-> face j+1/2 of cell (i+1, j, k+1); z-face (i, j, k)
  // <-> face k+1/2 of cell (i+1, j+1, k)
  struct { int i1, j1, k1; double xoff, eoff; } fr[3] = {
      {ie, jn - 1, kn - 1, 2.0, 0.5}, {ie - 1, jn, kn - 1, 1.5, 1.0}, {ie - 1, jn - 1, kn, 1.5, 0.5}};
  for (int d = 0; d < 3; d++)
    for (int i = 2; i <= fr[d].i1; i++)
      for (int j = 1; j <= fr[d].j1; j++) {
        double J, etdx, etdy;
        point((i - fr[d].xoff) * dxi, (j - fr[d].eoff) * det, J, etdx, etdy);
        for (int k = 1; k <= fr[d].k1; k++) {
          size_t c = id(i, j, k);
          M.mf[d][0][c] = 1; M.mf[d][3][c] = etdx; M.mf[d][4][c] = etdy; M.mf[d][8][c] = 1;
          M.Jf[d][c] = J;
        }
      }
  for (int i = 2; i <= ie - 1; i++)
    for (int k = 1; k < kn; k++) {
      size_t f1 = id(i, 1, k), fn = id(i, jn, k), g1 = id(i, 1, k), gn = id(i, nyy, k);
      for (int v = 3; v < 6; v++) { M.mf[1][v][f1] = M.m[v][g1]; M.mf[1][v][fn] = M.m[v][gn]; }
      M.Jf[1][fn] = M.J[gn];
      M.Jf[1][f1] = M.J[g1];
    }
}

// Hyperplane.cpp:50-78 in O(N): planes m = 7..ie+ny+nz ascending, inside a
// plane i, then j ascending, k = m - i - j.
bool hyperplane(int nx, int ny, int nz, int *Nijk, long nijk_len, int *ijk, long ijk_len) {
  const int ie = nx + 2, jn = ny + 1, kn = nz + 1, nyy = jn + 1, nzz = kn + 1;
  if (nijk_len < 2L * (ie + jn + kn + 1) || ijk_len < 3L * ((long)nx * ny * nz + 1)) return false;
  long ii = 0;
  for (int m = 7; m <= ie + jn + kn; m++) {
    int mi = 0;
    for (int i = 3; i <= ie; i++)
      for (int j = 2; j < nyy; j++) {
        int k = m - i - j;
        if (k >= 2 && k < nzz) {
          ii++; mi++;
          ijk[3 * ii] = i; ijk[3 * ii + 1] = j; ijk[3 * ii + 2] = k;
        }
      }
    Nijk[2 * m] = (int)ii;
    Nijk[2 * m + 1] = mi;
  }
  return true;
}

}  // namespace cgli
