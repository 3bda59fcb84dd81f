// Host-side set-up helpers (analytic metrics, hyperplane enumeration).
#pragma once
#include <vector>

namespace cgli {

struct MetricSet {
  std::vector<double> J, m[9], Jf[3], mf[3][9];
};

// x_open: the first and last rank's end planes (Jacobian.cpp:53-58, :110-157)
void channel_metrics(int nx, int ny, int nz, double det, double high, double g, MetricSet &M, bool x_open = false);
void wavy_metrics(int nx, int ny, int nz, double dxi, double det, double high, double g, double amp, MetricSet &M);
bool hyperplane(int nx, int ny, int nz, int *Nijk, long nijk_len, int *ijk, long ijk_len);

}  // namespace cgli
