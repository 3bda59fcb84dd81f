// Buffers and launcher of the filter sensor (kernels_filter.cu).
#pragma once
#include <cuda_runtime.h>

#include "cgli_dev.cuh"

namespace cgli {

struct FilterBufs {
  double *yp = nullptr;             // Y_point, reference layout
  double *ep[3] = {};               // EpX, EpY, EpZ
  double *lev[2][4] = {};           // two consecutive filter levels, momentum and density
  double *acc[4] = {};              // running high-pass sum
  double *eh = nullptr, *e2h = nullptr;
};

// EpX/EpY/EpZ of Filter.cpp from d.U_, d.J and b.yp: 13 launches on s
cudaError_t launch_filter(const Dev &d, const FilterBufs &b, double crit, double e_high, double e_low,
                          cudaStream_t s);
int filter_smem_bytes();

}  // namespace cgli
