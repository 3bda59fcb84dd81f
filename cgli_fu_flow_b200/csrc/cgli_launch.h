// Host-side launchers of the kernel translation units.
#pragma once
#include <cuda_runtime.h>

#include <vector>

#include "cgli_dev.cuh"

namespace cgli {

// tile shape of the wavefront sweeps: TI x TJ (i, j) columns per CTA
constexpr int SWEEP_TI = 8;
constexpr int SWEEP_TJ = 16;
constexpr int CGLI_TIMEOUT_CODE = 6;

// buffers of the tile-wavefront sweeps (kernels_sweep.cu)
struct SweepArgs {
  double *dq[5];                  // dQ: forward result, then backward result (in place)
  double *halo_f[5], *halo_b[5];  // lagged periodic halo planes, Y_m x Z_m each
  double *xbuf, *ybuf;            // products handed between tiles
  unsigned long long *prog;       // per-tile progress counters
  unsigned int *ticket;           // tile ticket counter
  const int *order;               // tile visiting order (anti-diagonals)
  const double *Jtab, *etdytab;   // per-j metrics of a grid uniform in x and z
  int channel_metrics;            // 1: use Jtab / etdytab instead of the 3-D arrays
  int final_pass;                 // backward pass of the last sweep: apply the update
  int spin_limit;                 // bounded wait (polls) for a neighbouring tile
};

void sweep_tile_order(int nti, int ntj, std::vector<int> &order);
void launch_sweeps(const Dev &d, const SweepArgs &a, cudaStream_t s);
// residual assembly writing MR and the first sweep's lagged halo planes
void launch_residual_fast(const Dev &d, const SweepArgs &a, cudaStream_t s);

void launch_halo_bc(const Dev &d, cudaStream_t s);
void launch_halo_x(const Dev &d, cudaStream_t s);
void launch_bc_y(const Dev &d, cudaStream_t s);
void launch_bc_z(const Dev &d, cudaStream_t s);
void launch_flux_x(const Dev &d, cudaStream_t s);
void launch_flux_y(const Dev &d, cudaStream_t s);
void launch_flux_z(const Dev &d, cudaStream_t s);
void launch_viscous(const Dev &d, cudaStream_t s);
// residual, sweeps and update of the reference-granularity path; leaves
// per-block partial sums of the squared increments in d.partial
void launch_dts(const Dev &d, cudaStream_t s, int update_blocks_x);
// reduces d.partial (nblocks x 5) into out[5] = sqrt(sum) * scale
void launch_norms(const Dev &d, cudaStream_t s, int nblocks, double scale, double *out);
// bulk mass flux (Driven_force.cpp:38-62) into out[0]
void launch_bulk_flux(const Dev &d, cudaStream_t s, double *out);
// time-level shift over planes 2..ie+1 (main.cpp:364-386)
void launch_end_step(const Dev &d, cudaStream_t s);

// one complete inner iteration on the fast path (halo, boundaries, residual,
// sweeps, update, partial norms); capturable into a CUDA graph
void launch_fused_iteration(const Dev &d, const SweepArgs &a, cudaStream_t s, int precision);

}  // namespace cgli
