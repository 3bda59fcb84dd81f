// Host-side launchers of the kernel translation units.
#pragma once
#include <cuda_runtime.h>
#include "cgli_dev.cuh"

namespace cgli {

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
void launch_fused_iteration(const Dev &d, cudaStream_t s, int precision, int update_blocks);

}  // namespace cgli
