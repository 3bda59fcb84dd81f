// Fast path of one inner iteration.
#include "cgli_dev.cuh"
#include "cgli_launch.h"

namespace cgli {

void launch_fused_iteration(const Dev &d, cudaStream_t s, int precision, int update_blocks) {
  (void)precision;
  launch_halo_bc(d, s);
  launch_flux_x(d, s);
  launch_flux_y(d, s);
  launch_flux_z(d, s);
  launch_viscous(d, s);
  launch_dts(d, s, update_blocks);
}

}  // namespace cgli
