// Host-side launchers of the kernel translation units.
#pragma once
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "cgli_dev.cuh"

namespace cgli {

// words per slot of SweepArgs::cellrec: record, MR (16 words: whole 16-byte
// vectors in both precisions)
constexpr int CR_N = REC_N + 5;
constexpr int CR_MR = REC_N;
static_assert(CR_N == 16, "record + MR fill 16 words");
// position of 16-byte vector u (0..7 FP64, 0..3 FP32) within the slot whose
// index in its step block is t: rotated by t so that the slots' vectors,
// read one per lane, spread over the shared-memory banks
template <typename T>
__host__ __device__ __forceinline__ int rec_vec_pos(int u, int t) {
  return sizeof(T) == 8 ? (u ^ (t & 7)) : (u ^ ((t >> 1) & 3));
}

// Wavefront geometry per arithmetic type of the passes: TI x TJ (i, j)
// columns per CTA (one thread each, so TI * TJ <= 1024 and a multiple of
// 32), the depth of the ring of record stages in shared memory, and the
// largest cluster of CTAs along x (1: no clusters).  Measured at
// 256x192x192: the FP64 passes are fastest on 16 x 16 tiles with a 3-step
// ring, the FP32 passes on 8 x 16 tiles in clusters of 8.
#ifndef CGLI_SWEEP_TI
#define CGLI_SWEEP_TI 16
#endif
#ifndef CGLI_SWEEP_TJ
#define CGLI_SWEEP_TJ 16
#endif
#ifndef CGLI_SWEEP_RING
#define CGLI_SWEEP_RING 3
#endif
#ifndef CGLI_SWEEP_CLUSTER_MAX
#define CGLI_SWEEP_CLUSTER_MAX 1
#endif
#ifndef CGLI_SWEEP_TI_F32
#define CGLI_SWEEP_TI_F32 8
#endif
#ifndef CGLI_SWEEP_TJ_F32
#define CGLI_SWEEP_TJ_F32 16
#endif
#ifndef CGLI_SWEEP_RING_F32
#define CGLI_SWEEP_RING_F32 2
#endif
#ifndef CGLI_SWEEP_CLUSTER_MAX_F32
#define CGLI_SWEEP_CLUSTER_MAX_F32 8
#endif
template <typename T> struct SweepTile;
template <> struct SweepTile<double> {
  static constexpr int TI = CGLI_SWEEP_TI, TJ = CGLI_SWEEP_TJ, RING = CGLI_SWEEP_RING;
  static constexpr int CLUSTER_MAX = CGLI_SWEEP_CLUSTER_MAX;
};
template <> struct SweepTile<float> {
  static constexpr int TI = CGLI_SWEEP_TI_F32, TJ = CGLI_SWEEP_TJ_F32, RING = CGLI_SWEEP_RING_F32;
  static constexpr int CLUSTER_MAX = CGLI_SWEEP_CLUSTER_MAX_F32;
};
static_assert(SweepTile<double>::TI * SweepTile<double>::TJ <= 1024 &&
                  (SweepTile<double>::TI * SweepTile<double>::TJ) % 32 == 0, "FP64 sweep tile shape");
static_assert(SweepTile<float>::TI * SweepTile<float>::TJ <= 1024 &&
                  (SweepTile<float>::TI * SweepTile<float>::TJ) % 32 == 0, "FP32 sweep tile shape");
constexpr int CGLI_TIMEOUT_CODE = 6;

// buffers of the tile-wavefront sweeps (kernels_sweep.cu)
struct SweepArgs {
  // per-cell sweep data in the tile-skewed layout: slot (tile, forward step,
  // thread) = (tile * S + s) * TI*TJ + t, S = Nz + TI + TJ - 2
  double *dq[5];                  // dQ: forward result, then backward result (in place)
  // per slot, CR_N consecutive words: the split-Jacobian / diagonal record
  // (REC_N) and the residual MR (5), so that the residual writes and the
  // sweep reads whole 16-byte vectors of one cell
  double *cellrec;
  // the same in float for CGLI_MIXED
  float *dqf[5], *cellrecf;
  // periodic lagged halos, indexed j*Z_m + k: dQ of plane ie (forward) / 3
  // (backward) and the records of planes 2 / ie+1
  double *halo_f[5], *halo_b[5], *hrec_f[REC_N], *hrec_b[REC_N];
  float *halo_ff[5], *halo_bf[5], *hrecf_f[REC_N], *hrecf_b[REC_N];
  // the halo neighbour's product A.dQ of the current pass per (j, k), formed
  // before the pass from the halo record and the lagged dQ
  double *hxp[5];
  float *hxpf[5];
  double *xbuf, *ybuf;            // products handed between tiles
  float *xbuff, *ybuff;
  unsigned int *ticket;           // tile ticket counter
  const int *order;               // tile visiting order (anti-diagonals)
  const double *Jtab, *etdytab;   // per-j metrics of a grid uniform in x and z
  int channel_metrics;            // 1: use Jtab / etdytab instead of the 3-D arrays
  int spin_limit;                 // bounded wait (polls) for a neighbouring tile
  int cluster_x;                  // wavefront CTAs per cluster along x (1: no clusters)
};

// slot of cell (i, j, k) in the tile-skewed layout of the passes in type T
template <typename T>
__host__ __device__ __forceinline__ long long skew_slot(const Dev &d, int i, int j, int k) {
  constexpr int TI = SweepTile<T>::TI, TJ = SweepTile<T>::TJ;
  const int ntj = (d.ny + TJ - 1) / TJ;
  const int S = d.nz + TI + TJ - 2;
  const int il = (i - 3) % TI, jl = (j - 2) % TJ;
  const int tile = ((i - 3) / TI) * ntj + (j - 2) / TJ;
  const int s = (k - 2) + il + jl;
  return ((long long)tile * S + s) * (TI * TJ) + il * TJ + jl;
}
template <typename T>
__host__ __device__ __forceinline__ long long skew_size(const Dev &d) {
  constexpr int TI = SweepTile<T>::TI, TJ = SweepTile<T>::TJ;
  const long long ntiles = (long long)((d.nx + TI - 1) / TI) * ((d.ny + TJ - 1) / TJ);
  return ntiles * (d.nz + TI + TJ - 2) * (TI * TJ);
}
// tiles of the wavefront in x and y for the passes in type T
template <typename T> inline int sweep_tiles_x(int nx) { return (nx + SweepTile<T>::TI - 1) / SweepTile<T>::TI; }
template <typename T> inline int sweep_tiles_y(int ny) { return (ny + SweepTile<T>::TJ - 1) / SweepTile<T>::TJ; }

void sweep_tile_order(int nti, int ntj, std::vector<int> &order);
// shared-memory opt-in of the wavefront kernels (once per process and device)
cudaError_t sweep_kernel_attributes();
int sweep_cluster_x(int nti, int ntj, bool mixed);
// the four wavefront passes (two sweeps) of one inner iteration
void launch_sweeps(const Dev &d, const SweepArgs &a, cudaStream_t s, bool mixed);
// the update and norm partials after the last pass (k_update_skewed)
void launch_sweep_update(const Dev &d, const SweepArgs &a, cudaStream_t s, bool mixed);
// partial sums (blocks) the update after the wavefront passes writes
int sweep_update_blocks(const Dev &d, bool mixed);
// everything of a fused inner iteration before the sweeps
void launch_fused_residual(const Dev &d, const SweepArgs &a, cudaStream_t s, int precision);
// one pass (forward / backward, final with the update) of the sweeps
void launch_sweep_pass(const Dev &d, const SweepArgs &a, cudaStream_t s, bool mixed, bool backward, bool final_pass);
// Dual_time_stepping.cpp:737-922 residual on the natural layout: MR and
// NL = NR = D^-1 MR on the interior cells
void launch_dts_residual(const Dev &d, cudaStream_t s);
// DP-LUR inner solver of DPLUSGS.cpp (kernels_dplur.cu): residual, four
// Jacobi relaxations (final result in NR), update with per-block partial
// sums of the squared squared increments in d.partial (nx * ny blocks).
// Reads the per-j metric tables of sw when sw.channel_metrics is set.
void launch_dplur(const Dev &d, const SweepArgs &sw, cudaStream_t s);
// one relaxation NR -> NL (from_nr) or NL -> NR
void launch_dplur_relax(const Dev &d, const SweepArgs &sw, cudaStream_t s, bool from_nr);
// halo, boundaries, fluxes, viscous terms, then launch_dplur
void launch_dplur_iteration(const Dev &d, const SweepArgs &sw, cudaStream_t s);
// residual assembly writing MR and the first sweep's lagged halo planes
void launch_residual_fast(const Dev &d, const SweepArgs &a, cudaStream_t s, bool mixed);

// adds the per-(i, j) sums over k of Statistic.cpp:120-160 to sums
// [11][nx][ny] (U, V, W, T, UU, VV, WW, TT, UV, UT, VT)
void launch_statistics(const Dev &d, cudaStream_t s, double *sums);
// d.iJ = 1/J on every cell (0 where J = 0)
void launch_inverse_j(const Dev &d, cudaStream_t s);
// main.cpp:167-210: x halo (periodic slab only), Y, X (open slab only), Z
void launch_halo_bc(const Dev &d, cudaStream_t s);
// true (and d.ftab filled) when every face metric has the channel's form
// with a per-row etdy and J; dflag: one device int of scratch
bool check_face_tables(const Dev &d, int *dflag, cudaStream_t s);
// X_boundary_condition.cpp on an open slab (no-op on a periodic one)
void launch_bc_x(const Dev &d, cudaStream_t s);
// outlet sponge target velocity into d.scal[1] (open slab with an outlet layer)
void launch_target_u(const Dev &d, cudaStream_t s);
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
// bulk mass flux (Driven_force.cpp:38-62) into out[0]; out holds 8 + 296
// doubles (per-block partial sums at out + 8)
void launch_bulk_flux(const Dev &d, cudaStream_t s, double *out);
// time-level shift over planes 2..ie+1 (main.cpp:364-386)
void launch_end_step(const Dev &d, cudaStream_t s);
// extrapolated initial guess of a step (order 1 or 2) on the interior cells
void launch_predict(const Dev &d, cudaStream_t s, int order);

// message returned by cgli_last_error() on this thread
void set_last_error(const std::string &msg);

}  // namespace cgli
