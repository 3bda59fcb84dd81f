// LU-SGS forward / backward sweeps as persistent tile wavefronts.
//
// The reference visits the cells of one x-slab hyperplane by hyperplane
// (i+j+k = m, Dual_time_stepping.cpp:983-1664), one OpenMP barrier per
// plane.  A cell's update depends only on its three upwind neighbours, so
// any order that respects that dependency graph gives the same numbers.
// Here each CTA owns a TI x TJ tile of (i, j) columns and marches along k.
// Thread (il, jl) handles cell k = 2 + s - il - jl at step s of the forward
// pass: its i- and j-neighbours were handled by the neighbouring threads one
// step earlier and hand over their products A.dQ through shared memory; its
// k-neighbour is its own previous step.  The backward pass runs the mirror
// image, and its step s visits exactly the cells of forward step S-1-s.
//
// Storage.  Everything the sweeps read per cell -- the split-Jacobian /
// diagonal record, the residual MR and dQ -- lives in a tile-skewed layout,
// slot (tile, forward step, thread), so at every step the threads of a tile
// read and write consecutive words (the residual kernel writes it).  Only the
// final update touches the reference layout.
//
// Hand-over between tiles.  Tiles pass the products of their last row /
// column through global buffers filled with a sentinel bit pattern before the
// pass; the consumer spins (bounded) on the values themselves until none is
// the sentinel, so a hand-over needs no fence and no counter (4- and 8-byte
// stores are single-copy atomic).  A wait on another tile gives up after
// SweepArgs::spin_limit polls, or at once when its CTA or any tile has
// already given up (the CTA's dead flag, the status word): it records the
// timeout code in the status word and the tile carries on to the end of the
// pass without waiting, computing values nobody will use.  So no wait is
// ever repeated at full length, every bulk copy is still awaited in order
// (those waits have a fixed bound: the copies complete on their own), the
// fast path carries no exit test, the update kernel leaves the state alone
// and the host reports CGLI_ETIMEOUT.
// Tiles take tickets in an order where every dependency holds a smaller
// ticket, so a waiting CTA only ever waits on CTAs that are already running.
//
// Thread-block clusters (SweepArgs::cluster_x > 1, the CL instantiation):
// the CTAs of a cluster are consecutive tiles along x, launched together.
// Inside a cluster the x hand-over is pushed, not pulled: the producing
// tile writes the products of its edge row straight into the consuming
// tile's shared-memory ring with st.async, which counts the bytes on that
// slot's mbarrier in the consumer (armed by the consumer with the bytes it
// expects); the consumer waits on its own barrier and gives the slot back
// with a relaxed arrival on the producer's "empty" barrier.  No fence is on
// either path.  The first (last) tile of a cluster still receives (sends)
// through the global buffers.  A cluster takes one ticket for its whole row
// of tiles.  A CTA must not leave while a push into its shared memory is
// still in flight, and a slot must not be re-armed before its phase has
// completed, so the receiving lanes wait on every hand-over step, whether
// their own cell is inside the slab or not, and these waits do not give up
// at the tile wait limit or on the dead flag: the producer always pushes
// every step (it is co-scheduled with the consumer and its own waits are
// bounded), so they have the fixed bound of a copy wait, scaled by the wait
// limit because the producer may itself sit in one wait of that length.
//
// The periodic x halo keeps the reference's lag: the forward pass at i = 3
// uses dQ of plane Nx+2 as it was at the start of the sweep (halo_f), the
// backward pass at i = Nx+2 uses dQ of plane 3 (halo_b).  The backward pass of
// the first sweep writes both halos for the second sweep; after the final
// backward pass a separate, fully parallel kernel applies the primitive
// update of Dual_time_stepping.cpp:1702-1743 and accumulates the squared
// increments of the residual norms.
//
// T is the arithmetic type of the sweep (double, or float for CGLI_MIXED).
#include "cgli_dev.cuh"
#include "cgli_launch.h"
#include "tc_sm100.cuh"

// steps ahead that a tile loads the products its neighbouring tiles hand over
#ifndef CGLI_SWEEP_PREFETCH
#define CGLI_SWEEP_PREFETCH 2
#endif
// tiles per SM the wavefront kernel is compiled for (a register cap)
#ifndef CGLI_SWEEP_MINBLOCKS
#define CGLI_SWEEP_MINBLOCKS 1
#endif
// backward pass: the forward result dQ of each step arrives with the
// records' bulk copy (five rows of one value per thread)

namespace cgli {

using F64 = SweepTile<double>;
using F32 = SweepTile<float>;

template <typename T> struct SweepPtrs;
template <> struct SweepPtrs<double> {
  __device__ __forceinline__ static double *const *dq(const SweepArgs &a) { return a.dq; }
  __device__ __forceinline__ static const double *cellrec(const SweepArgs &a) { return a.cellrec; }
  __device__ __forceinline__ static double *const *hf(const SweepArgs &a) { return a.halo_f; }
  __device__ __forceinline__ static double *const *hb(const SweepArgs &a) { return a.halo_b; }
  __device__ __forceinline__ static double *const *hrec(const SweepArgs &a, bool b) { return b ? a.hrec_b : a.hrec_f; }
  __device__ __forceinline__ static double *xb(const SweepArgs &a) { return a.xbuf; }
  __device__ __forceinline__ static double *yb(const SweepArgs &a) { return a.ybuf; }
  __device__ __forceinline__ static double *const *hxp(const SweepArgs &a) { return a.hxp; }
};
template <> struct SweepPtrs<float> {
  __device__ __forceinline__ static float *const *dq(const SweepArgs &a) { return a.dqf; }
  __device__ __forceinline__ static const float *cellrec(const SweepArgs &a) { return a.cellrecf; }
  __device__ __forceinline__ static float *const *hf(const SweepArgs &a) { return a.halo_ff; }
  __device__ __forceinline__ static float *const *hb(const SweepArgs &a) { return a.halo_bf; }
  __device__ __forceinline__ static float *const *hrec(const SweepArgs &a, bool b) { return b ? a.hrecf_b : a.hrecf_f; }
  __device__ __forceinline__ static float *xb(const SweepArgs &a) { return a.xbuff; }
  __device__ __forceinline__ static float *yb(const SweepArgs &a) { return a.ybuff; }
  __device__ __forceinline__ static float *const *hxp(const SweepArgs &a) { return a.hxpf; }
};

// face-direction metrics of a cell: general 3-D arrays, or a grid uniform in
// x and z (channel) whose only varying term is etdy(j), held in shared memory
struct MetricsGeneral {
  static constexpr bool kChannel = false;
  template <typename T>
  __device__ __forceinline__ static void dirs(const Dev &d, const double *, long long c, int, T mm[9]) {
#pragma unroll
    for (int v = 0; v < 9; v++) mm[v] = (T)d.m[v][c];
  }
};
struct MetricsChannel {
  static constexpr bool kChannel = true;
  template <typename T>
  __device__ __forceinline__ static void dirs(const Dev &, const double *et, long long, int jl, T mm[9]) {
    mm[0] = 1; mm[1] = 0; mm[2] = 0;
    mm[3] = 0; mm[4] = (T)et[jl]; mm[5] = 0;
    mm[6] = 0; mm[7] = 0; mm[8] = 1;
  }
};

__device__ __forceinline__ double ld_gpu(const double *p) {
  double v;
  asm volatile("ld.relaxed.gpu.global.f64 %0, [%1];" : "=d"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ float ld_gpu(const float *p) {
  float v;
  asm volatile("ld.relaxed.gpu.global.f32 %0, [%1];" : "=f"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ bool is_sentinel(double v) { return __double_as_longlong(v) == -1ll; }
__device__ __forceinline__ bool is_sentinel(float v) { return __float_as_int(v) == -1; }

// a wait on another tile has given up somewhere: this CTA's dead flag or
// the grid's status word
__device__ __forceinline__ bool given_up(const volatile int *dead, const int *status) {
  return *dead || *(const volatile int *)status;
}
__device__ __forceinline__ void give_up(volatile int *dead, int *status) {
  atomicExch(status, CGLI_TIMEOUT_CODE);
  *dead = 1;
}

// bounded spin on five values handed over by a neighbouring tile; false when
// it gives up (after `limit` polls, or at once once anything gave up)
template <typename T>
__device__ __forceinline__ bool recv5(const T *src, T out[5], int *status, int limit, volatile int *dead) {
  for (int it = 0;; it++) {
    bool ok = true;
#pragma unroll
    for (int v = 0; v < 5; v++) {
      out[v] = ld_gpu(src + v);
      ok = ok && !is_sentinel(out[v]);
    }
    if (ok) return true;
    if (it >= limit || given_up(dead, status)) {
      give_up(dead, status);
      return false;
    }
    __nanosleep(20);
  }
}

// polls of the wait on a tile's own bulk copy of records (the copies complete
// on their own; this only bounds the wait against a failing device)
constexpr int kCopyPolls = 1 << 20;

// REC_N record words and (mr non-null) the 5 MR words of one slot, through
// the read-only path (CGLI_SWEEP_LDG) or plain loads
#ifndef CGLI_SWEEP_LDG
#define CGLI_SWEEP_LDG 0
#endif
__device__ __forceinline__ double2 ld_rec(const double2 *q) {
#if CGLI_SWEEP_LDG
  return __ldg(q);
#else
  return *q;
#endif
}
__device__ __forceinline__ float4 ld_rec(const float4 *q) {
#if CGLI_SWEEP_LDG
  return __ldg(q);
#else
  return *q;
#endif
}
// The 16-byte vectors of a slot are stored in an order rotated by the
// slot's position t in its step block (rec_vec_pos): a warp's vector loads
// of its slots (one per lane, consecutive slots 128 B (FP64) or 64 B (FP32)
// apart) then fall on distinct shared-memory banks in every phase of eight
// lanes.
__device__ __forceinline__ void load_cellrec(const double *p, int t, double rec[REC_N], double *mr) {
  // words 0..10 the record, 11..15 MR
  const double2 *q = reinterpret_cast<const double2 *>(p);
#pragma unroll
  for (int u = 0; u < 5; u++) {
    const double2 v = ld_rec(q + rec_vec_pos<double>(u, t));
    rec[2 * u] = v.x;
    rec[2 * u + 1] = v.y;
  }
  const double2 a = ld_rec(q + rec_vec_pos<double>(5, t));
  rec[10] = a.x;
  if (mr) {
    const double2 b = ld_rec(q + rec_vec_pos<double>(6, t)), c = ld_rec(q + rec_vec_pos<double>(7, t));
    mr[0] = a.y; mr[1] = b.x; mr[2] = b.y; mr[3] = c.x; mr[4] = c.y;
  }
}
__device__ __forceinline__ void load_cellrec(const float *p, int t, float rec[REC_N], float *mr) {
  const float4 *q = reinterpret_cast<const float4 *>(p);
  const float4 a = ld_rec(q + rec_vec_pos<float>(0, t)), b = ld_rec(q + rec_vec_pos<float>(1, t)),
               c = ld_rec(q + rec_vec_pos<float>(2, t));
  rec[0] = a.x; rec[1] = a.y; rec[2] = a.z; rec[3] = a.w;
  rec[4] = b.x; rec[5] = b.y; rec[6] = b.z; rec[7] = b.w;
  rec[8] = c.x; rec[9] = c.y; rec[10] = c.z;
  if (mr) {
    const float4 e = ld_rec(q + rec_vec_pos<float>(3, t));
    mr[0] = c.w; mr[1] = e.x; mr[2] = e.y; mr[3] = e.z; mr[4] = e.w;
  }
}

// The x neighbour of the slab's first plane (forward) / last plane
// (backward) is the periodic halo plane 2 / ie+1, a copy of plane ie / 3 made
// by the Q halo exchange; its record and the lagged dQ are kept per (j, k).
// Its product A+.dQ (forward) / A-.dQ (backward) is formed here once per
// pass for every (j, k), off the wavefront's critical path.
template <class Met, bool BACKWARD, typename T>
__global__ void k_halo_products(Dev d, SweepArgs a) {
  const int k = 2 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 2 + blockIdx.y;
  if (k > d.nz + 1) return;
  const long long h = (long long)j * d.dj + k;
  T rn[REC_N], mm[9];
#pragma unroll
  for (int v = 0; v < REC_N; v++) rn[v] = SweepPtrs<T>::hrec(a, BACKWARD)[v][h];
  Met::template dirs<T>(d, a.etdytab, h + (BACKWARD ? (long long)(d.nx + 3) : 2LL) * d.di, j, mm);
  Split<T> An = split_from_record<T>(rn, 0, mm[0], mm[1], mm[2]);
  T nh[5], o[5];
#pragma unroll
  for (int v = 0; v < 5; v++) nh[v] = BACKWARD ? SweepPtrs<T>::hb(a)[v][h] : SweepPtrs<T>::hf(a)[v][h];
  if (BACKWARD) upper_terms<T>(An, nh, o); else lower_terms<T>(An, nh, o);
#pragma unroll
  for (int v = 0; v < 5; v++) SweepPtrs<T>::hxp(a)[v][h] = o[v];
}

// The split products of one direction for a face metric with a single
// nonzero component m on momentum component q = DIR + 1 (the channel grid:
// xi = (1,0,0), eta = (0,etdy,0), zeta = (0,0,1)): lower_terms / upper_terms
// of split_from_record with the zero entries left out.
template <typename T, int DIR, bool BACKWARD>
__device__ __forceinline__ void channel_products(const T r[REC_N], T m, const T n[5], T o[5]) {
  constexpr int q = DIR + 1;
  const T U = r[R_UX + DIR], lam = r[R_LX + DIR], beta = r[R_BETA];
  const T p1q = r[R_H] * m, pq1 = r[R_HR] * m, p5q = rec_hbt<T>(r) * m, p51 = rec_g<T>(r) * U;
  if (!BACKWARD) {
    const T p11 = (T)0.5 * (beta * U + lam), p22 = (T)0.5 * (U + lam);
    o[0] = -p11 * n[0] - p1q * n[q];
#pragma unroll
    for (int v = 1; v <= 3; v++) o[v] = v == q ? -pq1 * n[0] - p22 * n[v] : -p22 * n[v];
    o[4] = -p51 * n[0] - p5q * n[q] - p22 * n[4];
  } else {
    const T m11 = (T)0.5 * (beta * U - lam), m22 = (T)0.5 * (U - lam);
    o[0] = +m11 * n[0] + p1q * n[q];
#pragma unroll
    for (int v = 1; v <= 3; v++) o[v] = v == q ? +pq1 * n[0] + m22 * n[v] : m22 * n[v];
    o[4] = +p51 * n[0] + p5q * n[q] + m22 * n[4];
  }
}

template <int TI, int TJ, class Met, bool BACKWARD, typename T, bool CL>
__global__ void __launch_bounds__(TI *TJ, CGLI_SWEEP_MINBLOCKS) k_sweep(Dev d, SweepArgs a) {
  __shared__ T sx[2][TI][TJ][5];   // i-direction products, double-buffered by step parity
  __shared__ T sy[2][TI][TJ][5];   // j-direction products
  __shared__ double s_jt[TJ], s_et[TJ];
  __shared__ int s_tile;
  __shared__ int s_dead;       // a wait of this CTA gave up: no more waiting
  // x hand-over ring inside a cluster: RX steps x TJ lanes x XW words
  constexpr int RX = 8, XW = sizeof(T) == 8 ? 6 : 8;
  __shared__ __align__(8) uint64_t s_full[CL ? RX : 1], s_empty[CL ? RX : 1];
  // steps of records in flight: the ring holds RING steps' blocks, the copy
  // of step s + RING - 1 is issued at step s
  constexpr int RING = SweepTile<T>::RING;
  constexpr bool DQB = BACKWARD;
  __shared__ __align__(8) uint64_t s_bar[RING];
  // the CTA's records of RING steps: step s's TI*TJ slots are one contiguous
  // block of TI*TJ*CR_N words in the tile-skewed layout, brought in with one
  // bulk copy RING - 1 steps ahead (backward, optionally followed by the five
  // rows of the step's forward result dQ)
  extern __shared__ __align__(128) unsigned char s_dyn[];
  T *const s_rec = reinterpret_cast<T *>(s_dyn);
  constexpr int kStage = TI * TJ * (CR_N + (DQB ? 5 : 0));   // words per ring stage
  T *const s_rx = s_rec + RING * kStage;   // the cluster ring follows the record ring
  const int il = threadIdx.x / TJ, jl = threadIdx.x % TJ;
  const int nti = (d.nx + TI - 1) / TI, ntj = (d.ny + TJ - 1) / TJ;
  // cluster of ncl consecutive x tiles (1 without clusters): one ticket per
  // cluster, taken by its first CTA and written into every CTA's s_tile
  const uint32_t ncl = CL ? tc::cluster_nctarank() : 1u, crank = CL ? tc::cluster_ctarank() : 0u;
  const int nunits = (nti / (int)ncl) * ntj;
  if (threadIdx.x == 0) {
    if (!CL) {
      s_tile = (int)atomicAdd(a.ticket, 1u);
    } else if (crank == 0) {
      const uint32_t t = atomicAdd(a.ticket, 1u);
      for (uint32_t r = 0; r < ncl; r++) tc::st_cluster_u32(tc::mapa(tc::smem_addr(&s_tile), r), t);
    }
    s_dead = 0;
    if (CL) {
#pragma unroll
      for (int r = 0; r < RX; r++) {
        tc::mbar_init(tc::smem_addr(&s_full[r]), 1);    // the consumer's own arm per use
        tc::mbar_init(tc::smem_addr(&s_empty[r]), 1);   // the consumer's release per use
      }
      // a receiving CTA arms its first RX slots with the bytes of one push
      // before its producer can start (the cluster barrier below)
      if (ncl > 1 && (BACKWARD ? crank + 1 < ncl : crank > 0))
        for (int r = 0; r < RX && r < d.nz + TJ - 1; r++)
          tc::mbar_expect_tx(tc::smem_addr(&s_full[r]), TJ * 5 * sizeof(T));
    }
#pragma unroll
    for (int r = 0; r < RING; r++) tc::mbar_init(tc::smem_addr(&s_bar[r]), 1);
    tc::mbar_fence_init();
  }
  // tickets and barriers visible cluster-wide before any remote access
  if (CL) tc::cluster_sync(); else __syncthreads();
  const int ticket = s_tile;
  if (!CL && ticket >= nunits) return;   // (a cluster's ticket is always in range)
  const int unit = a.order[BACKWARD ? nunits - 1 - ticket : ticket];
  const int ta = (unit / ntj) * (int)ncl + (int)crank, tb = unit % ntj;
  const int tile = ta * ntj + tb;
  const int ie = d.nx + 2, jn = d.ny + 1;
  const int i = 3 + ta * TI + il, j = 2 + tb * TJ + jl;
  const bool inside = (i <= ie) && (j <= jn);
  if (threadIdx.x < TJ) {
    int jj = 2 + tb * TJ + threadIdx.x;
    s_jt[threadIdx.x] = (Met::kChannel && jj <= jn) ? a.Jtab[jj] : 1.0;
    s_et[threadIdx.x] = (Met::kChannel && jj <= jn) ? a.etdytab[jj] : 0.0;
  }
  __syncthreads();
  const int Nz = d.nz;
  const int S = Nz + TI - 1 + TJ - 1;
  const long long tile_base = (long long)tile * S * (TI * TJ);
  constexpr uint32_t kBlock = TI * TJ * CR_N * sizeof(T);
  constexpr uint32_t kRow = TI * TJ * sizeof(T);
  const T *const crec = SweepPtrs<T>::cellrec(a);
  auto issue = [&](int step) {   // one thread
    const int sf = BACKWARD ? S - 1 - step : step;
    const int b = step % RING;
    const uint32_t bar = tc::smem_addr(&s_bar[b]);
    T *const dst = s_rec + b * kStage;
    const long long slot0 = tile_base + (long long)sf * (TI * TJ);
    tc::mbar_expect_tx(bar, kBlock + (DQB ? 5 * kRow : 0));
    tc::bulk_load(tc::smem_addr(dst), crec + slot0 * CR_N, kBlock, bar);
    if (DQB)
#pragma unroll
      for (int v = 0; v < 5; v++)
        tc::bulk_load(tc::smem_addr(dst + TI * TJ * CR_N + v * TI * TJ), SweepPtrs<T>::dq(a)[v] + slot0, kRow, bar);
  };
  if (threadIdx.x == 0)
    for (int r = 0; r < RING - 1 && r < S; r++) issue(r);
  const int pa = BACKWARD ? ta + 1 : ta - 1, pb = BACKWARD ? tb + 1 : tb - 1;
  const int tile_pa = pa * ntj + tb, tile_pb = ta * ntj + pb;
  const bool halo_edge = BACKWARD ? (i == ie) : (i == 3);
  const bool recv_x = !halo_edge && (BACKWARD ? il == TI - 1 : il == 0);
  const bool recv_y = BACKWARD ? (jl == TJ - 1 || j == jn) : (jl == 0);
  const bool wall_y = BACKWARD ? (j == jn) : (j == 2);
  const bool send_x = BACKWARD ? (il == 0) : (il == TI - 1);
  const bool send_y = BACKWARD ? (jl == 0) : (jl == TJ - 1);
  // x hand-over inside the cluster: received from / sent to the neighbouring
  // CTA's shared memory; at the cluster's ends through the global buffers
  const bool dsm_recv = CL && ncl > 1 && (BACKWARD ? crank + 1 < ncl : crank > 0);
  const bool dsm_send = CL && ncl > 1 && (BACKWARD ? crank > 0 : crank + 1 < ncl);
  const uint32_t producer = BACKWARD ? crank + 1 : crank - 1, consumer = BACKWARD ? crank - 1 : crank + 1;
  // the step q of the consumer's wait is the producer's step q + TI - 1
  const int QN = S - TI + 1;   // hand-over steps per pass
  constexpr uint32_t kPush = TJ * 5 * sizeof(T);   // bytes pushed per hand-over step (armed above for the first RX)
  // the lanes that wait on the pushes: the tile's receiving edge, all of them
  const bool wait_x = dsm_recv && (BACKWARD ? il == TI - 1 : il == 0);
  const int push_polls = a.spin_limit > (0x7fffffff - kCopyPolls) / 64 ? 0x7fffffff : 64 * a.spin_limit + kCopyPolls;
  const T rdx = (T)d.rdxi, rdy = (T)d.rdet, rdz = (T)d.rdzt, rdt = (T)(1.0 / d.dt);
  T *xb = SweepPtrs<T>::xb(a), *yb = SweepPtrs<T>::yb(a);
  T *const *dq = SweepPtrs<T>::dq(a);
  T carry_z[5] = {0, 0, 0, 0, 0};

  // hand-over values of the next PD steps, loaded ahead: a neighbouring
  // tile runs just far enough ahead for its value to exist when needed, so
  // a load issued then would wait one L2 round trip per step; loaded PD
  // steps early it is usually there (a sentinel falls back to the bounded
  // poll)
  constexpr int PD = CGLI_SWEEP_PREFETCH;
  auto kl_of = [&](int step) {
    const int r = BACKWARD ? step - (TI - 1 - il) - (TJ - 1 - jl) : step - il - jl;
    return (inside && r >= 0 && r < Nz) ? (BACKWARD ? Nz - 1 - r : r) : -1;
  };
  const T *xsrc = xb + ((long long)tile_pa * TJ + jl) * Nz * 5;
  const T *ysrc = yb + ((long long)tile_pb * TI + il) * Nz * 5;
  const bool pre_x = recv_x && !dsm_recv, pre_y = recv_y && !wall_y;
  T px[PD][5], py[PD][5];
  auto preload = [&](int step, T *qx, T *qy) {
    const int k2 = kl_of(step);
#pragma unroll
    for (int v = 0; v < 5; v++) { qx[v] = (T)0; qy[v] = (T)0; }
    if (k2 < 0) return;
    if (pre_x)
#pragma unroll
      for (int v = 0; v < 5; v++) qx[v] = ld_gpu(xsrc + (long long)k2 * 5 + v);
    if (pre_y)
#pragma unroll
      for (int v = 0; v < 5; v++) qy[v] = ld_gpu(ysrc + (long long)k2 * 5 + v);
  };
#pragma unroll
  for (int p = 0; p < PD; p++) preload(p, px[p], py[p]);

  // the periodic lagged halo of the slab's x edge: the x neighbour's product,
  // formed before the pass (k_halo_products), loaded a step ahead by the
  // edge lanes
  T hx_cur[5], hx_nxt[5];
  auto load_hx = [&](int step, T *out) {
    const int k2 = kl_of(step);
    if (k2 < 0) return;
    const long long h = (long long)j * d.dj + 2 + k2;
#pragma unroll
    for (int v = 0; v < 5; v++) out[v] = SweepPtrs<T>::hxp(a)[v][h];
  };
  if (halo_edge) load_hx(0, hx_cur);
  // this thread's slot of step s: slot0 + (forward step) * TI * TJ
  const long long slot0 = tile_base + threadIdx.x;
  const int rel0 = BACKWARD ? -(TI - 1 - il) - (TJ - 1 - jl) : -il - jl;

  // unrolled twice: the ring and buffer indices of the two halves are
  // constants, and the compiler overlaps the halves' independent work
#pragma unroll 2
  for (int s = 0; s < S; s++) {
    const int rel = rel0 + s;
    const int kl = BACKWARD ? Nz - 1 - rel : rel;
    const bool active = inside && rel >= 0 && rel < Nz;
    // the slot read in step s - 1 is free again (every receiving lane read it
    // before the barrier that ended that step): arm it for its next use, then
    // give it back to the producer
    if (dsm_recv && threadIdx.x == 0 && s >= 1 && s - 1 < QN) {
      if (s - 1 + RX < QN) tc::mbar_expect_tx(tc::smem_addr(&s_full[(s - 1) % RX]), kPush);
      tc::mbar_arrive_cluster_relaxed(tc::mapa(tc::smem_addr(&s_empty[(s - 1) % RX]), producer));
    }
    // loads of the next cell go out first and land during the dependent part
    // stage (s + RING - 1) % RING was last read at step s - 1, before the previous barrier
    if (threadIdx.x == 0 && s + RING - 1 < S) issue(s + RING - 1);
    if (halo_edge && s + 1 < S) load_hx(s + 1, hx_nxt);
    // this step's records (bounded wait; a timeout is reported like a tile's)
    if (!tc::mbar_wait(tc::smem_addr(&s_bar[s % RING]), (s / RING) & 1, kCopyPolls)) give_up(&s_dead, d.status);
    // the cluster neighbour's push of this step (every receiving lane, so
    // that every push has landed before the slot is re-armed or the CTA leaves)
    if (wait_x && s < QN &&
        !tc::mbar_wait_cluster(tc::smem_addr(&s_full[s % RX]), (s / RX) & 1, push_polls))
      give_up(&s_dead, d.status);
    // the record and MR (forward) or this cell's forward result (backward)
    T rec[REC_N], mr[5];
    if (active) {
      const T *st = s_rec + (s % RING) * kStage;
      load_cellrec(st + threadIdx.x * CR_N, (int)threadIdx.x, rec, BACKWARD ? (T *)nullptr : mr);
      if (DQB)
#pragma unroll
        for (int v = 0; v < 5; v++) mr[v] = st[TI * TJ * CR_N + v * TI * TJ + threadIdx.x];
    }
    T ox[5];
    if (active) {
      const int pbuf = (s - 1) & 1;
      T tx[5], ty[5];
      if (halo_edge) {
#pragma unroll
        for (int v = 0; v < 5; v++) tx[v] = hx_cur[v];
      } else if (!recv_x) {
        const int sil = BACKWARD ? il + 1 : il - 1;
#pragma unroll
        for (int v = 0; v < 5; v++) tx[v] = sx[pbuf][sil][jl][v];
      } else if (dsm_recv) {
        // pushed by the producing CTA of the cluster (step s < QN here; the
        // wait above has seen it land)
        const T *src = s_rx + ((s % RX) * TJ + jl) * XW;
#pragma unroll
        for (int v = 0; v < 5; v++) tx[v] = src[v];
      } else {
        bool ok = true;
#pragma unroll
        for (int v = 0; v < 5; v++) { tx[v] = px[0][v]; ok = ok && !is_sentinel(px[0][v]); }
        if (!ok) recv5<T>(xsrc + (long long)kl * 5, tx, d.status, a.spin_limit, &s_dead);
      }
      if (!recv_y) {
        const int sjl = BACKWARD ? jl + 1 : jl - 1;
#pragma unroll
        for (int v = 0; v < 5; v++) ty[v] = sy[pbuf][il][sjl][v];
      } else if (!wall_y) {
        bool ok = true;
#pragma unroll
        for (int v = 0; v < 5; v++) { ty[v] = py[0][v]; ok = ok && !is_sentinel(py[0][v]); }
        if (!ok) recv5<T>(ysrc + (long long)kl * 5, ty, d.status, a.spin_limit, &s_dead);
      } else {
#pragma unroll
        for (int v = 0; v < 5; v++) ty[v] = 0;  // wall ghost row: dQ = 0 there
      }
      const bool zedge = rel == 0;             // z ghost row: dQ = 0 there
      T L[5];
#pragma unroll
      for (int v = 0; v < 5; v++) L[v] = tx[v] * rdx + ty[v] * rdy + (zedge ? (T)0 : carry_z[v]) * rdz;
      const T d11 = rec[R_D11], d22 = rec[R_D22], d51 = rec_d51<T>(rec, rdt);
      T n[5];
      if (!BACKWARD) {
        // Dual_time_stepping.cpp:1289-1293
        T r1 = mr[0] - L[0];
        n[0] = d11 * r1;
        n[1] = d22 * (mr[1] - L[1]);
        n[2] = d22 * (mr[2] - L[2]);
        n[3] = d22 * (mr[3] - L[3]);
        n[4] = d51 * r1 + d22 * (mr[4] - L[4]);
      } else {
        // Dual_time_stepping.cpp:1651-1655 (mr holds this cell's forward result)
        n[0] = mr[0] - d11 * L[0];
        n[1] = mr[1] - d22 * L[1];
        n[2] = mr[2] - d22 * L[2];
        n[3] = mr[3] - d22 * L[3];
        n[4] = mr[4] - (d51 * L[0] + d22 * L[4]);
      }
      const long long c = Met::kChannel ? 0 : ix(d, i, j, 2 + kl);
      T mm[9];
      Met::template dirs<T>(d, s_et, c, jl, mm);
      T oy[5];
      if (Met::kChannel) {
        // the channel's face metrics have one nonzero component per
        // direction (1, etdy, 1 on the x, y, z components), so only the
        // nonzero split entries are formed and applied
        channel_products<T, 0, BACKWARD>(rec, (T)1, n, ox);
        channel_products<T, 1, BACKWARD>(rec, mm[4], n, oy);
        channel_products<T, 2, BACKWARD>(rec, (T)1, n, carry_z);
      } else {
        Split<T> Ax = split_from_record<T>(rec, 0, mm[0], mm[1], mm[2]);
        Split<T> Ay = split_from_record<T>(rec, 1, mm[3], mm[4], mm[5]);
        Split<T> Az = split_from_record<T>(rec, 2, mm[6], mm[7], mm[8]);
        if (BACKWARD) {
          upper_terms<T>(Ax, n, ox);
          upper_terms<T>(Ay, n, oy);
          upper_terms<T>(Az, n, carry_z);
        } else {
          lower_terms<T>(Ax, n, ox);
          lower_terms<T>(Ay, n, oy);
          lower_terms<T>(Az, n, carry_z);
        }
      }
      const int cb = s & 1;
#pragma unroll
      for (int v = 0; v < 5; v++) { sx[cb][il][jl][v] = ox[v]; sy[cb][il][jl][v] = oy[v]; }
      if (send_x && !dsm_send) {
        T *dst = xb + (((long long)tile * TJ + jl) * Nz + kl) * 5;
#pragma unroll
        for (int v = 0; v < 5; v++) __stcg(dst + v, ox[v]);
      }
      if (send_y) {
        T *dst = yb + (((long long)tile * TI + il) * Nz + kl) * 5;
#pragma unroll
        for (int v = 0; v < 5; v++) __stcg(dst + v, oy[v]);
      }
      {
#pragma unroll
        for (int v = 0; v < 5; v++) dq[v][slot0 + (long long)(BACKWARD ? S - 1 - s : s) * (TI * TJ)] = n[v];
        if (BACKWARD && !d.x_open) {
          // lagged halos of the next sweep: plane ie feeds its forward pass,
          // plane 3 its backward pass (an open slab's halos stay zero)
          const long long h = (long long)j * d.dj + 2 + kl;
          if (i == ie)
            for (int v = 0; v < 5; v++) SweepPtrs<T>::hf(a)[v][h] = n[v];
          if (i == 3)
            for (int v = 0; v < 5; v++) SweepPtrs<T>::hb(a)[v][h] = n[v];
        }
      }
    }
    if (dsm_send && send_x && s >= TI - 1) {
      const int q = s - (TI - 1);
      // the slot's previous use must have been read by the consumer (after
      // a give-up the push goes ahead regardless: its values are unused, and
      // an early push only counts its bytes ahead on the consumer's next
      // phase, which the consumer arms once it has seen the previous one)
      const uint32_t eb = tc::smem_addr(&s_empty[q % RX]);
      if (q >= RX && !tc::mbar_wait_cluster(eb, ((q / RX) - 1) & 1, 1) &&
          !tc::mbar_wait_cluster(eb, ((q / RX) - 1) & 1, given_up(&s_dead, d.status) ? 0 : a.spin_limit))
        give_up(&s_dead, d.status);
      {
        // every lane pushes its five words each step (zeros for a cell
        // outside the slab), so the consumer's byte count always completes
        T o5[5];
#pragma unroll
        for (int v = 0; v < 5; v++) o5[v] = active ? ox[v] : (T)0;
        const uint32_t dst = tc::mapa(tc::smem_addr(s_rx + ((q % RX) * TJ + jl) * XW), consumer);
        const uint32_t bar = tc::mapa(tc::smem_addr(&s_full[q % RX]), consumer);
        if (sizeof(T) == 8) {
          tc::st_async_v2(dst, (double)o5[0], (double)o5[1], bar);
          tc::st_async_v2(dst + 16, (double)o5[2], (double)o5[3], bar);
          tc::st_async(dst + 32, (double)o5[4], bar);
        } else {
          tc::st_async_v4(dst, (float)o5[0], (float)o5[1], (float)o5[2], (float)o5[3], bar);
          tc::st_async(dst + 16, (float)o5[4], bar);
        }
      }
    }
    if (pre_x || pre_y) {
#pragma unroll
      for (int p = 0; p + 1 < PD; p++)
#pragma unroll
        for (int v = 0; v < 5; v++) { px[p][v] = px[p + 1][v]; py[p][v] = py[p + 1][v]; }
      if (s + PD < S) preload(s + PD, px[PD - 1], py[PD - 1]);
    }
    if (halo_edge)
#pragma unroll
      for (int v = 0; v < 5; v++) hx_cur[v] = hx_nxt[v];
    __syncthreads();
  }
  // the cluster's CTAs leave together: none while another can still write
  // into its shared memory
  if (CL) tc::cluster_sync();
}

// Dual_time_stepping.cpp:1702-1743 after the last backward pass: the
// primitive update of every interior cell from its final dQ (read from the
// tile-skewed layout), fully parallel rather than inside the wavefront's
// chain of dependent steps, with per-block partial sums of the squared
// increments (:1761-1776).  The divisions by q1, rho, T and J are
// Newton-refined reciprocals (1/J from the table).
//
// A block owns one row il of one tile's TJ columns and UPD_KC consecutive k
// of them.  In the tile-skewed layout those cells lie in UPD_KC + TJ - 1
// consecutive steps, each holding the row's TJ slots side by side: the block
// reads them whole (TJ consecutive words per step and variable) into shared
// memory, then each warp updates 32 consecutive k of one column, so the
// reads and writes of the state in the reference layout are coalesced too.
constexpr int UPD_KC = 32;
template <typename T>
inline unsigned sweep_update_grid_x(const Dev &d) {
  constexpr int TI = SweepTile<T>::TI, TJ = SweepTile<T>::TJ;
  return (unsigned)(((d.nx + TI - 1) / TI) * ((d.ny + TJ - 1) / TJ) * TI);
}
template <typename T>
inline unsigned sweep_update_grid_y(const Dev &d) { return (unsigned)((d.nz + UPD_KC - 1) / UPD_KC); }

template <typename T>
__global__ void __launch_bounds__(256) k_update_skewed(Dev d, SweepArgs a) {
  constexpr int TI = SweepTile<T>::TI, TJ = SweepTile<T>::TJ;
  constexpr int NS = UPD_KC + TJ - 1;   // steps holding the block's cells
  static_assert(256 % TJ == 0 && TJ % 8 == 0, "row staging");
  __shared__ T sdq[5][NS][TJ + 1];       // (+1: the update reads a column down the steps)
  // a wavefront pass that gave up left dQ incomplete: keep the state
  if (*(volatile int *)d.status) return;
  const int ntj = (d.ny + TJ - 1) / TJ, S = d.nz + TI + TJ - 2;
  const int tile = blockIdx.x / TI, il = blockIdx.x % TI;
  const int ta = tile / ntj, tb = tile % ntj;
  const int k0 = blockIdx.y * UPD_KC;    // first k of the block (0-based)
  const int s0 = k0 + il;                // step of the cell (il, jl = 0, k0)
  const long long base = (long long)tile * S * (TI * TJ) + il * TJ;
  T *const *dq = SweepPtrs<T>::dq(a);
  for (int e = threadIdx.x; e < NS * TJ; e += blockDim.x) {
    const int ls = e / TJ, jl = e % TJ, st = s0 + ls;
    if (st < S) {
      const long long g = base + (long long)st * (TI * TJ) + jl;
#pragma unroll
      for (int v = 0; v < 5; v++) sdq[v][ls][jl] = dq[v][g];
    }
  }
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int i = 3 + ta * TI + il;
  double acc[5] = {0, 0, 0, 0, 0};
  for (int jl = warp; jl < TJ; jl += nw) {
    const int j = 2 + tb * TJ + jl, kl = k0 + lane;
    if (i > d.nx + 2 || j > d.ny + 1 || kl >= d.nz) continue;
    const int ls = lane + jl;            // step kl + il + jl, relative to s0
    const long long c = ix(d, i, j, 2 + kl);
    const double J = d.J[c], iJ = d.iJ[c];
    const double q1 = d.U_[0][c], iq1 = nr_rcp(q1);
    const double rhoold = q1 * J;
    const double Uold = d.U_[1][c] * iq1, Vold = d.U_[2][c] * iq1, Wold = d.U_[3][c] * iq1;
    const double VVold = Uold * Uold + Vold * Vold + Wold * Wold;
    const double Pold = (d.U_[4][c] * J - 0.5 * rhoold * VVold) * (KG - 1);
    const double Told = Pold * (iq1 * iJ);   // 1 / rho = 1 / (q1 J)
    const double P = Pold + (double)sdq[0][ls][jl] * J, U = Uold + (double)sdq[1][ls][jl] * J;
    const double V = Vold + (double)sdq[2][ls][jl] * J, W = Wold + (double)sdq[3][ls][jl] * J;
    const double Tn = Told + (double)sdq[4][ls][jl] * J;
    const double rho = P * nr_rcp(Tn), rJ = rho * iJ;
    d.U_[0][c] = rJ;
    d.U_[1][c] = rJ * U;
    d.U_[2][c] = rJ * V;
    d.U_[3][c] = rJ * W;
    d.U_[4][c] = (P * (1 / (KG - 1)) + 0.5 * rho * (U * U + V * V + W * W)) * iJ;
    acc[0] += (rho - rhoold) * (rho - rhoold);
    acc[1] += (U - Uold) * (U - Uold);
    acc[2] += (V - Vold) * (V - Vold);
    acc[3] += (W - Wold) * (W - Wold);
    acc[4] += (Tn - Told) * (Tn - Told);
  }
  block_sum5(acc, d.partial + 5 * ((long long)blockIdx.y * gridDim.x + blockIdx.x));
}

template <typename T>
static void launch_update_skewed(const Dev &d, const SweepArgs &a, cudaStream_t s) {
  k_update_skewed<T><<<dim3(sweep_update_grid_x<T>(d), sweep_update_grid_y<T>(d)), 256, 0, s>>>(d, a);
}
int sweep_update_blocks(const Dev &d, bool mixed) {
  return mixed ? (int)(sweep_update_grid_x<float>(d) * sweep_update_grid_y<float>(d))
               : (int)(sweep_update_grid_x<double>(d) * sweep_update_grid_y<double>(d));
}

// dynamic shared memory of a wavefront pass: the ring of record stages
template <int TI, int TJ, typename T>
constexpr int sweep_smem_bytes(bool backward, bool cluster) {
  return SweepTile<T>::RING * TI * TJ * (CR_N + (backward ? 5 : 0)) * (int)sizeof(T) +
         (cluster ? 8 * TJ * (sizeof(T) == 8 ? 6 : 8) * (int)sizeof(T) : 0);   // the cluster's x hand-over ring
}

// tickets follow the anti-diagonals ta + tb of the tile grid
void sweep_tile_order(int nti, int ntj, std::vector<int> &order) {
  order.clear();
  for (int dsum = 0; dsum <= nti + ntj - 2; dsum++)
    for (int ta = 0; ta < nti; ta++) {
      int tb = dsum - ta;
      if (tb >= 0 && tb < ntj) order.push_back(ta * ntj + tb);
    }
}

// One wavefront pass: ticket reset and sentinel fill of the hand-over
// buffers, the halo products, then the pass itself (with the cluster
// dimension a.cluster_x along x when it is above 1).
template <int TI, int TJ, class Met, typename T>
static void run_one_pass(const Dev &d, const SweepArgs &a, cudaStream_t s, bool backward, bool final_pass) {
  const int nti = (d.nx + TI - 1) / TI, ntj = (d.ny + TJ - 1) / TJ, ntiles = nti * ntj;
  const size_t xbytes = (size_t)ntiles * TJ * d.nz * 5 * sizeof(T), ybytes = (size_t)ntiles * TI * d.nz * 5 * sizeof(T);
  T *xb = sizeof(T) == 8 ? (T *)a.xbuf : (T *)a.xbuff;
  T *yb = sizeof(T) == 8 ? (T *)a.ybuf : (T *)a.ybuff;
  cudaMemsetAsync(a.ticket, 0, sizeof(unsigned int), s);
  cudaMemsetAsync(xb, 0xff, xbytes, s);
  cudaMemsetAsync(yb, 0xff, ybytes, s);
  const dim3 hg((d.nz + 63) / 64, d.ny);
  if (!backward) k_halo_products<Met, false, T><<<hg, 64, 0, s>>>(d, a);
  else k_halo_products<Met, true, T><<<hg, 64, 0, s>>>(d, a);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(ntiles);
  cfg.blockDim = dim3(TI * TJ);
  cfg.dynamicSmemBytes = sweep_smem_bytes<TI, TJ, T>(backward, a.cluster_x > 1);
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  if (a.cluster_x > 1) {
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = a.cluster_x;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
  }
  if (a.cluster_x > 1) {
    if (!backward) cudaLaunchKernelEx(&cfg, k_sweep<TI, TJ, Met, false, T, true>, d, a);
    else cudaLaunchKernelEx(&cfg, k_sweep<TI, TJ, Met, true, T, true>, d, a);
  } else {
    if (!backward) cudaLaunchKernelEx(&cfg, k_sweep<TI, TJ, Met, false, T, false>, d, a);
    else cudaLaunchKernelEx(&cfg, k_sweep<TI, TJ, Met, true, T, false>, d, a);
  }
  if (final_pass) launch_update_skewed<T>(d, a, s);
}

template <int TI, int TJ, class Met, typename T>
static void run_sweeps(const Dev &d, const SweepArgs &a, cudaStream_t s) {
  for (int sweep = 0; sweep < 2; sweep++)
    for (int pass = 0; pass < 2; pass++) run_one_pass<TI, TJ, Met, T>(d, a, s, pass == 1, false);
}

void launch_sweep_pass(const Dev &d, const SweepArgs &a, cudaStream_t s, bool mixed, bool backward, bool final_pass) {
  if (mixed) {
    if (a.channel_metrics) run_one_pass<F32::TI, F32::TJ, MetricsChannel, float>(d, a, s, backward, final_pass);
    else run_one_pass<F32::TI, F32::TJ, MetricsGeneral, float>(d, a, s, backward, final_pass);
  } else {
    if (a.channel_metrics) run_one_pass<F64::TI, F64::TJ, MetricsChannel, double>(d, a, s, backward, final_pass);
    else run_one_pass<F64::TI, F64::TJ, MetricsGeneral, double>(d, a, s, backward, final_pass);
  }
}

// the wavefront kernels' shared memory (static products plus the dynamic
// two-step record buffer) exceeds 48 KB: opt in once, outside any capture
template <class Met, typename T, bool CL>
static cudaError_t opt_in() {
  constexpr int TI = SweepTile<T>::TI, TJ = SweepTile<T>::TJ;
  cudaError_t e = cudaFuncSetAttribute(k_sweep<TI, TJ, Met, false, T, CL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       sweep_smem_bytes<TI, TJ, T>(false, CL));
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_sweep<TI, TJ, Met, true, T, CL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             sweep_smem_bytes<TI, TJ, T>(true, CL));
  return e;
}
cudaError_t sweep_kernel_attributes() {
  cudaError_t e = opt_in<MetricsChannel, double, false>();
  if (e == cudaSuccess) e = opt_in<MetricsGeneral, double, false>();
  if (e == cudaSuccess) e = opt_in<MetricsChannel, float, false>();
  if (e == cudaSuccess) e = opt_in<MetricsGeneral, float, false>();
  if (SweepTile<double>::CLUSTER_MAX > 1) {
    if (e == cudaSuccess) e = opt_in<MetricsChannel, double, true>();
    if (e == cudaSuccess) e = opt_in<MetricsGeneral, double, true>();
  }
  if (SweepTile<float>::CLUSTER_MAX > 1) {
    if (e == cudaSuccess) e = opt_in<MetricsChannel, float, true>();
    if (e == cudaSuccess) e = opt_in<MetricsGeneral, float, true>();
  }
  return e;
}

// The cluster size along x of the passes in type T for a grid of nti x ntj
// tiles: the largest of CLUSTER_MAX, CLUSTER_MAX/2, ... (at least 2) that
// divides nti and of which the device can hold at least one cluster of the
// largest wavefront kernel; 1 (no clusters) otherwise.
template <typename T>
static int cluster_x_for(int nti, int ntj) {
  constexpr int TI = SweepTile<T>::TI, TJ = SweepTile<T>::TJ;
  for (int cx = SweepTile<T>::CLUSTER_MAX; cx >= 2; cx /= 2) {
    if (nti % cx) continue;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nti * ntj);
    cfg.blockDim = dim3(TI * TJ);
    cfg.dynamicSmemBytes = sweep_smem_bytes<TI, TJ, T>(true, true);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cx;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int n = 0;
    if (cudaOccupancyMaxActiveClusters(&n, k_sweep<TI, TJ, MetricsGeneral, true, T, true>, &cfg) != cudaSuccess) {
      cudaGetLastError();
      continue;
    }
    if (n >= 1) return cx;
  }
  return 1;
}
int sweep_cluster_x(int nti, int ntj, bool mixed) {
  return mixed ? cluster_x_for<float>(nti, ntj) : cluster_x_for<double>(nti, ntj);
}

void launch_sweep_update(const Dev &d, const SweepArgs &a, cudaStream_t s, bool mixed) {
  if (mixed) launch_update_skewed<float>(d, a, s);
  else launch_update_skewed<double>(d, a, s);
}

void launch_sweeps(const Dev &d, const SweepArgs &a, cudaStream_t s, bool mixed) {
  if (mixed) {
    if (a.channel_metrics) run_sweeps<F32::TI, F32::TJ, MetricsChannel, float>(d, a, s);
    else run_sweeps<F32::TI, F32::TJ, MetricsGeneral, float>(d, a, s);
  } else {
    if (a.channel_metrics) run_sweeps<F64::TI, F64::TJ, MetricsChannel, double>(d, a, s);
    else run_sweeps<F64::TI, F64::TJ, MetricsGeneral, double>(d, a, s);
  }
}

}  // namespace cgli
