// LU-SGS forward / backward sweeps as persistent tile wavefronts.
//
// The reference visits the cells of one x-slab hyperplane by hyperplane
// (i+j+k = m, Dual_time_stepping.cpp:983-1664), one OpenMP barrier per
// plane.  A cell's update depends only on its three upwind neighbours, so
// any order that respects that dependency graph gives the same numbers.
// Here each CTA owns a TI x TJ tile of (i, j) columns and marches along k
// (the contiguous direction, so every thread streams its own k-line).
// Thread (il, jl) handles cell k = 2 + s - il - jl at step s: its i- and
// j-neighbours were handled by the neighbouring threads one step earlier and
// hand over their lower-triangular products through shared memory; its
// k-neighbour is its own previous step.  Tiles exchange the products of their
// last row / column through global buffers, guarded by per-tile progress
// counters with a bounded spin (no unbounded waits: on timeout the kernel
// records CGLI_ETIMEOUT in the status word and carries on).  Tiles take
// tickets in an order where every dependency holds a smaller ticket, so a
// waiting CTA only waits on CTAs that are already running.
//
// Every cell computes its own primitive state, diagonal and split Jacobians
// once per pass (the reference recomputes each neighbour's Jacobians for
// every consumer), and each product A+ . dQ is formed by the cell that owns A+.
//
// The periodic x halo keeps the reference's lag: the forward pass at i = 3
// uses dQ of plane Nx+2 as it was at the start of the sweep (halo_f), the
// backward pass at i = Nx+2 uses dQ of plane 3 (halo_b).  The backward pass of
// the first sweep writes both halos for the second sweep; the final backward
// pass also applies the primitive update of Dual_time_stepping.cpp:1702-1743
// and accumulates the squared increments of the residual norms.
#include "cgli_dev.cuh"
#include "cgli_launch.h"

namespace cgli {

// cell metrics: general 3-D arrays, or a grid uniform in x and z (channel)
// whose only varying terms are J(j) and etdy(j)
struct MetricsGeneral {
  __device__ __forceinline__ static void load(const Dev &d, const SweepArgs &, long long c, int, double &J, double mm[9]) {
    J = d.J[c];
#pragma unroll
    for (int v = 0; v < 9; v++) mm[v] = d.m[v][c];
  }
};
struct MetricsChannel {
  __device__ __forceinline__ static void load(const Dev &, const SweepArgs &a, long long, int j, double &J, double mm[9]) {
    J = a.Jtab[j];
    mm[0] = 1; mm[1] = 0; mm[2] = 0;
    mm[3] = 0; mm[4] = a.etdytab[j]; mm[5] = 0;
    mm[6] = 0; mm[7] = 0; mm[8] = 1;
  }
};

// bounded wait until counter >= need; thread 0 only
__device__ __forceinline__ void wait_counter(const unsigned long long *ctr, unsigned long long need,
                                             unsigned long long &cache, int *status, int spin_limit) {
  if (cache >= need) return;
  int it = 0;
  while (true) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(ctr) : "memory");
    cache = v;
    if (v >= need) return;
    if (++it > spin_limit) {
      atomicExch(status, CGLI_TIMEOUT_CODE);
      cache = need;  // give up waiting; results of this pass are invalid
      return;
    }
    __nanosleep(64);
  }
}

__device__ __forceinline__ void publish(unsigned long long *ctr, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(ctr), "l"(v) : "memory");
}

template <int TI, int TJ, class Met, bool BACKWARD>
__global__ void __launch_bounds__(TI *TJ) k_sweep(Dev d, SweepArgs a) {
  __shared__ double sx[2][TI][TJ][5];   // i-direction products, double-buffered by step parity
  __shared__ double sy[2][TI][TJ][5];   // j-direction products
  __shared__ int s_tile;
  __shared__ double s_red[5];
  const int il = threadIdx.x / TJ, jl = threadIdx.x % TJ;
  const int nti = (d.nx + TI - 1) / TI, ntj = (d.ny + TJ - 1) / TJ, ntiles = nti * ntj;
  if (threadIdx.x == 0) s_tile = (int)atomicAdd(a.ticket, 1u);
  __syncthreads();
  const int ticket = s_tile;
  if (ticket >= ntiles) return;
  // tickets follow anti-diagonals of the tile grid (reversed for the backward pass)
  const int tile = a.order[BACKWARD ? ntiles - 1 - ticket : ticket];
  const int ta = tile / ntj, tb = tile % ntj;
  const int ie = d.nx + 2, jn = d.ny + 1;
  const int i = 3 + ta * TI + il, j = 2 + tb * TJ + jl;
  const bool inside = (i <= ie) && (j <= jn);
  const int Nz = d.nz;
  const int S = Nz + TI - 1 + TJ - 1;
  // neighbouring tiles this one depends on
  const int pa = BACKWARD ? ta + 1 : ta - 1, pb = BACKWARD ? tb + 1 : tb - 1;
  const bool has_pa = pa >= 0 && pa < nti, has_pb = pb >= 0 && pb < ntj;
  const int tile_pa = pa * ntj + tb, tile_pb = ta * ntj + pb;
  // threads on the tile edge that read from / write to the neighbour tiles
  const bool recv_x = BACKWARD ? (il == TI - 1 || i == ie) : (il == 0);
  const bool recv_y = BACKWARD ? (jl == TJ - 1 || j == jn) : (jl == 0);
  const bool send_x = BACKWARD ? (il == 0) : (il == TI - 1);
  const bool send_y = BACKWARD ? (jl == 0) : (jl == TJ - 1);
  const double rdx = 1.0 / d.dxi, rdy = 1.0 / d.det, rdz = 1.0 / d.dzt;
  (void)rdx; (void)rdy; (void)rdz;
  unsigned long long cache_a = 0, cache_b = 0;
  double carry_z[5] = {0, 0, 0, 0, 0};
  double acc[5] = {0, 0, 0, 0, 0};
  const bool last_x_tile = BACKWARD ? (ta == nti - 1) : (ta == 0);

  for (int s = 0; s < S; s++) {
    const int rel = BACKWARD ? s - (TI - 1 - il) - (TJ - 1 - jl) : s - il - jl;
    const int kl = BACKWARD ? Nz - 1 - rel : rel;
    const bool active = inside && rel >= 0 && rel < Nz;
    const int k = 2 + kl;
    const long long c = active ? ix(d, i, j, k) : 0;
    // own state and coefficients (independent of the sweep)
    CPrim<double> q;
    Diag<double> dg;
    Split<double> Ax, Ay, Az;
    double mr[5];
    double J = 1.0;
    if (active) {
      double mm[9];
      Met::load(d, a, c, j, J, mm);
      q = cprim<double>(d.U_[0][c], d.U_[1][c], d.U_[2][c], d.U_[3][c], d.U_[4][c], J, d.e);
      dg = diag<double>(q, mm, d.dxi, d.det, d.dzt, d.dt);
      Ax = split<double>(q, mm[0], mm[1], mm[2], true);
      Ay = split<double>(q, mm[3], mm[4], mm[5], false);
      Az = split<double>(q, mm[6], mm[7], mm[8], false);
#pragma unroll
      for (int v = 0; v < 5; v++) mr[v] = BACKWARD ? a.dq[v][c] : d.MR[v][c];
    }
    // wait for the neighbouring tiles' products of this step
    if (threadIdx.x == 0) {
      if (has_pa) wait_counter(a.prog + tile_pa, (unsigned long long)min(s + TI, S), cache_a, d.status, a.spin_limit);
      if (has_pb) wait_counter(a.prog + tile_pb, (unsigned long long)min(s + TJ, S), cache_b, d.status, a.spin_limit);
    }
    __syncthreads();
    if (active) {
      double tx[5], ty[5], tz[5];
      const int pb_ = (s - 1) & 1;
      // x neighbour
      if (!recv_x) {
        const int sil = BACKWARD ? il + 1 : il - 1;
#pragma unroll
        for (int v = 0; v < 5; v++) tx[v] = sx[pb_][sil][jl][v];
      } else if (last_x_tile && (BACKWARD ? i == ie : i == 3)) {
        // periodic lagged halo: the neighbour is plane 2 (forward) / ie+1 (backward)
        const long long cn = BACKWARD ? c + d.di : c - d.di;
        double Jn, mn[9];
        Met::load(d, a, cn, j, Jn, mn);
        CPrim<double> qn = cprim<double>(d.U_[0][cn], d.U_[1][cn], d.U_[2][cn], d.U_[3][cn], d.U_[4][cn], Jn, d.e);
        Split<double> An = split<double>(qn, mn[0], mn[1], mn[2], true);
        const long long h = (long long)j * d.dj + k;
        double nh[5];
#pragma unroll
        for (int v = 0; v < 5; v++) nh[v] = BACKWARD ? a.halo_b[v][h] : a.halo_f[v][h];
        if (BACKWARD) upper_terms<double>(An, nh, tx); else lower_terms<double>(An, nh, tx);
      } else if (has_pa) {
        const double *src = a.xbuf + (((long long)tile_pa * TJ + jl) * Nz + kl) * 5;
#pragma unroll
        for (int v = 0; v < 5; v++) tx[v] = __ldcg(src + v);
      } else {
#pragma unroll
        for (int v = 0; v < 5; v++) tx[v] = 0;
      }
      // y neighbour
      if (!recv_y) {
        const int sjl = BACKWARD ? jl + 1 : jl - 1;
#pragma unroll
        for (int v = 0; v < 5; v++) ty[v] = sy[pb_][il][sjl][v];
      } else if (has_pb && (BACKWARD ? j < jn : j > 2)) {
        const double *src = a.ybuf + (((long long)tile_pb * TI + il) * Nz + kl) * 5;
#pragma unroll
        for (int v = 0; v < 5; v++) ty[v] = __ldcg(src + v);
      } else {
#pragma unroll
        for (int v = 0; v < 5; v++) ty[v] = 0;  // wall ghost row: dQ = 0 there
      }
      // k neighbour: own previous step (zero next to the z ghost rows)
#pragma unroll
      for (int v = 0; v < 5; v++) tz[v] = (rel > 0) ? carry_z[v] : 0.0;
      double L[5];
#pragma unroll
      for (int v = 0; v < 5; v++) L[v] = tx[v] / d.dxi + ty[v] / d.det + tz[v] / d.dzt;
      double n[5];
      if (!BACKWARD) {
        // Dual_time_stepping.cpp:1289-1293
        double r1 = mr[0] - L[0];
        n[0] = dg.d11 * r1;
        n[1] = dg.d22 * (mr[1] - L[1]);
        n[2] = dg.d22 * (mr[2] - L[2]);
        n[3] = dg.d22 * (mr[3] - L[3]);
        n[4] = dg.d51 * r1 + dg.d22 * (mr[4] - L[4]);
      } else {
        // Dual_time_stepping.cpp:1651-1655 (mr holds this cell's forward result)
        n[0] = mr[0] - dg.d11 * L[0];
        n[1] = mr[1] - dg.d22 * L[1];
        n[2] = mr[2] - dg.d22 * L[2];
        n[3] = mr[3] - dg.d22 * L[3];
        n[4] = mr[4] - (dg.d51 * L[0] + dg.d22 * L[4]);
      }
      if (BACKWARD && a.final_pass) {
        // Dual_time_stepping.cpp:1702-1743: primitive update in place
        double P = q.P + n[0] * J, U = q.u + n[1] * J, V = q.v + n[2] * J, W = q.w + n[3] * J;
        double T = q.Tt + n[4] * J;
        double rho = P / T;
        d.U_[0][c] = rho / J;
        d.U_[1][c] = rho * U / J;
        d.U_[2][c] = rho * V / J;
        d.U_[3][c] = rho * W / J;
        d.U_[4][c] = (P / (KG - 1) + 0.5 * rho * (U * U + V * V + W * W)) / J;
        acc[0] += (rho - q.rho) * (rho - q.rho);
        acc[1] += (U - q.u) * (U - q.u);
        acc[2] += (V - q.v) * (V - q.v);
        acc[3] += (W - q.w) * (W - q.w);
        acc[4] += (T - q.Tt) * (T - q.Tt);
      } else {
#pragma unroll
        for (int v = 0; v < 5; v++) a.dq[v][c] = n[v];
        if (BACKWARD) {
          // lagged halos of the next sweep: plane ie feeds its forward pass,
          // plane 3 its backward pass
          const long long h = (long long)j * d.dj + k;
          if (i == ie)
            for (int v = 0; v < 5; v++) a.halo_f[v][h] = n[v];
          if (i == 3)
            for (int v = 0; v < 5; v++) a.halo_b[v][h] = n[v];
        }
      }
      // products handed to the downwind neighbours
      double ox[5], oy[5];
      if (BACKWARD) {
        upper_terms<double>(Ax, n, ox);
        upper_terms<double>(Ay, n, oy);
        upper_terms<double>(Az, n, carry_z);
      } else {
        lower_terms<double>(Ax, n, ox);
        lower_terms<double>(Ay, n, oy);
        lower_terms<double>(Az, n, carry_z);
      }
      const int cb = s & 1;
      if (send_x) {
        double *dst = a.xbuf + (((long long)tile * TJ + jl) * Nz + kl) * 5;
#pragma unroll
        for (int v = 0; v < 5; v++) __stcg(dst + v, ox[v]);
      }
#pragma unroll
      for (int v = 0; v < 5; v++) sx[cb][il][jl][v] = ox[v];
      if (send_y) {
        double *dst = a.ybuf + (((long long)tile * TI + il) * Nz + kl) * 5;
#pragma unroll
        for (int v = 0; v < 5; v++) __stcg(dst + v, oy[v]);
      }
#pragma unroll
      for (int v = 0; v < 5; v++) sy[cb][il][jl][v] = oy[v];
      if (send_x || send_y) __threadfence();
    }
    __syncthreads();
    if (threadIdx.x == 0) publish(a.prog + tile, (unsigned long long)(s + 1));
  }
  if (BACKWARD && a.final_pass) {
    __syncthreads();
    block_sum5(acc, s_red);
    __syncthreads();
    if (threadIdx.x == 0)
      for (int v = 0; v < 5; v++) d.partial[5 * (long long)tile + v] = s_red[v];
  }
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

template <int TI, int TJ, class Met>
static void run_sweeps(const Dev &d, const SweepArgs &a, cudaStream_t s) {
  const int nti = (d.nx + TI - 1) / TI, ntj = (d.ny + TJ - 1) / TJ, ntiles = nti * ntj;
  for (int sweep = 0; sweep < 2; sweep++) {
    SweepArgs f = a, b = a;
    f.final_pass = 0;
    b.final_pass = sweep == 1;
    cudaMemsetAsync(a.ticket, 0, sizeof(unsigned int), s);
    cudaMemsetAsync(a.prog, 0, sizeof(unsigned long long) * ntiles, s);
    k_sweep<TI, TJ, Met, false><<<ntiles, TI * TJ, 0, s>>>(d, f);
    cudaMemsetAsync(a.ticket, 0, sizeof(unsigned int), s);
    cudaMemsetAsync(a.prog, 0, sizeof(unsigned long long) * ntiles, s);
    k_sweep<TI, TJ, Met, true><<<ntiles, TI * TJ, 0, s>>>(d, b);
  }
}

void launch_sweeps(const Dev &d, const SweepArgs &a, cudaStream_t s) {
  if (a.channel_metrics) run_sweeps<SWEEP_TI, SWEEP_TJ, MetricsChannel>(d, a, s);
  else run_sweeps<SWEEP_TI, SWEEP_TJ, MetricsGeneral>(d, a, s);
}

}  // namespace cgli
