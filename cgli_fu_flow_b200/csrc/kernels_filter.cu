// High-order filter sensor of Filter.cpp:12-1720 (EpX/EpY/EpZ from U_).
//
// Per scale (h: (1,6,1)/8 weights, 2h: (1,2,1)/4) the reference applies six
// iterated filter levels, each an x pass, a y pass on the stretched grid and
// a z pass over full-size scratch arrays, then the high-pass
// fU = 6 L1 - 15 L2 + 20 L3 - 15 L4 + 6 L5 - L6 and E = |u - fu/frho|^2.
//
// Here one kernel launch is one level: a CTA owns an (8 x 32) (j, k) tile
// and marches over a chunk of x planes with a 3-plane ring of the previous
// level in shared memory, so each level reads its input once and writes its
// output once; the x, y and z passes of a plane are done in shared memory.
// The high-pass sum is accumulated in the order the reference writes it as
// the levels are produced, and the last level computes E in its epilogue,
// so no level is kept beyond the next one.  A last kernel forms the face
// ratios and EpX/EpY/EpZ.
//
// Every operation is an explicitly rounded double operation (no fused
// multiply-add) in the reference's evaluation order, so E and the face
// ratios are bit-identical to the reference's and Ep is exact.
#include <cuda_runtime.h>

#include "cgli_filter.h"

namespace cgli {
namespace {

constexpr int FTJ = 8, FTK = 32;                 // output tile (j, k)
constexpr int FRJ = FTJ + 2, FRK = FTK + 2;      // tile with a one-cell halo
constexpr int FCHUNK = 16;                       // x planes per CTA

__device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dvd(double a, double b) { return __ddiv_rn(a, b); }

// (a + w*b + c) * s: the x and z passes (Filter.cpp:160, :227; :841, :902)
template <bool TWO_H>
__device__ __forceinline__ double smooth3(double a, double b, double c) {
  return TWO_H ? mul(0.25, add(add(a, mul(2.0, b)), c)) : mul(0.125, add(add(a, mul(6.0, b)), c));
}

struct LevelArgs {
  const double *P[4];   // previous level (U_ for level 0)
  double *L[4];         // this level (not written by the last level)
  double *acc[4];       // running high-pass sum on the interior planes
  const double *U[4];   // U_: wall and z ghost values and E
  const double *J, *Yp;
  double *E;            // written by the last level
  int nx, ny, nz;       // interior cells
  int X, Y, Z;
  int i0, i1;           // x planes of this level
  int level;            // 0..5
  int wrap;             // read P through its periodic image: the 3-plane
                        // exchange of level 3 on a single periodic slab
                        // (Filter.cpp:447-466) without a copy
};

__device__ __forceinline__ int wrap_plane(int p, int nx) { return p < 3 ? p + nx : (p > nx + 2 ? p - nx : p); }

template <bool TWO_H>
__global__ void __launch_bounds__(FTJ *FTK) k_filter_level(LevelArgs a) {
  extern __shared__ double sm[];
  double *ring = sm;                                // [3][4][FRJ*FRK]
  double *gx = ring + 3 * 4 * FRJ * FRK;            // [4][FRJ*FRK]
  double *gy = gx + 4 * FRJ * FRK;                  // [4][FTJ*FRK]
  double *w1 = gy + 4 * FTJ * FRK;                  // [FTJ*FRK]
  double *w3 = w1 + FTJ * FRK;                      // [FTJ*FRK]
  double *jt = w3 + FTJ * FRK;                      // [FRJ*FRK]

  const int tid = threadIdx.x;
  const int k0 = 2 + blockIdx.x * FTK, j0 = 2 + blockIdx.y * FTJ;
  const int ia = a.i0 + blockIdx.z * FCHUNK;
  const int ib = min(a.i1, ia + FCHUNK - 1);
  const int ny = a.ny + 1, nz = a.nz + 1;           // the reference's ny, nz
  const long long di = (long long)a.Y * a.Z, dj = a.Z;
  const int gend = a.nx + 2;

  auto load_plane = [&](int p) {
    const int slot = p % 3;
    const int src = a.wrap ? wrap_plane(p, a.nx) : p;
    for (int t = tid; t < FRJ * FRK; t += FTJ * FTK) {
      const int j = j0 - 1 + t / FRK, k = k0 - 1 + t % FRK;
      if (j >= 2 && j <= ny && k >= 2 && k <= nz) {
        const long long o = src * di + j * dj + k;
#pragma unroll
        for (int v = 0; v < 4; v++) ring[(slot * 4 + v) * FRJ * FRK + t] = a.P[v][o];
      }
    }
  };

  load_plane(ia - 1);
  load_plane(ia);
  for (int i = ia; i <= ib; i++) {
    __syncthreads();
    load_plane(i + 1);
    // J of plane i on the tile with halo, y-pass weights (Filter.cpp:187-191)
    for (int t = tid; t < FRJ * FRK; t += FTJ * FTK) {
      const int j = j0 - 1 + t / FRK, k = k0 - 1 + t % FRK;
      if (j >= 1 && j <= ny + 1 && k >= 1 && k <= nz + 1) jt[t] = a.J[i * di + j * dj + k];
    }
    for (int t = tid; t < FTJ * FRK; t += FTJ * FTK) {
      const int j = j0 + t / FRK, k = k0 - 1 + t % FRK;
      if (j <= ny && k >= 2 && k <= nz) {
        const long long o = i * di + j * dj + k;
        const double yp = a.Yp[o + dj], yc = a.Yp[o], ym = a.Yp[o - dj];
        const double A = sub(yp, ym), B = sub(yp, yc), C = sub(yc, ym);
        w1[t] = TWO_H ? dvd(B, A) : dvd(mul(2.0, B), A);
        w3[t] = TWO_H ? dvd(C, A) : dvd(mul(2.0, C), A);
      }
    }
    __syncthreads();
    // x pass; the wall rows keep U_ (the scratch arrays start as U_ copies,
    // Filter.cpp:121-138, and the passes only write j = 2..ny)
    const int sm1 = (i - 1) % 3, s0 = i % 3, sp1 = (i + 1) % 3;
    for (int t = tid; t < FRJ * FRK; t += FTJ * FTK) {
      const int j = j0 - 1 + t / FRK, k = k0 - 1 + t % FRK;
      if (k < 2 || k > nz) continue;
      if (j >= 2 && j <= ny) {
#pragma unroll
        for (int v = 0; v < 4; v++)
          gx[v * FRJ * FRK + t] = smooth3<TWO_H>(ring[(sm1 * 4 + v) * FRJ * FRK + t], ring[(s0 * 4 + v) * FRJ * FRK + t],
                                                 ring[(sp1 * 4 + v) * FRJ * FRK + t]);
      } else if (j == 1 || j == ny + 1) {
        const long long o = i * di + j * dj + k;
#pragma unroll
        for (int v = 0; v < 4; v++) gx[v * FRJ * FRK + t] = a.U[v][o];
      }
    }
    __syncthreads();
    // y pass (Filter.cpp:193 for h, :875 for 2h); z ghosts keep U_
    for (int t = tid; t < FTJ * FRK; t += FTJ * FTK) {
      const int r = t / FRK, c = t % FRK;
      const int j = j0 + r, k = k0 - 1 + c;
      if (j > ny) continue;
      if (k >= 2 && k <= nz) {
        const int tm = r * FRK + c, tc = tm + FRK, tp = tc + FRK;
        const double Jm = jt[tm], Jc = jt[tc], Jp = jt[tp];
        const double wa = w1[t], wc = w3[t];
#pragma unroll
        for (int v = 0; v < 4; v++) {
          const double *g = gx + v * FRJ * FRK;
          const double s = add(add(mul(mul(wa, g[tm]), Jm), mul(mul(TWO_H ? 1.0 : 6.0, g[tc]), Jc)), mul(mul(wc, g[tp]), Jp));
          gy[v * FTJ * FRK + t] = TWO_H ? dvd(mul(0.5, s), Jc) : dvd(mul(0.125, s), Jc);
        }
      } else if (k == 1 || k == nz + 1) {
        const long long o = i * di + j * dj + k;
#pragma unroll
        for (int v = 0; v < 4; v++) gy[v * FTJ * FRK + t] = a.U[v][o];
      }
    }
    __syncthreads();
    // z pass, high-pass accumulation, E on the last level
    {
      const int r = tid / FTK, c = tid % FTK;
      const int j = j0 + r, k = k0 + c;
      if (j <= ny && k <= nz) {
        const long long o = i * di + j * dj + k;
        const bool interior = i >= 3 && i <= gend;
        double f[4];
#pragma unroll
        for (int v = 0; v < 4; v++) {
          const double *g = gy + v * FTJ * FRK + r * FRK + c;
          const double L = smooth3<TWO_H>(g[0], g[1], g[2]);
          if (a.level < 5) a.L[v][o] = L;
          if (interior) {
            // Filter.cpp:769 / :1444, left to right
            switch (a.level) {
              case 0: a.acc[v][o] = mul(6.0, L); break;
              case 1: a.acc[v][o] = sub(a.acc[v][o], mul(15.0, L)); break;
              case 2: a.acc[v][o] = add(a.acc[v][o], mul(20.0, L)); break;
              case 3: a.acc[v][o] = sub(a.acc[v][o], mul(15.0, L)); break;
              case 4: a.acc[v][o] = add(a.acc[v][o], mul(6.0, L)); break;
              default: f[v] = sub(a.acc[v][o], L); break;
            }
          }
        }
        if (a.level == 5 && interior) {
          // Filter.cpp:796-800 / :1471-1475
          const double u1 = a.U[0][o];
          const double ue = sub(dvd(a.U[1][o], u1), dvd(f[1], f[0]));
          const double ve = sub(dvd(a.U[2][o], u1), dvd(f[2], f[0]));
          const double we = sub(dvd(a.U[3][o], u1), dvd(f[3], f[0]));
          a.E[o] = add(add(mul(ue, ue), mul(ve, ve)), mul(we, we));
        }
      }
    }
  }
}

struct EpArgs {
  const double *Eh, *E2h;
  double *Ep[3];
  double crit, e_high, e_low;
  int nx, ny, nz, X, Y, Z;
};

// E with the ghost rules of Filter.cpp:1521-1552 (nearest interior cell in
// y and z) and the periodic image in x
__device__ __forceinline__ long long e_at(const EpArgs &a, int i, int j, int k) {
  const int ny = a.ny + 1, nz = a.nz + 1, gend = a.nx + 2;
  if (j == 1) j = 2;
  else if (j == ny + 1) j = ny;
  if (k == 1) k = 2;
  else if (k == nz + 1) k = nz;
  if (i == 2) i = gend;
  else if (i == gend + 1) i = 3;
  return (long long)i * a.Y * a.Z + (long long)j * a.Z + k;
}

__device__ __forceinline__ double ep_of(const EpArgs &a, long long p, long long q) {
  const double r = dvd(add(a.Eh[p], a.Eh[q]), add(a.E2h[p], a.E2h[q]));
  return r >= a.crit ? a.e_high : a.e_low;
}

// EpX: i = 2..gend, j = 1..ny-1, k = 1..nz-1 (Filter.cpp:1564-1585);
// EpY: i = 2..gend-1, j = 1..ny, k = 1..nz-1 (:1593-1615);
// EpZ: i = 2..gend-1, j = 1..ny-1, k = 1..nz (:1624-1645)
__global__ void k_filter_ep(EpArgs a) {
  const int k = 1 + blockIdx.x * blockDim.x + threadIdx.x;
  const int j = 1 + blockIdx.y;
  const int i = 2 + blockIdx.z;
  const int ny = a.ny + 1, nz = a.nz + 1, gend = a.nx + 2;
  if (k > nz) return;
  const long long o = (long long)i * a.Y * a.Z + (long long)j * a.Z + k;
  if (j < ny && k < nz) a.Ep[0][o] = ep_of(a, e_at(a, i, j + 1, k + 1), e_at(a, i + 1, j + 1, k + 1));
  if (i < gend) {
    if (k < nz) a.Ep[1][o] = ep_of(a, e_at(a, i + 1, j, k + 1), e_at(a, i + 1, j + 1, k + 1));
    if (j < ny) a.Ep[2][o] = ep_of(a, e_at(a, i + 1, j + 1, k), e_at(a, i + 1, j + 1, k + 1));
  }
}

constexpr size_t level_smem() {
  return sizeof(double) * (3 * 4 * FRJ * FRK + 4 * FRJ * FRK + 4 * FTJ * FRK + 2 * FTJ * FRK + FRJ * FRK);
}

}  // namespace

int filter_smem_bytes() { return (int)level_smem(); }

cudaError_t launch_filter(const Dev &d, const FilterBufs &b, double crit, double e_high, double e_low,
                          cudaStream_t s) {
  cudaError_t err = cudaFuncSetAttribute(k_filter_level<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)level_smem());
  if (err == cudaSuccess)
    err = cudaFuncSetAttribute(k_filter_level<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)level_smem());
  if (err != cudaSuccess) return err;
  const int gend = d.nx + 2;
  const int range[6][2] = {{1, gend + 2}, {2, gend + 1}, {3, gend}, {1, gend + 2}, {2, gend + 1}, {3, gend}};
  for (int sc = 0; sc < 2; sc++) {
    LevelArgs a{};
    for (int lev = 0; lev < 6; lev++) {
      for (int v = 0; v < 4; v++) {
        a.P[v] = lev == 0 ? d.U_[v] : b.lev[(lev - 1) & 1][v];
        a.L[v] = b.lev[lev & 1][v];
        a.acc[v] = b.acc[v];
        a.U[v] = d.U_[v];
      }
      a.J = d.J;
      a.Yp = b.yp;
      a.E = sc == 0 ? b.eh : b.e2h;
      a.nx = d.nx; a.ny = d.ny; a.nz = d.nz;
      a.X = d.X; a.Y = d.Y; a.Z = d.Z;
      a.i0 = range[lev][0];
      a.i1 = range[lev][1];
      a.level = lev;
      a.wrap = lev == 3;
      dim3 grid((d.nz + FTK - 1) / FTK, (d.ny + FTJ - 1) / FTJ, (a.i1 - a.i0 + 1 + FCHUNK - 1) / FCHUNK);
      if (sc == 0) k_filter_level<false><<<grid, FTJ * FTK, level_smem(), s>>>(a);
      else k_filter_level<true><<<grid, FTJ * FTK, level_smem(), s>>>(a);
    }
  }
  EpArgs e{};
  e.Eh = b.eh; e.E2h = b.e2h;
  for (int f = 0; f < 3; f++) e.Ep[f] = b.ep[f];
  e.crit = crit; e.e_high = e_high; e.e_low = e_low;
  e.nx = d.nx; e.ny = d.ny; e.nz = d.nz; e.X = d.X; e.Y = d.Y; e.Z = d.Z;
  // j = 1..ny (Y_out + 1 rows cover every face range), i = 2..gend
  dim3 grid((d.nz + 1 + 127) / 128, d.ny + 1, d.nx + 1);
  k_filter_ep<<<grid, 128, 0, s>>>(e);
  return cudaGetLastError();
}

}  // namespace cgli
