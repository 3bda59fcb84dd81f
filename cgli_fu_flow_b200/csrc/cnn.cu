// Learned initial guess for the inner iterations: a 3-D convolutional network
// (15 -> 32 -> 32 -> 32 -> 32 -> 5 channels, 3x3x3 kernels, GELU, periodic
// in x and z, zero padded at the walls) that predicts the correction to
// second-order extrapolation of Q^(n+1) from Q^n, Q^(n-1), Q^(n-2).  There is
// no counterpart in the reference; this file holds its tensor-core training
// and inference kernels and their C ABI.
//
// Inputs per variable: the level Q^n (less its mean, over its spread), and
// its first and second time differences Q^n - Q^(n-1) and
// Q^n - 2 Q^(n-1) + Q^(n-2), each over its own RMS.  A step changes Q by
// about one part in the grid size of its spatial spread, which is below the
// resolution of a BF16 level; the differences, formed in FP32 / FP64 before
// the conversion, keep that information.
//
// Data layout.  Activations and gradients are BF16, channel-last, on the
// interior grid padded by one cell in every direction: [Nx+2][Ny+2][Nz+2][32]
// (64 bytes per cell; layer inputs with fewer channels are zero padded to
// 32).  The x and z halos hold periodic copies, the y halo rows stay zero.
//
// Convolution = implicit GEMM on tcgen05.  One CTA owns a column of
// 4 (y) x 32 (z) cells and marches over a chunk of x planes; an output tile
// is the 128 cells of one x plane (M = 128), 32 output channels,
// K = 27 taps x 32 input channels.  A TMA producer warp loads, per x plane,
// three copies of the 6 (y) x 32 (z) x 32-channel halo box shifted by
// dz = -1, 0, +1, 64-byte swizzled, into a 4-plane ring: the rows of tap
// (dy, dz) of a plane are then the 128 consecutive rows starting at row
// 32 dy of copy dz, a shared-memory descriptor with no data movement.
// Plane p is the A operand of the dx = 0, 1, 2 taps of output tiles p, p-1,
// p-2, so one MMA per (dy, dz, K half) multiplies it by the three dx blocks
// of weights side by side (N = 96; all 27 taps stay resident in shared
// memory, stored (dy, dz)-major with the dx blocks adjacent) into the three
// tiles' accumulators: a ring of eight 32-column TMEM slots in which tile
// q - 1 sits 32 columns after tile q (the block is split where the ring
// wraps, and narrowed where a tile does not exist).  Each plane is read by
// its 18 MMAs once, and its ring slot is free as soon as they complete.
// Four epilogue warps drain each finished tile (tcgen05.ld), zero its slot
// for its next use, add the bias and apply GELU (forward), or multiply by
// GELU'(z) of the layer below (input gradient, same kernel with the
// transposed, flipped weights).
//
// Weight gradient = the same operand images read as MN-major matrices:
// D[(dy, c_in)][c_out] = sum over cells of X(shifted by (dx, dy, dz))[c_in]
// x dZ[c_out], M = 4 dy-shifts x 32 = 128 (the fourth shift is discarded),
// N = 32, K = the CTA's cells; the nine (dx, dz) groups accumulate in 288
// TMEM columns over the CTA's whole chunk, then a deterministic reduction
// over CTAs gives dW.
//
// Every wait on an mbarrier is bounded; on a timeout the kernel records an
// error in the status word, lets its copies in flight finish (bounded),
// frees its TMEM and returns.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cgli_fu_flow.h"
#include "cgli_launch.h"
#include "cnn.h"
#include "tc_sm100.cuh"

namespace cgli {
namespace {

using bf16 = __nv_bfloat16;

constexpr int NL = 5;                                  // layers
constexpr int CIN[NL] = {15, 32, 32, 32, 32};
constexpr int COUT[NL] = {32, 32, 32, 32, 5};
constexpr int CH = 32;                                 // padded channels (64-byte rows)
constexpr int ROW = CH * 2;                            // bytes per cell row
constexpr int FWD_COPY = 6 * 32 * ROW;                 // 12288: 6 y rows x 32 z cells
constexpr int FWD_PLANE = 3 * FWD_COPY;                // three dz copies
constexpr int W_BYTES = 27 * 32 * ROW;                 // 55296: all taps of one layer
constexpr int WG_COPY = 7 * 32 * ROW;                  // 14336: 7 y rows (the 4th dy shift)
constexpr int WG_PLANE = 3 * WG_COPY;
constexpr int G_TILE = 4 * 32 * ROW;                   // 8192: dZ of one output tile
constexpr int CONV_SLOTS = 8;                          // TMEM accumulators of k_conv (32 columns each)
constexpr int CONV_SMEM = 1024 + 4 * FWD_PLANE + W_BYTES + 512;
constexpr int WGRAD_SMEM = 1024 + 4 * WG_PLANE + 2 * G_TILE + 256;

constexpr uint32_t IDESC_WG = tc::idesc_bf16(128, 32, true, true);
constexpr int SPIN = 1 << 22;

enum ConvMode { CONV_HIDDEN = 0, CONV_HIDDEN_INFER = 1, CONV_OUT = 2, CONV_DGRAD = 3 };

struct ConvArgs {
  const float *bias;        // 32 (forward)
  bf16 *act_out;            // padded BF16 output (hidden / input gradient)
  bf16 *zbuf;               // HIDDEN: pre-activation written; DGRAD: pre-activation of the layer below, read
  float *out32;             // CONV_OUT: [nx][ny][nz][8]
  int nx, ny, nz, Yp, Zp;
  int xchunk;
  int spin;
  int *status;
};

struct WgradArgs {
  float *partial;           // [blocks][27][32 cout][32 cin]
  int nx, ny, nz;
  int xchunk;
  int spin;
  int *status;
};

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float z) {
  return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

__device__ __forceinline__ uint32_t pack2(float a, float b) {
  __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<uint32_t *>(&h);
}
__device__ __forceinline__ void unpack8(uint4 u, float f[8]) {
  const __nv_bfloat162 *h = reinterpret_cast<const __nv_bfloat162 *>(&u);
#pragma unroll
  for (int i = 0; i < 4; i++) {
    float2 t = __bfloat1622float2(h[i]);
    f[2 * i] = t.x;
    f[2 * i + 1] = t.y;
  }
}

// all lanes wait; the warp proceeds only if every lane saw the phase
__device__ __forceinline__ bool warp_wait(uint32_t bar, uint32_t parity, int limit, volatile int *abort_flag) {
  bool ok = false;
  for (int n = 0; n < limit; n++) {
    if (tc::mbar_try(bar, parity)) { ok = true; break; }
    if (*abort_flag) break;
    if (n > 32) __nanosleep(128);
  }
  return __all_sync(0xffffffffu, ok);
}
__device__ __forceinline__ bool one_wait(uint32_t bar, uint32_t parity, int limit, volatile int *abort_flag) {
  for (int n = 0; n < limit; n++) {
    if (tc::mbar_try(bar, parity)) return true;
    if (*abort_flag) return false;
    if (n > 32) __nanosleep(128);
  }
  return false;
}

// ---------------------------------------------------------------- conv
template <int MODE>
__global__ void __launch_bounds__(192, 1)
    k_conv(const __grid_constant__ CUtensorMap in_map, const __grid_constant__ CUtensorMap w_map, ConvArgs a) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = tc::smem_addr(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t *sb = smem_raw + (base - raw);
  const uint32_t A0 = base;
  const uint32_t W0 = base + 4 * FWD_PLANE;
  uint64_t *bars = reinterpret_cast<uint64_t *>(sb + 4 * FWD_PLANE + W_BYTES);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 32);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);
  auto bar = [&](int i) { return tc::smem_addr(bars + i); };
  constexpr int RS = CONV_SLOTS;
  enum { FULL = 0, FREE = 4, ACCF = 8, ACCE = 8 + RS, WBAR = 8 + 2 * RS, NBAR = 9 + 2 * RS };
  static_assert(NBAR <= 32, "barrier area");

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nyb = a.ny >> 2;
  const int yb = blockIdx.x % nyb, zb = blockIdx.x / nyb;
  const int xa = blockIdx.y * a.xchunk;
  const int n = min(a.xchunk, a.nx - xa);

  if (threadIdx.x == 0) {
    for (int i = 0; i < NBAR; i++) tc::mbar_init(bar(i), (i >= ACCE && i < ACCE + RS) ? 128 : 1);
    *abort_flag = 0;
    tc::mbar_fence_init();
  }
  if (warp == 1) {
    tc::tmem_alloc(tc::smem_addr(tmem_slot), 32 * RS);
    tc::tmem_relinquish();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tmem_slot;
  // every accumulator starts at zero (the MMAs only accumulate; the epilogue
  // zeroes a slot again once it has read it)
  if (warp >= 2)
    for (int sl = 0; sl < RS; sl++) tc::tmem_zero_32x32(tmem + ((uint32_t)((warp & 3) * 32) << 16) + 32 * sl);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  bool ok = true;

  if (warp == 0) {
    if (lane == 0) {
      // producer: weights once, then x planes into the ring
      tc::tma_prefetch_desc(&in_map);
      tc::tma_prefetch_desc(&w_map);
      tc::mbar_expect_tx(bar(WBAR), W_BYTES);
      for (int r = 0; r < 4; r++) tc::tma_load_2d(W0 + r * 216 * ROW, &w_map, bar(WBAR), 0, r * 216);
      int issued = 0;
      for (int p = 0; p < n + 2; p++) {
        const int s = p & 3;
        if (p >= 4 && !one_wait(bar(FREE + s), ((p >> 2) - 1) & 1, a.spin, abort_flag)) { ok = false; break; }
        tc::mbar_expect_tx(bar(FULL + s), FWD_PLANE);
        for (int dz = 0; dz < 3; dz++)
          tc::tma_load_4d(A0 + s * FWD_PLANE + dz * FWD_COPY, &in_map, bar(FULL + s), 0, zb * 32 + dz, yb * 4, xa + p);
        issued = p + 1;
      }
      if (!ok) *abort_flag = 1;
      // copies in flight complete before the CTA leaves (weights, last planes)
      tc::mbar_wait(bar(WBAR), 0, a.spin);
      for (int p = max(0, issued - 4); p < issued; p++) tc::mbar_wait(bar(FULL + (p & 3)), (p >> 2) & 1, a.spin);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // Plane p (x = xa + p - 1) is the A operand of the taps dx = 0, 1, 2 of
      // output tiles p, p - 1, p - 2.  For each (dy, dz, K half) one MMA
      // multiplies it by the three dx blocks of weights side by side (N = 96)
      // into the three tiles' accumulators, which sit in adjacent TMEM slots
      // (tile q in slot q % RS at column 32 (RS - 1 - q % RS), so tile q - 1
      // is 32 columns to the right of tile q); where the slots wrap, or only
      // one or two of the tiles exist (the first and last planes), the block
      // is split or narrowed.  A plane is read from shared memory once, by
      // 18 MMAs, and its ring slot is free as soon as they complete.
      int last = -1;
      const uint64_t adesc = tc::desc_sw64(A0, 16, 512), wdesc = tc::desc_sw64(W0, 16, 512);
      if (!one_wait(bar(WBAR), 0, a.spin, abort_flag)) ok = false;
      for (int p = 0; p < n + 2 && ok; p++) {
        const int lo = p > n - 1 ? p - (n - 1) : 0, hi = p < 2 ? p : 2;   // dx whose tile p - dx exists
        // tile p (dx = 0) starts in slot p % RS, last used by tile p - RS
        if (lo == 0 && p >= RS && !one_wait(bar(ACCE + p % RS), ((p / RS) - 1) & 1, a.spin, abort_flag)) {
          ok = false;
          break;
        }
        if (!one_wait(bar(FULL + (p & 3)), (p >> 2) & 1, a.spin, abort_flag)) { ok = false; break; }
        tc::fence_after_sync();
        const uint64_t ap = adesc + (uint64_t)((p & 3) * (FWD_PLANE >> 4));
        for (int d0 = lo; d0 <= hi;) {
          int d1 = d0;   // the segment d0..d1 of adjacent slots
          while (d1 < hi && (p - d1) % RS != 0) d1++;
          const uint32_t dcol = tmem + 32 * (RS - 1 - (p - d0) % RS);
          const uint32_t idesc = d1 == d0 ? tc::idesc_bf16(128, 32, false, false)
                                 : d1 == d0 + 1 ? tc::idesc_bf16(128, 64, false, false)
                                                : tc::idesc_bf16(128, 96, false, false);
          const uint64_t wp = wdesc + (uint64_t)((d0 * 32 * ROW) >> 4);
#pragma unroll
          for (int g = 0; g < 9; g++) {
            const int dy = g / 3, dz = g % 3;
            const uint64_t a_d = ap + (uint64_t)((dz * FWD_COPY + dy * 32 * ROW) >> 4);
            const uint64_t w_d = wp + (uint64_t)((g * 96 * ROW) >> 4);
#pragma unroll
            for (int kk = 0; kk < 2; kk++) tc::mma_f16(dcol, a_d + 2 * kk, w_d + 2 * kk, idesc, 1u);
          }
          d0 = d1 + 1;
        }
        tc::mma_commit(bar(FREE + (p & 3)));
        if (hi == 2) tc::mma_commit(bar(ACCF + (p - 2) % RS));   // tile p - 2 is complete
        last = p;
      }
      if (!ok) *abort_flag = 1;
      // the MMAs issued complete before TMEM is released
      if (last >= 0) tc::mbar_wait(bar(FREE + (last & 3)), (last >> 2) & 1, a.spin);
    }
  } else {
    // epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31
    const int ew = warp & 3;
    const int y = yb * 4 + ew, z = zb * 32 + lane;
    float bias[32];
    if (MODE != CONV_DGRAD) {
#pragma unroll
      for (int c = 0; c < 32; c++) bias[c] = __ldg(a.bias + c);
    }
    for (int t = 0; t < n; t++) {
      const int sl = t % RS;
      if (!warp_wait(bar(ACCF + sl), (t / RS) & 1, a.spin, abort_flag)) { ok = false; break; }
      tc::fence_after_sync();
      float acc[32];
      const uint32_t ta = tmem + ((uint32_t)(ew * 32) << 16) + 32 * (RS - 1 - sl);
      tc::tmem_ld_32x32(ta, acc);
      tc::tmem_zero_32x32(ta);
      tc::fence_before_sync();
      tc::mbar_arrive(bar(ACCE + sl));
      const int x = xa + t;
      const size_t pidx = ((size_t)(x + 1) * a.Yp + (y + 1)) * a.Zp + (z + 1);
      if (MODE == CONV_OUT) {
        float4 *o = reinterpret_cast<float4 *>(a.out32 + (((size_t)x * a.ny + y) * a.nz + z) * 8);
        o[0] = make_float4(acc[0] + bias[0], acc[1] + bias[1], acc[2] + bias[2], acc[3] + bias[3]);
        o[1] = make_float4(acc[4] + bias[4], acc[5] + bias[5], acc[6] + bias[6], acc[7] + bias[7]);
      } else if (MODE == CONV_DGRAD) {
        const uint4 *zp = reinterpret_cast<const uint4 *>(a.zbuf + pidx * CH);
        uint4 *o = reinterpret_cast<uint4 *>(a.act_out + pidx * CH);
#pragma unroll
        for (int q = 0; q < 4; q++) {
          float zf[8];
          unpack8(zp[q], zf);
          uint4 u;
          u.x = pack2(acc[8 * q + 0] * gelu_grad(zf[0]), acc[8 * q + 1] * gelu_grad(zf[1]));
          u.y = pack2(acc[8 * q + 2] * gelu_grad(zf[2]), acc[8 * q + 3] * gelu_grad(zf[3]));
          u.z = pack2(acc[8 * q + 4] * gelu_grad(zf[4]), acc[8 * q + 5] * gelu_grad(zf[5]));
          u.w = pack2(acc[8 * q + 6] * gelu_grad(zf[6]), acc[8 * q + 7] * gelu_grad(zf[7]));
          o[q] = u;
        }
      } else {
        uint4 *o = reinterpret_cast<uint4 *>(a.act_out + pidx * CH);
        uint4 *zo = MODE == CONV_HIDDEN ? reinterpret_cast<uint4 *>(a.zbuf + pidx * CH) : nullptr;
#pragma unroll
        for (int q = 0; q < 4; q++) {
          float zr[8];
#pragma unroll
          for (int i = 0; i < 8; i++) zr[i] = __bfloat162float(__float2bfloat16_rn(acc[8 * q + i] + bias[8 * q + i]));
          if (MODE == CONV_HIDDEN) {
            uint4 u;
            u.x = pack2(zr[0], zr[1]); u.y = pack2(zr[2], zr[3]); u.z = pack2(zr[4], zr[5]); u.w = pack2(zr[6], zr[7]);
            zo[q] = u;
          }
          uint4 g;
          g.x = pack2(gelu(zr[0]), gelu(zr[1])); g.y = pack2(gelu(zr[2]), gelu(zr[3]));
          g.z = pack2(gelu(zr[4]), gelu(zr[5])); g.w = pack2(gelu(zr[6]), gelu(zr[7]));
          o[q] = g;
        }
      }
    }
    if (!ok) *abort_flag = 1;
  }
  if (!ok) atomicExch(a.status, 1);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 1) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, 32 * RS);
  }
}

// ------------------------------------------------------------- wgrad
__global__ void __launch_bounds__(192, 1)
    k_wgrad(const __grid_constant__ CUtensorMap x_map, const __grid_constant__ CUtensorMap g_map, WgradArgs a) {
  extern __shared__ uint8_t smem_raw[];
  const uint32_t raw = tc::smem_addr(smem_raw);
  const uint32_t base = (raw + 1023u) & ~1023u;
  uint8_t *sb = smem_raw + (base - raw);
  const uint32_t X0 = base;
  const uint32_t G0 = base + 4 * WG_PLANE;
  uint64_t *bars = reinterpret_cast<uint64_t *>(sb + 4 * WG_PLANE + 2 * G_TILE);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(bars + 16);
  volatile int *abort_flag = reinterpret_cast<volatile int *>(tmem_slot + 1);
  auto bar = [&](int i) { return tc::smem_addr(bars + i); };
  enum { FULL = 0, FREE = 4, GFULL = 8, GFREE = 10, DONE = 12 };

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int nyb = a.ny >> 2;
  const int yb = blockIdx.x % nyb, zb = blockIdx.x / nyb;
  const int xa = blockIdx.y * a.xchunk;
  const int n = min(a.xchunk, a.nx - xa);
  const size_t blk = (size_t)blockIdx.y * gridDim.x + blockIdx.x;

  if (threadIdx.x == 0) {
    for (int i = 0; i < 13; i++) tc::mbar_init(bar(i), 1);
    *abort_flag = 0;
    tc::mbar_fence_init();
  }
  if (warp == 1) {
    tc::tmem_alloc(tc::smem_addr(tmem_slot), 512);
    tc::tmem_relinquish();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tmem_slot;
  bool ok = true;

  if (warp == 0) {
    if (lane == 0) {
      tc::tma_prefetch_desc(&x_map);
      tc::tma_prefetch_desc(&g_map);
      int planes = 0, gtiles = 0;
      auto load_plane = [&](int p) -> bool {
        const int s = p & 3;
        if (p >= 4 && !one_wait(bar(FREE + s), ((p >> 2) - 1) & 1, a.spin, abort_flag)) return false;
        tc::mbar_expect_tx(bar(FULL + s), WG_PLANE);
        for (int dz = 0; dz < 3; dz++)
          tc::tma_load_4d(X0 + s * WG_PLANE + dz * WG_COPY, &x_map, bar(FULL + s), 0, zb * 32 + dz, yb * 4, xa + p);
        planes = p + 1;
        return true;
      };
      ok = load_plane(0) && load_plane(1);
      for (int t = 0; t < n && ok; t++) {
        if (!load_plane(t + 2)) { ok = false; break; }
        const int g = t & 1;
        if (t >= 2 && !one_wait(bar(GFREE + g), ((t >> 1) - 1) & 1, a.spin, abort_flag)) { ok = false; break; }
        tc::mbar_expect_tx(bar(GFULL + g), G_TILE);
        tc::tma_load_4d(G0 + g * G_TILE, &g_map, bar(GFULL + g), 0, zb * 32 + 1, yb * 4 + 1, xa + t + 1);
        gtiles = t + 1;
      }
      if (!ok) *abort_flag = 1;
      for (int p = max(0, planes - 4); p < planes; p++) tc::mbar_wait(bar(FULL + (p & 3)), (p >> 2) & 1, a.spin);
      for (int t = max(0, gtiles - 2); t < gtiles; t++) tc::mbar_wait(bar(GFULL + (t & 1)), (t >> 1) & 1, a.spin);
    }
  } else if (warp == 1) {
    if (lane == 0) {
      bool issued = false;
      const uint64_t xdesc = tc::desc_sw64(X0, 32 * ROW, 512), gdesc = tc::desc_sw64(G0, 512, 512);
      for (int t = 0; t < n && ok; t++) {
        for (int q = 0; q < 3 && ok; q++)
          if (!one_wait(bar(FULL + ((t + q) & 3)), ((t + q) >> 2) & 1, a.spin, abort_flag)) ok = false;
        if (ok && !one_wait(bar(GFULL + (t & 1)), (t >> 1) & 1, a.spin, abort_flag)) ok = false;
        if (!ok) break;
        tc::fence_after_sync();
        // 72 MMAs fully unrolled on base descriptors plus compile-time offsets
        // (as in k_conv)
        const uint64_t xp[3] = {xdesc + (uint64_t)(((t + 0) & 3) * (WG_PLANE >> 4)),
                                xdesc + (uint64_t)(((t + 1) & 3) * (WG_PLANE >> 4)),
                                xdesc + (uint64_t)(((t + 2) & 3) * (WG_PLANE >> 4))};
        const uint64_t g_d = gdesc + (uint64_t)((t & 1) * (G_TILE >> 4));
#pragma unroll
        for (int g = 0; g < 9; g++) {
          const int dx = g / 3, dz = g % 3;
          const uint64_t x_d = xp[dx] + (uint64_t)((dz * WG_COPY) >> 4);
#pragma unroll
          for (int kk = 0; kk < 8; kk++)
            tc::mma_f16(tmem + g * 32, x_d + (uint64_t)(kk * (1024 >> 4)), g_d + (uint64_t)(kk * (1024 >> 4)), IDESC_WG,
                        (t > 0 || kk > 0) ? 1u : 0u);
        }
        tc::mma_commit(bar(FREE + (t & 3)));
        tc::mma_commit(bar(GFREE + (t & 1)));
        issued = true;
      }
      if (!ok) *abort_flag = 1;
      if (issued) tc::mma_commit(bar(DONE));
      else tc::mbar_arrive(bar(DONE));
    }
  } else {
    const int ew = warp & 3;
    if (!warp_wait(bar(DONE), 0, a.spin, abort_flag)) ok = false;
    if (ok && !*abort_flag) {
      tc::fence_after_sync();
      for (int g = 0; g < 9; g++) {
        float v[32];
        tc::tmem_ld_32x32(tmem + ((uint32_t)(ew * 32) << 16) + g * 32, v);
        const int dy = ew;
        if (dy < 3) {
          const int tap = ((g / 3) * 3 + dy) * 3 + (g % 3);
          float *p = a.partial + (blk * 27 + tap) * 1024 + lane;
#pragma unroll
          for (int c = 0; c < 32; c++) p[c * 32] = v[c];
        }
      }
    }
  }
  if (!ok) atomicExch(a.status, 1);
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 1) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, 512);
  }
}

// ------------------------------------------------ CUDA-core helpers
// periodic x and z halos of a padded buffer (sources are interior cells)
__global__ void k_halo(bf16 *buf, int nx, int ny, int nz) {
  const int Yp = ny + 2, Zp = nz + 2;
  const long long nz_halo = (long long)nx * ny * 2;           // z halos of interior x planes
  const long long nx_halo = 2LL * ny * Zp;                      // whole x-halo rows (z halos included)
  const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  int x, y, z, sx, sz;
  if (id < nz_halo) {
    const int side = id & 1;
    const long long r = id >> 1;
    x = 1 + (int)(r / ny); y = 1 + (int)(r % ny);
    z = side ? nz + 1 : 0; sz = side ? 1 : nz; sx = x;
  } else if (id < nz_halo + nx_halo) {
    const long long r = id - nz_halo;
    const int side = (int)(r / ((long long)ny * Zp));
    const long long q = r % ((long long)ny * Zp);
    y = 1 + (int)(q / Zp); z = (int)(q % Zp);
    x = side ? nx + 1 : 0; sx = side ? 1 : nx;
    sz = z == 0 ? nz : (z == nz + 1 ? 1 : z);
  } else {
    return;
  }
  const uint4 *src = reinterpret_cast<const uint4 *>(buf + (((size_t)sx * Yp + y) * Zp + sz) * CH);
  uint4 *dst = reinterpret_cast<uint4 *>(buf + (((size_t)x * Yp + y) * Zp + z) * CH);
#pragma unroll
  for (int q = 0; q < 4; q++) dst[q] = src[q];
}

// Input scales: per variable the level's mean and 1/std, and 1/RMS of its
// first and second time differences; output scale of the correction.
struct Scales { float mean[5], inv_std[5], inv_d1[5], inv_d2[5], oscale[5], inv_oscale[5]; };

// network input from 15 host-normalised channels [15][cells] (tests)
__global__ void k_pack_normalised(const float *x0, bf16 *act, int nx, int ny, int nz) {
  const long long cells = (long long)nx * ny * nz;
  const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (id >= cells) return;
  const int z = (int)(id % nz), y = (int)((id / nz) % ny), x = (int)(id / ((long long)ny * nz));
  float f[32];
#pragma unroll
  for (int c = 0; c < 32; c++) f[c] = c < 15 ? x0[c * cells + id] : 0.f;
  uint4 *o = reinterpret_cast<uint4 *>(act + (((size_t)(x + 1) * (ny + 2) + y + 1) * (nz + 2) + z + 1) * CH);
#pragma unroll
  for (int q = 0; q < 4; q++) {
    uint4 u;
    u.x = pack2(f[8 * q], f[8 * q + 1]); u.y = pack2(f[8 * q + 2], f[8 * q + 3]);
    u.z = pack2(f[8 * q + 4], f[8 * q + 5]); u.w = pack2(f[8 * q + 6], f[8 * q + 7]);
    o[q] = u;
  }
}

// [5][cells] float -> [cells][8] float
__global__ void k_pack_target(const float *t, float *t8, long long cells) {
  const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (id >= cells) return;
  float4 *o = reinterpret_cast<float4 *>(t8 + id * 8);
  o[0] = make_float4(t[id], t[cells + id], t[2 * cells + id], t[3 * cells + id]);
  o[1] = make_float4(t[4 * cells + id], 0.f, 0.f, 0.f);
}

// network input and target from four stored levels (physical Q, [5][cells]):
// lv[0] = Q^(n-2), lv[1] = Q^(n-1), lv[2] = Q^n, lv[3] = Q^(n+1) (or null)
__global__ void k_pack_levels(const float *l0, const float *l1, const float *l2, const float *l3, bf16 *act,
                              float *t8, Scales s, int nx, int ny, int nz) {
  const long long cells = (long long)nx * ny * nz;
  const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (id >= cells) return;
  const int z = (int)(id % nz), y = (int)((id / nz) % ny), x = (int)(id / ((long long)ny * nz));
  float f[32];
  float ex[5];
#pragma unroll
  for (int v = 0; v < 5; v++) {
    const float qn = l2[v * cells + id], q1 = l1[v * cells + id], q2 = l0[v * cells + id];
    f[v] = (qn - s.mean[v]) * s.inv_std[v];
    f[5 + v] = (qn - q1) * s.inv_d1[v];
    f[10 + v] = ((qn - q1) - (q1 - q2)) * s.inv_d2[v];
    ex[v] = 3.f * qn - 3.f * q1 + q2;
  }
#pragma unroll
  for (int c = 15; c < 32; c++) f[c] = 0.f;
  uint4 *o = reinterpret_cast<uint4 *>(act + (((size_t)(x + 1) * (ny + 2) + y + 1) * (nz + 2) + z + 1) * CH);
#pragma unroll
  for (int q = 0; q < 4; q++) {
    uint4 u;
    u.x = pack2(f[8 * q], f[8 * q + 1]); u.y = pack2(f[8 * q + 2], f[8 * q + 3]);
    u.z = pack2(f[8 * q + 4], f[8 * q + 5]); u.w = pack2(f[8 * q + 6], f[8 * q + 7]);
    o[q] = u;
  }
  if (l3) {
    float tt[5];
#pragma unroll
    for (int v = 0; v < 5; v++) tt[v] = (l3[v * cells + id] - ex[v]) * s.inv_oscale[v];
    float4 *to = reinterpret_cast<float4 *>(t8 + id * 8);
    to[0] = make_float4(tt[0], tt[1], tt[2], tt[3]);
    to[1] = make_float4(tt[4], 0.f, 0.f, 0.f);
  }
}

// network input from the solver's time levels (Q/J in the reference layout)
__global__ void k_pack_state(Dev d, bf16 *act, Scales s) {
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  const long long cells = (long long)nx * ny * nz;
  const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (id >= cells) return;
  const int z = (int)(id % nz), y = (int)((id / nz) % ny), x = (int)(id / ((long long)ny * nz));
  const long long o = ix(d, x + 3, y + 2, z + 2);
  const double J = d.J[o];
  float f[32];
#pragma unroll
  for (int v = 0; v < 5; v++) {
    const float qn = (float)(d.U[v][o] * J), q1 = (float)(d.Uq[v][o] * J), q2 = (float)(d.Uqq[v][o] * J);
    f[v] = (qn - s.mean[v]) * s.inv_std[v];
    f[5 + v] = (qn - q1) * s.inv_d1[v];
    f[10 + v] = ((qn - q1) - (q1 - q2)) * s.inv_d2[v];
  }
#pragma unroll
  for (int c = 15; c < 32; c++) f[c] = 0.f;
  uint4 *op = reinterpret_cast<uint4 *>(act + (((size_t)(x + 1) * (ny + 2) + y + 1) * (nz + 2) + z + 1) * CH);
#pragma unroll
  for (int q = 0; q < 4; q++) {
    uint4 u;
    u.x = pack2(f[8 * q], f[8 * q + 1]); u.y = pack2(f[8 * q + 2], f[8 * q + 3]);
    u.z = pack2(f[8 * q + 4], f[8 * q + 5]); u.w = pack2(f[8 * q + 6], f[8 * q + 7]);
    op[q] = u;
  }
}

// U_ = 3 U - 3 Uq + Uqq + correction * oscale / J on the interior; a
// non-finite correction falls back to the extrapolation of that cell
__global__ void k_apply(Dev d, const float *out8, Scales s) {
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  const long long cells = (long long)nx * ny * nz;
  const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (id >= cells) return;
  const int z = (int)(id % nz), y = (int)((id / nz) % ny), x = (int)(id / ((long long)ny * nz));
  const long long o = ix(d, x + 3, y + 2, z + 2);
  const double J = d.J[o];
#pragma unroll
  for (int v = 0; v < 5; v++) {
    const double ext = 3.0 * d.U[v][o] - 3.0 * d.Uq[v][o] + d.Uqq[v][o];
    const float c = out8[id * 8 + v];
    d.U_[v][o] = isfinite(c) ? ext + (double)c * (double)s.oscale[v] / J : ext;
  }
}

// level store: physical Q of the context's current level U (Q/J)
__global__ void k_store_level(Dev d, float *lv) {
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  const long long cells = (long long)nx * ny * nz;
  const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (id >= cells) return;
  const int z = (int)(id % nz), y = (int)((id / nz) % ny), x = (int)(id / ((long long)ny * nz));
  const long long o = ix(d, x + 3, y + 2, z + 2);
  const double J = d.J[o];
#pragma unroll
  for (int v = 0; v < 5; v++) lv[v * cells + id] = (float)(d.U[v][o] * J);
}

// mean squared error, its gradient (BF16, padded) and per-block loss sums
__global__ void k_loss(const float *out8, const float *t8, bf16 *g, double *blk_loss, int nx, int ny, int nz) {
  const long long cells = (long long)nx * ny * nz;
  const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  double l = 0.0;
  if (id < cells) {
    const int z = (int)(id % nz), y = (int)((id / nz) % ny), x = (int)(id / ((long long)ny * nz));
    const float inv = 2.0f / (5.0f * (float)cells);
    float gg[8];
#pragma unroll
    for (int v = 0; v < 8; v++) {
      const float df = v < 5 ? out8[id * 8 + v] - t8[id * 8 + v] : 0.f;
      l += (double)df * df;
      gg[v] = df * inv;
    }
    uint4 *o = reinterpret_cast<uint4 *>(g + (((size_t)(x + 1) * (ny + 2) + y + 1) * (nz + 2) + z + 1) * CH);
    uint4 u;
    u.x = pack2(gg[0], gg[1]); u.y = pack2(gg[2], gg[3]); u.z = pack2(gg[4], gg[5]); u.w = pack2(gg[6], gg[7]);
    o[0] = u;
    o[1] = make_uint4(0, 0, 0, 0); o[2] = make_uint4(0, 0, 0, 0); o[3] = make_uint4(0, 0, 0, 0);
  }
  __shared__ double red[256];
  red[threadIdx.x] = l;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0) blk_loss[blockIdx.x] = red[0];
}

__global__ void k_sum_loss(const double *blk, int n, long long cells, float *loss_out) {
  __shared__ double red[256];
  double s = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s += blk[i];
  red[threadIdx.x] = s;
  __syncthreads();
  for (int k = blockDim.x / 2; k > 0; k >>= 1) {
    if ((int)threadIdx.x < k) red[threadIdx.x] += red[threadIdx.x + k];
    __syncthreads();
  }
  if (threadIdx.x == 0) *loss_out = (float)(red[0] / (5.0 * (double)cells));
}

// dW = sum of the per-CTA partials (fixed order)
__global__ void k_reduce_wgrad(const float *partial, int nblk, float *dW) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 27 * 1024) return;
  float s = 0.f;
  for (int b = 0; b < nblk; b++) s += partial[(size_t)b * 27 * 1024 + e];
  dW[e] = s;
}

// per-block channel sums of a padded gradient (bias gradient), then total
__global__ void k_bias_partial(const bf16 *g, float *part, int nx, int ny, int nz) {
  const long long cells = (long long)nx * ny * nz;
  float s[32];
#pragma unroll
  for (int c = 0; c < 32; c++) s[c] = 0.f;
  for (long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x; id < cells; id += (long long)gridDim.x * blockDim.x) {
    const int z = (int)(id % nz), y = (int)((id / nz) % ny), x = (int)(id / ((long long)ny * nz));
    const uint4 *p = reinterpret_cast<const uint4 *>(g + (((size_t)(x + 1) * (ny + 2) + y + 1) * (nz + 2) + z + 1) * CH);
#pragma unroll
    for (int q = 0; q < 4; q++) {
      float f[8];
      unpack8(p[q], f);
#pragma unroll
      for (int i = 0; i < 8; i++) s[8 * q + i] += f[i];
    }
  }
  __shared__ float red[256][33];
#pragma unroll
  for (int c = 0; c < 32; c++) red[threadIdx.x][c] = s[c];
  __syncthreads();
  if (threadIdx.x < 32) {
    float t = 0.f;
    for (int i = 0; i < (int)blockDim.x; i++) t += red[i][threadIdx.x];
    part[blockIdx.x * 32 + threadIdx.x] = t;
  }
}
__global__ void k_bias_total(const float *part, int nblk, float *db) {
  const int c = threadIdx.x;
  if (c >= 32) return;
  float t = 0.f;
  for (int b = 0; b < nblk; b++) t += part[b * 32 + c];
  db[c] = t;
}

// BF16 copies of the float32 master weights: forward [27][cout][cin] and
// input-gradient [27][cin][cout] with the taps reversed
// BF16 weights of the forward (wf) and input-gradient (wt: transposed,
// tap-reversed) convolutions, tap t = 9 dx + 3 dy + dz stored as block
// 3 (3 dy + dz) + dx: the three dx taps of one (dy, dz) are 96 consecutive
// rows (output channel, 32 input channels), the N = 96 B operand of k_conv
__device__ __forceinline__ int wblock(int t) { return ((t / 3) % 3 * 3 + t % 3) * 3 + t / 9; }
__global__ void k_prep_weights(const float *W, bf16 *wf, bf16 *wt) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= 27 * 1024) return;
  const int t = e / 1024, co = (e / 32) % 32, ci = e % 32;
  const bf16 h = __float2bfloat16_rn(W[e]);
  wf[wblock(t) * 1024 + co * 32 + ci] = h;
  wt[wblock(26 - t) * 1024 + ci * 32 + co] = h;
}

// Adam (Kingma & Ba 2015), bias-corrected, float32
__global__ void k_adam(float *p, const float *g, float *m, float *v, int n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= n) return;
  const float gg = g[e];
  const float mm = b1 * m[e] + (1.f - b1) * gg;
  const float vv = b2 * v[e] + (1.f - b2) * gg * gg;
  m[e] = mm;
  v[e] = vv;
  p[e] -= lr * (mm / c1) / (sqrtf(vv / c2) + eps);
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// 4-D map over a padded activation buffer, box 32 channels x 32 z x box_y y x 1 x
bool act_map(CUtensorMap *m, void *base, int nx, int ny, int nz, int box_y) {
  auto enc = encode_fn();
  if (!enc) return false;
  const cuuint64_t dims[4] = {(cuuint64_t)CH, (cuuint64_t)(nz + 2), (cuuint64_t)(ny + 2), (cuuint64_t)(nx + 2)};
  const cuuint64_t strides[3] = {(cuuint64_t)ROW, (cuuint64_t)ROW * (nz + 2), (cuuint64_t)ROW * (nz + 2) * (ny + 2)};
  const cuuint32_t box[4] = {CH, 32, (cuuint32_t)box_y, 1};
  const cuuint32_t es[4] = {1, 1, 1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// 2-D map over [27*32 rows][32] BF16 weights, box 32 x 216 rows
bool weight_map(CUtensorMap *m, void *base) {
  auto enc = encode_fn();
  if (!enc) return false;
  const cuuint64_t dims[2] = {(cuuint64_t)CH, 27 * 32};
  const cuuint64_t strides[1] = {(cuuint64_t)ROW};
  const cuuint32_t box[2] = {CH, 216};
  const cuuint32_t es[2] = {1, 1};
  return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
             CU_TENSOR_MAP_SWIZZLE_64B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace
}  // namespace cgli

// ===================================================================== ABI
using namespace cgli;

struct cgli_cnn {
  int nx, ny, nz, device;
  long long cells, padded;
  cudaStream_t stream = nullptr;
  std::vector<void *> allocs;
  // parameters (padded to 32 x 32 per tap), float32 masters + BF16 copies
  float *W[NL], *b[NL], *dW[NL], *db[NL], *mW[NL], *vW[NL], *mb[NL], *vb[NL];
  bf16 *wf[NL], *wt[NL];
  CUtensorMap wf_map[NL], wt_map[NL];
  // activations: act[l] = input of layer l; z[l] = pre-activation of layer l
  bf16 *act[NL] = {}, *z[NL - 1] = {}, *g[2] = {};
  CUtensorMap act6[NL], act7[NL], g6[2], g4[2];
  float *out8 = nullptr, *t8 = nullptr, *partial = nullptr, *bpart = nullptr, *loss = nullptr;
  double *blk_loss = nullptr;
  int *status = nullptr;
  int xchunk = 0, nblk_cols = 0, nblk_x = 0, nbias = 0;
  bool training = false;
  Scales sc{};
  int adam_step = 0;
  // stored time levels (ring) for training
  std::vector<float *> levels;
  long long nlevels = 0;   // levels pushed so far
  float *h_loss = nullptr;
};

namespace {

thread_local std::string g_cnn_err;

int cfail(int code, const std::string &m) {
  g_cnn_err = m;
  set_last_error(m);
  return code;
}

#define CC(call)                                                                                  \
  do {                                                                                            \
    cudaError_t e_ = (call);                                                                      \
    if (e_ != cudaSuccess) return cfail(CGLI_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
  } while (0)

int calloc_dev(cgli_cnn *n, size_t bytes, void **out) {
  void *p = nullptr;
  cudaError_t e = cudaMalloc(&p, bytes);
  if (e != cudaSuccess) return cfail(CGLI_ENOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
  e = cudaMemset(p, 0, bytes);
  if (e != cudaSuccess) return cfail(CGLI_ECUDA, std::string("cudaMemset: ") + cudaGetErrorString(e));
  n->allocs.push_back(p);
  *out = p;
  return CGLI_OK;
}

int act_alloc(cgli_cnn *n, bf16 **p) { return calloc_dev(n, (size_t)n->padded * ROW, (void **)p); }

int ensure_training(cgli_cnn *n) {
  if (n->training) return CGLI_OK;
  int rc = CGLI_OK;
  for (int l = 0; l < NL - 1 && !rc; l++) rc = act_alloc(n, &n->z[l]);
  for (int i = 0; i < 2 && !rc; i++) rc = act_alloc(n, &n->g[i]);
  if (!rc) rc = calloc_dev(n, (size_t)n->nblk_cols * n->nblk_x * 27 * 1024 * sizeof(float), (void **)&n->partial);
  if (!rc) rc = calloc_dev(n, (size_t)n->cells * 8 * sizeof(float), (void **)&n->t8);
  if (rc) return rc;
  for (int i = 0; i < 2; i++)
    if (!act_map(&n->g6[i], n->g[i], n->nx, n->ny, n->nz, 6) || !act_map(&n->g4[i], n->g[i], n->nx, n->ny, n->nz, 4))
      return cfail(CGLI_ECUDA, "cuTensorMapEncodeTiled failed (gradient buffers)");
  n->training = true;
  return CGLI_OK;
}

int check_status(cgli_cnn *n, cudaStream_t s) {
  int st = 0;
  CC(cudaMemcpyAsync(&st, n->status, sizeof(int), cudaMemcpyDeviceToHost, s));
  CC(cudaStreamSynchronize(s));
  if (st) {
    cudaMemsetAsync(n->status, 0, sizeof(int), s);
    return cfail(CGLI_ETIMEOUT, "tensor-core kernel gave up waiting on a pipeline barrier");
  }
  return CGLI_OK;
}

dim3 conv_grid(const cgli_cnn *n) { return dim3(n->nblk_cols, n->nblk_x); }

void launch_halo(cgli_cnn *n, bf16 *buf, cudaStream_t s) {
  const long long work = (long long)n->nx * n->ny * 2 + 2LL * n->ny * (n->nz + 2);
  k_halo<<<(unsigned)((work + 255) / 256), 256, 0, s>>>(buf, n->nx, n->ny, n->nz);
}

ConvArgs conv_args(cgli_cnn *n) {
  ConvArgs a{};
  a.nx = n->nx; a.ny = n->ny; a.nz = n->nz; a.Yp = n->ny + 2; a.Zp = n->nz + 2;
  a.xchunk = n->xchunk; a.spin = SPIN; a.status = n->status;
  return a;
}

// forward through the five layers from act[0]; training keeps the
// pre-activations; the output goes to out8
void forward(cgli_cnn *n, bool train, cudaStream_t s) {
  for (int l = 0; l < NL; l++) {
    ConvArgs a = conv_args(n);
    a.bias = n->b[l];
    if (l < NL - 1) {
      a.act_out = n->act[l + 1];
      a.zbuf = train ? n->z[l] : nullptr;
      if (train) k_conv<CONV_HIDDEN><<<conv_grid(n), 192, CONV_SMEM, s>>>(n->act6[l], n->wf_map[l], a);
      else k_conv<CONV_HIDDEN_INFER><<<conv_grid(n), 192, CONV_SMEM, s>>>(n->act6[l], n->wf_map[l], a);
      launch_halo(n, n->act[l + 1], s);
    } else {
      a.out32 = n->out8;
      k_conv<CONV_OUT><<<conv_grid(n), 192, CONV_SMEM, s>>>(n->act6[l], n->wf_map[l], a);
    }
  }
}

void prep_weights(cgli_cnn *n, cudaStream_t s) {
  for (int l = 0; l < NL; l++) k_prep_weights<<<(27 * 1024 + 255) / 256, 256, 0, s>>>(n->W[l], n->wf[l], n->wt[l]);
}

// loss on out8 vs t8, gradients of every layer into dW/db
void backward(cgli_cnn *n, cudaStream_t s) {
  const long long cells = n->cells;
  const int lb = (int)((cells + 255) / 256);
  k_loss<<<lb, 256, 0, s>>>(n->out8, n->t8, n->g[0], n->blk_loss, n->nx, n->ny, n->nz);
  k_sum_loss<<<1, 256, 0, s>>>(n->blk_loss, lb, cells, n->loss);
  launch_halo(n, n->g[0], s);
  int cur = 0;
  const int nblk = n->nblk_cols * n->nblk_x;
  for (int l = NL - 1; l >= 0; l--) {
    WgradArgs w{};
    w.partial = n->partial; w.nx = n->nx; w.ny = n->ny; w.nz = n->nz; w.xchunk = n->xchunk; w.spin = SPIN;
    w.status = n->status;
    k_wgrad<<<conv_grid(n), 192, WGRAD_SMEM, s>>>(n->act7[l], n->g4[cur], w);
    k_reduce_wgrad<<<(27 * 1024 + 255) / 256, 256, 0, s>>>(n->partial, nblk, n->dW[l]);
    k_bias_partial<<<n->nbias, 256, 0, s>>>(n->g[cur], n->bpart, n->nx, n->ny, n->nz);
    k_bias_total<<<1, 32, 0, s>>>(n->bpart, n->nbias, n->db[l]);
    if (l > 0) {
      ConvArgs a = conv_args(n);
      a.act_out = n->g[cur ^ 1];
      a.zbuf = n->z[l - 1];
      k_conv<CONV_DGRAD><<<conv_grid(n), 192, CONV_SMEM, s>>>(n->g6[cur], n->wt_map[l], a);
      launch_halo(n, n->g[cur ^ 1], s);
      cur ^= 1;
    }
  }
}

void adam_step(cgli_cnn *n, float lr, cudaStream_t s) {
  n->adam_step++;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  const float c1 = 1.f - powf(b1, (float)n->adam_step), c2 = 1.f - powf(b2, (float)n->adam_step);
  for (int l = 0; l < NL; l++) {
    k_adam<<<(27 * 1024 + 255) / 256, 256, 0, s>>>(n->W[l], n->dW[l], n->mW[l], n->vW[l], 27 * 1024, lr, b1, b2, eps, c1, c2);
    k_adam<<<1, 32, 0, s>>>(n->b[l], n->db[l], n->mb[l], n->vb[l], 32, lr, b1, b2, eps, c1, c2);
  }
  prep_weights(n, s);
}

int set_smem_attrs() {
  static bool done = false;
  if (done) return CGLI_OK;
  CC(cudaFuncSetAttribute(k_conv<CONV_HIDDEN>, cudaFuncAttributeMaxDynamicSharedMemorySize, CONV_SMEM));
  CC(cudaFuncSetAttribute(k_conv<CONV_HIDDEN_INFER>, cudaFuncAttributeMaxDynamicSharedMemorySize, CONV_SMEM));
  CC(cudaFuncSetAttribute(k_conv<CONV_OUT>, cudaFuncAttributeMaxDynamicSharedMemorySize, CONV_SMEM));
  CC(cudaFuncSetAttribute(k_conv<CONV_DGRAD>, cudaFuncAttributeMaxDynamicSharedMemorySize, CONV_SMEM));
  CC(cudaFuncSetAttribute(k_wgrad, cudaFuncAttributeMaxDynamicSharedMemorySize, WGRAD_SMEM));
  done = true;
  return CGLI_OK;
}

// host flat parameters (real shapes) <-> padded device layout
void unpack_params(const float *theta, std::vector<float> *Wp, std::vector<float> *bp) {
  size_t o = 0;
  for (int l = 0; l < NL; l++) {
    Wp[l].assign(27 * 1024, 0.f);
    bp[l].assign(32, 0.f);
    for (int t = 0; t < 27; t++)
      for (int co = 0; co < COUT[l]; co++)
        for (int ci = 0; ci < CIN[l]; ci++) Wp[l][t * 1024 + co * 32 + ci] = theta[o++];
    for (int co = 0; co < COUT[l]; co++) bp[l][co] = theta[o++];
  }
}
void pack_params(const std::vector<float> *Wp, const std::vector<float> *bp, float *theta) {
  size_t o = 0;
  for (int l = 0; l < NL; l++) {
    for (int t = 0; t < 27; t++)
      for (int co = 0; co < COUT[l]; co++)
        for (int ci = 0; ci < CIN[l]; ci++) theta[o++] = Wp[l][t * 1024 + co * 32 + ci];
    for (int co = 0; co < COUT[l]; co++) theta[o++] = bp[l][co];
  }
}

long long nparams() {
  long long s = 0;
  for (int l = 0; l < NL; l++) s += 27LL * CIN[l] * COUT[l] + COUT[l];
  return s;
}

}  // namespace

namespace cgli {

bool cnn_matches(const cgli_cnn *n, int nx, int ny, int nz) { return n && n->nx == nx && n->ny == ny && n->nz == nz; }

cudaError_t cnn_predict(cgli_cnn *n, const Dev &d, cudaStream_t s) {
  const unsigned nb = (unsigned)((n->cells + 255) / 256);
  k_pack_state<<<nb, 256, 0, s>>>(d, n->act[0], n->sc);
  launch_halo(n, n->act[0], s);
  forward(n, false, s);
  k_apply<<<nb, 256, 0, s>>>(d, n->out8, n->sc);
  return cudaGetLastError();
}

}  // namespace cgli

extern "C" {

long long cgli_cnn_param_count(void) { return nparams(); }

int cgli_cnn_create(int nx, int ny, int nz, cgli_cnn **out) {
  if (!out) return cfail(CGLI_EINVAL, "null argument");
  *out = nullptr;
  if (nx < 2 || ny < 4 || nz < 32 || ny % 4 || nz % 32)
    return cfail(CGLI_EINVAL, "network grid needs Nx >= 2, Ny a multiple of 4, Nz a multiple of 32");
  int rc = set_smem_attrs();
  if (rc) return rc;
  if (!encode_fn()) return cfail(CGLI_ECUDA, "cuTensorMapEncodeTiled entry point unavailable");
  cgli_cnn *n = new cgli_cnn();
  n->nx = nx; n->ny = ny; n->nz = nz;
  cudaGetDevice(&n->device);
  n->cells = (long long)nx * ny * nz;
  n->padded = (long long)(nx + 2) * (ny + 2) * (nz + 2);
  n->xchunk = nx <= 32 ? nx : 32;
  n->nblk_cols = (ny / 4) * (nz / 32);
  n->nblk_x = (nx + n->xchunk - 1) / n->xchunk;
  n->nbias = 296;
  if (cudaStreamCreateWithFlags(&n->stream, cudaStreamNonBlocking) != cudaSuccess) {
    delete n;
    return cfail(CGLI_ECUDA, "cudaStreamCreate failed");
  }
  for (int l = 0; l < NL && !rc; l++) {
    rc = calloc_dev(n, 27 * 1024 * 4, (void **)&n->W[l]);
    if (!rc) rc = calloc_dev(n, 27 * 1024 * 4, (void **)&n->dW[l]);
    if (!rc) rc = calloc_dev(n, 27 * 1024 * 4, (void **)&n->mW[l]);
    if (!rc) rc = calloc_dev(n, 27 * 1024 * 4, (void **)&n->vW[l]);
    if (!rc) rc = calloc_dev(n, 32 * 4, (void **)&n->b[l]);
    if (!rc) rc = calloc_dev(n, 32 * 4, (void **)&n->db[l]);
    if (!rc) rc = calloc_dev(n, 32 * 4, (void **)&n->mb[l]);
    if (!rc) rc = calloc_dev(n, 32 * 4, (void **)&n->vb[l]);
    if (!rc) rc = calloc_dev(n, 27 * 1024 * 2, (void **)&n->wf[l]);
    if (!rc) rc = calloc_dev(n, 27 * 1024 * 2, (void **)&n->wt[l]);
    if (!rc) rc = act_alloc(n, &n->act[l]);
  }
  if (!rc) rc = calloc_dev(n, (size_t)n->cells * 8 * sizeof(float), (void **)&n->out8);
  if (!rc) rc = calloc_dev(n, (size_t)n->nbias * 32 * sizeof(float), (void **)&n->bpart);
  if (!rc) rc = calloc_dev(n, sizeof(float) * 4, (void **)&n->loss);
  if (!rc) rc = calloc_dev(n, sizeof(double) * ((n->cells + 255) / 256 + 1), (void **)&n->blk_loss);
  if (!rc) rc = calloc_dev(n, sizeof(int) * 4, (void **)&n->status);
  if (!rc && cudaMallocHost(&n->h_loss, sizeof(float) * 4) != cudaSuccess) rc = cfail(CGLI_ENOMEM, "cudaMallocHost failed");
  for (int l = 0; l < NL && !rc; l++) {
    if (!weight_map(&n->wf_map[l], n->wf[l]) || !weight_map(&n->wt_map[l], n->wt[l]) ||
        !act_map(&n->act6[l], n->act[l], nx, ny, nz, 6) || !act_map(&n->act7[l], n->act[l], nx, ny, nz, 7))
      rc = cfail(CGLI_ECUDA, "cuTensorMapEncodeTiled failed");
  }
  for (int v = 0; v < 5; v++) {
    n->sc.mean[v] = 0.f; n->sc.inv_std[v] = 1.f; n->sc.inv_d1[v] = 1.f; n->sc.inv_d2[v] = 1.f;
    n->sc.oscale[v] = 1.f; n->sc.inv_oscale[v] = 1.f;
  }
  if (rc) {
    for (void *p : n->allocs) cudaFree(p);
    if (n->h_loss) cudaFreeHost(n->h_loss);
    cudaStreamDestroy(n->stream);
    delete n;
    return rc;
  }
  *out = n;
  return CGLI_OK;
}

int cgli_cnn_destroy(cgli_cnn *n) {
  if (!n) return CGLI_OK;
  cudaStreamSynchronize(n->stream);
  for (void *p : n->allocs) cudaFree(p);
  for (float *p : n->levels) cudaFree(p);
  if (n->h_loss) cudaFreeHost(n->h_loss);
  cudaStreamDestroy(n->stream);
  delete n;
  return CGLI_OK;
}

int cgli_cnn_set_params(cgli_cnn *n, const float *theta) {
  if (!n || !theta) return cfail(CGLI_EINVAL, "null argument");
  std::vector<float> Wp[NL], bp[NL];
  unpack_params(theta, Wp, bp);
  for (int l = 0; l < NL; l++) {
    CC(cudaMemcpyAsync(n->W[l], Wp[l].data(), 27 * 1024 * 4, cudaMemcpyHostToDevice, n->stream));
    CC(cudaMemcpyAsync(n->b[l], bp[l].data(), 32 * 4, cudaMemcpyHostToDevice, n->stream));
    CC(cudaMemsetAsync(n->mW[l], 0, 27 * 1024 * 4, n->stream));
    CC(cudaMemsetAsync(n->vW[l], 0, 27 * 1024 * 4, n->stream));
    CC(cudaMemsetAsync(n->mb[l], 0, 32 * 4, n->stream));
    CC(cudaMemsetAsync(n->vb[l], 0, 32 * 4, n->stream));
  }
  n->adam_step = 0;
  prep_weights(n, n->stream);
  CC(cudaGetLastError());
  CC(cudaStreamSynchronize(n->stream));
  return CGLI_OK;
}

static int copy_out_params(cgli_cnn *n, float *const *src_w, float *const *src_b, float *theta) {
  std::vector<float> Wp[NL], bp[NL];
  for (int l = 0; l < NL; l++) {
    Wp[l].resize(27 * 1024);
    bp[l].resize(32);
    CC(cudaMemcpyAsync(Wp[l].data(), src_w[l], 27 * 1024 * 4, cudaMemcpyDeviceToHost, n->stream));
    CC(cudaMemcpyAsync(bp[l].data(), src_b[l], 32 * 4, cudaMemcpyDeviceToHost, n->stream));
  }
  CC(cudaStreamSynchronize(n->stream));
  pack_params(Wp, bp, theta);
  return CGLI_OK;
}

int cgli_cnn_get_params(cgli_cnn *n, float *theta) {
  if (!n || !theta) return cfail(CGLI_EINVAL, "null argument");
  return copy_out_params(n, n->W, n->b, theta);
}

int cgli_cnn_set_scales(cgli_cnn *n, const double mean[5], const double stdv[5], const double d1[5],
                        const double d2[5], const double oscale[5]) {
  if (!n || !mean || !stdv || !d1 || !d2 || !oscale) return cfail(CGLI_EINVAL, "null argument");
  for (int v = 0; v < 5; v++)
    if (!(stdv[v] > 0) || !(d1[v] > 0) || !(d2[v] > 0) || !(oscale[v] > 0))
      return cfail(CGLI_EINVAL, "scales must be positive");
  for (int v = 0; v < 5; v++) {
    n->sc.mean[v] = (float)mean[v];
    n->sc.inv_std[v] = (float)(1.0 / stdv[v]);
    n->sc.inv_d1[v] = (float)(1.0 / d1[v]);
    n->sc.inv_d2[v] = (float)(1.0 / d2[v]);
    n->sc.oscale[v] = (float)oscale[v];
    n->sc.inv_oscale[v] = (float)(1.0 / oscale[v]);
  }
  return CGLI_OK;
}

int cgli_cnn_forward_host(cgli_cnn *n, const float *x0, float *out) {
  if (!n || !x0 || !out) return cfail(CGLI_EINVAL, "null argument");
  cudaStream_t s = n->stream;
  const size_t in_bytes = (size_t)n->cells * 15 * 4;
  float *dx = nullptr;
  CC(cudaMallocAsync((void **)&dx, in_bytes, s));
  CC(cudaMemcpyAsync(dx, x0, in_bytes, cudaMemcpyHostToDevice, s));
  const unsigned nb = (unsigned)((n->cells + 255) / 256);
  k_pack_normalised<<<nb, 256, 0, s>>>(dx, n->act[0], n->nx, n->ny, n->nz);
  launch_halo(n, n->act[0], s);
  forward(n, false, s);
  CC(cudaGetLastError());
  std::vector<float> o8((size_t)n->cells * 8);
  CC(cudaMemcpyAsync(o8.data(), n->out8, o8.size() * 4, cudaMemcpyDeviceToHost, s));
  CC(cudaFreeAsync(dx, s));
  int rc = check_status(n, s);
  if (rc) return rc;
  for (long long c = 0; c < n->cells; c++)
    for (int v = 0; v < 5; v++) out[v * n->cells + c] = o8[c * 8 + v];
  return CGLI_OK;
}

int cgli_cnn_loss_grad_host(cgli_cnn *n, const float *x0, const float *target, float *loss, float *grad) {
  if (!n || !x0 || !target || !loss || !grad) return cfail(CGLI_EINVAL, "null argument");
  int rc = ensure_training(n);
  if (rc) return rc;
  cudaStream_t s = n->stream;
  const size_t in_bytes = (size_t)n->cells * 15 * 4, t_bytes = (size_t)n->cells * 5 * 4;
  float *dx = nullptr, *dt = nullptr;
  CC(cudaMallocAsync((void **)&dx, in_bytes, s));
  CC(cudaMallocAsync((void **)&dt, t_bytes, s));
  CC(cudaMemcpyAsync(dx, x0, in_bytes, cudaMemcpyHostToDevice, s));
  CC(cudaMemcpyAsync(dt, target, t_bytes, cudaMemcpyHostToDevice, s));
  const unsigned nb = (unsigned)((n->cells + 255) / 256);
  k_pack_normalised<<<nb, 256, 0, s>>>(dx, n->act[0], n->nx, n->ny, n->nz);
  k_pack_target<<<nb, 256, 0, s>>>(dt, n->t8, n->cells);
  launch_halo(n, n->act[0], s);
  forward(n, true, s);
  backward(n, s);
  CC(cudaGetLastError());
  CC(cudaMemcpyAsync(n->h_loss, n->loss, 4, cudaMemcpyDeviceToHost, s));
  CC(cudaFreeAsync(dx, s));
  CC(cudaFreeAsync(dt, s));
  rc = check_status(n, s);
  if (rc) return rc;
  *loss = n->h_loss[0];
  return copy_out_params(n, n->dW, n->db, grad);
}

int cgli_cnn_reserve_levels(cgli_cnn *n, int count) {
  if (!n || count < 4) return cfail(CGLI_EINVAL, "need at least 4 stored levels");
  for (float *p : n->levels) cudaFree(p);
  n->levels.clear();
  n->nlevels = 0;
  for (int i = 0; i < count; i++) {
    float *p = nullptr;
    cudaError_t e = cudaMalloc(&p, (size_t)n->cells * 5 * 4);
    if (e != cudaSuccess) return cfail(CGLI_ENOMEM, std::string("cudaMalloc (levels): ") + cudaGetErrorString(e));
    n->levels.push_back(p);
  }
  return CGLI_OK;
}

long long cgli_cnn_levels(const cgli_cnn *n) { return n ? n->nlevels : 0; }

int cgli_cnn_push_level_host(cgli_cnn *n, const float *q) {
  if (!n || !q) return cfail(CGLI_EINVAL, "null argument");
  if (n->levels.empty()) return cfail(CGLI_ESTATE, "no level storage (cgli_cnn_reserve_levels)");
  float *dst = n->levels[n->nlevels % (long long)n->levels.size()];
  CC(cudaMemcpyAsync(dst, q, (size_t)n->cells * 5 * 4, cudaMemcpyHostToDevice, n->stream));
  CC(cudaStreamSynchronize(n->stream));
  n->nlevels++;
  return CGLI_OK;
}

// levels i .. i+3 of the ring, or null if any is no longer (or not yet) stored
static bool pair_levels(cgli_cnn *n, long long i, float *lv[4]) {
  const long long cap = (long long)n->levels.size();
  if (i < 0 || i + 3 >= n->nlevels || i < n->nlevels - cap) return false;
  for (int k = 0; k < 4; k++) lv[k] = n->levels[(i + k) % cap];
  return true;
}

int cgli_cnn_pair_loss(cgli_cnn *n, long long pair, float *loss) {
  if (!n || !loss) return cfail(CGLI_EINVAL, "null argument");
  int rc = ensure_training(n);
  if (rc) return rc;
  float *lv[4];
  if (!pair_levels(n, pair, lv)) return cfail(CGLI_EINVAL, "pair not in the stored levels");
  cudaStream_t s = n->stream;
  const unsigned nb = (unsigned)((n->cells + 255) / 256);
  k_pack_levels<<<nb, 256, 0, s>>>(lv[0], lv[1], lv[2], lv[3], n->act[0], n->t8, n->sc, n->nx, n->ny, n->nz);
  launch_halo(n, n->act[0], s);
  forward(n, false, s);
  const int lb = (int)((n->cells + 255) / 256);
  k_loss<<<lb, 256, 0, s>>>(n->out8, n->t8, n->g[0], n->blk_loss, n->nx, n->ny, n->nz);
  k_sum_loss<<<1, 256, 0, s>>>(n->blk_loss, lb, n->cells, n->loss);
  CC(cudaGetLastError());
  CC(cudaMemcpyAsync(n->h_loss, n->loss, 4, cudaMemcpyDeviceToHost, s));
  rc = check_status(n, s);
  if (rc) return rc;
  *loss = n->h_loss[0];
  return CGLI_OK;
}

int cgli_cnn_train(cgli_cnn *n, int steps, float lr, unsigned long long seed, long long first_pair, long long npairs,
                   float *mean_loss) {
  if (!n || steps <= 0 || !(lr > 0) || npairs <= 0) return cfail(CGLI_EINVAL, "bad training arguments");
  int rc = ensure_training(n);
  if (rc) return rc;
  float *lv[4];
  for (long long i = first_pair; i < first_pair + npairs; i++)
    if (!pair_levels(n, i, lv)) return cfail(CGLI_EINVAL, "pair range not in the stored levels");
  cudaStream_t s = n->stream;
  const unsigned nb = (unsigned)((n->cells + 255) / 256);
  unsigned long long st = seed ? seed : 0x9E3779B97F4A7C15ull;
  double sum = 0.0;
  for (int k = 0; k < steps; k++) {
    // splitmix64 pick of the pair
    st += 0x9E3779B97F4A7C15ull;
    unsigned long long r = st;
    r = (r ^ (r >> 30)) * 0xBF58476D1CE4E5B9ull;
    r = (r ^ (r >> 27)) * 0x94D049BB133111EBull;
    r ^= r >> 31;
    const long long pair = first_pair + (long long)(r % (unsigned long long)npairs);
    pair_levels(n, pair, lv);
    k_pack_levels<<<nb, 256, 0, s>>>(lv[0], lv[1], lv[2], lv[3], n->act[0], n->t8, n->sc, n->nx, n->ny, n->nz);
    launch_halo(n, n->act[0], s);
    forward(n, true, s);
    backward(n, s);
    adam_step(n, lr, s);
    CC(cudaGetLastError());
    CC(cudaMemcpyAsync(n->h_loss, n->loss, 4, cudaMemcpyDeviceToHost, s));
    CC(cudaStreamSynchronize(s));
    sum += n->h_loss[0];
  }
  rc = check_status(n, s);
  if (rc) return rc;
  if (mean_loss) *mean_loss = (float)(sum / steps);
  return CGLI_OK;
}

const char *cgli_cnn_last_error(void) { return g_cnn_err.c_str(); }

}  // extern "C"

namespace cgli {
// device time of the network's inference on the context's levels (packing
// and the five layers, not the update of U_), mean over reps
int cnn_time_inference(cgli_cnn *n, const Dev &d, cudaStream_t s, int reps, float *ms) {
  cudaEvent_t e0, e1;
  CC(cudaEventCreate(&e0));
  CC(cudaEventCreate(&e1));
  const unsigned nb = (unsigned)((n->cells + 255) / 256);
  CC(cudaEventRecord(e0, s));
  for (int r = 0; r < reps; r++) {
    k_pack_state<<<nb, 256, 0, s>>>(d, n->act[0], n->sc);
    launch_halo(n, n->act[0], s);
    forward(n, false, s);
  }
  CC(cudaEventRecord(e1, s));
  CC(cudaEventSynchronize(e1));
  float t = 0.f;
  CC(cudaEventElapsedTime(&t, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  *ms = t / reps;
  return check_status(n, s);
}

// stores the context's current level (U = Q^n after cgli_end_step) as physical Q
int cnn_store_level(cgli_cnn *n, const Dev &d, cudaStream_t s) {
  if (n->levels.empty()) return cfail(CGLI_ESTATE, "no level storage (cgli_cnn_reserve_levels)");
  float *dst = n->levels[n->nlevels % (long long)n->levels.size()];
  k_store_level<<<(unsigned)((n->cells + 255) / 256), 256, 0, s>>>(d, dst);
  CC(cudaGetLastError());
  CC(cudaStreamSynchronize(s));
  n->nlevels++;
  return CGLI_OK;
}
}  // namespace cgli
