// cnn_kernels.cuh -- the learned coarse-grid correction: a 4-layer 3x3x3
// conv3d network (2 -> 16 -> 16 -> 16 -> 2 channels, GELU between layers,
// BF16 weights and activations, FP32 accumulation) applied to psi after a
// coarse time step, and its training kernels.
//
// Activation layout (global and shared memory): bf16 [Zp][Yp][H][Xp][8] with
// Xp = nx + 2, Yp = ny + 2, Zp = nz + 2 (one periodic ghost site per side,
// written by the kernel that writes the interior) and the 16 channels split
// into H = 2 halves of 8.  One x-row half is therefore a run of 16-byte
// records, which is exactly the no-swizzle K-major core-matrix layout of a
// tcgen05 A operand (8 sites x 8 channels per 128-byte core matrix): the A
// operand of tap (dz, dy, dx) for 128 consecutive sites of a row is the row's
// address + 16 * dx, with LBO = the half stride.  No im2col copy exists.
//
// Forward / dgrad kernel: one CTA per (y-slab of 6 rows, z-chunk) item;
// warp 0 streams input planes (6 + 2 rows, both halves, the full padded x
// extent) into a 3-slot ring -- in this layout those rows are one contiguous
// range, fetched by a single 1-D bulk copy (a tensor-map tile with its
// 16-byte innermost extent moved the same bytes several times slower); warp 1 issues, per input plane and
// per (input row, dx), ONE tcgen05.mma (M = 128 sites, N = 144, K = 16)
// whose D block covers every output site that input row feeds: 3 output
// rows x 3 output planes x 16 channels.  A small MMA costs about 50 issue
// cycles whatever its N, so 24 MMAs of N = 144 per plane (near the tensor
// pipe's rate) replace 162 of N = 16.  The accumulators of three output
// planes rotate in TMEM; when an input plane's MMAs complete, one output
// plane is finished: warps 2-9 copy its rows to registers (tcgen05.ld
// 32x32b), zero its slot, release it to the MMA warp, and only then run the
// epilogue and the stores, which overlap the next plane's MMAs.  Every MMA
// accumulates; slots are zero when a plane first receives data.
//
// Weight-gradient kernel: D[(dy, ci), co] += X[(row y + dy), ci, x + dx] *
// dY[row y, co, x] summed over x in 16-site K steps; A (X) and B (dY) are
// MN-major operands read in place (8 consecutive rows x 2 halves form the
// 16 M-groups of an M = 128 operand, three of which are the dy taps), one
// accumulator per (dz, dx).  All waits are bounded; a timeout sets *status.
#pragma once

#include <cuda_bf16.h>

#include "device_utils.cuh"
#include "tcgen05.cuh"

namespace gpe {
namespace cnn {

constexpr int CH = 16;
constexpr int NTAP = 27;
constexpr int NLAYER = 4;
constexpr int TAP_BYTES = 2 * CH * 8 * 2;  // [2 halves][16 rows][8] bf16 = 512

// forward / dgrad
constexpr int TYF = 4;          // output rows per item
constexpr int FSLOTS = 2;       // input planes in the shared-memory ring
constexpr int F_EPI_WARPS = 8;  // one epilogue group: 2 warps per lane quarter
constexpr int F_THREADS = 32 * (2 + F_EPI_WARPS);
constexpr int F_CTAS_PER_SM = 2;  // one CTA's MMAs overlap the other's drain
// Accumulators: three output planes in a rotating ring (plane z in slot
// z mod 3), each with the TYF output rows of the slab, column
// (row * 3 + slot) * 16 + co.  Input row y' (box row i) of input plane j
// feeds output rows y'-1, y', y'+1 of output planes j-1, j, j+1 (all three
// slots): for an interior input row one contiguous block of 144 columns,
// so a single MMA with N = 144 covers all nine (dz, dy) taps of one dx; the
// slab's first two and last two input rows feed only one or two of its
// rows and use N = 48 / 96 with the matching part of B.
constexpr int OSLOTS = 3;
constexpr int ACC_ROWS = TYF;
constexpr int NSTACK = 3 * OSLOTS * CH;          // 144
constexpr uint32_t F_TMEM_COLS = 256;
static_assert(ACC_ROWS * OSLOTS * CH <= (int)F_TMEM_COLS, "accumulator ring fits TMEM");
// B tile of one (rotation j mod 3, dx): rows n = (jrow * 3 + s) * 16 + co
// hold tap (dz index 2 - ((s - rot + 1) mod 3), dy index 2 - jrow, dx);
// K = 16 input channels in two halves: [2][144][8] bf16.
constexpr int WT_BYTES = 2 * NSTACK * 8 * 2;     // 4608
constexpr int W_TILES = 9;                       // 3 rotations x 3 dx
// Per output-channel count: accumulator columns per (row, slot) and the
// MMA's N.  The last layer has 2 output channels: 9 x 2 = 18 columns padded
// to N = 32 (the 14 extra B rows are zero; they add exact zeros to columns
// of the next rows, which accumulate in the same MMA stream).
template <int CO>
struct OutShape {
  static constexpr int CW = CO;
  static constexpr int NB = CO == 16 ? NSTACK : 32;  // rows of one B tile
  static constexpr int WTB = 2 * NB * 8 * 2;
  // N of an MMA feeding `cnt` (1..3) of the slab's rows, rounded up to 16
  __host__ __device__ static constexpr int n_of(int cnt) {
    return CO == 16 ? 48 * cnt : ((6 * cnt + 15) / 16) * 16;
  }
};
static_assert(OutShape<2>::NB >= 9 * 2, "padded N holds the 18 real columns");
// every MMA's D block (padded N included) stays inside the allocation
static_assert((TYF - 1) * OSLOTS * 2 + 32 <= (int)F_TMEM_COLS, "padded blocks fit");
constexpr int EPI_ROWS = TYF / 2;                // rows per epilogue warp
// after the weights: 2*FSLOTS + 5 mbarriers, TMEM address, abort flag, 16 biases
constexpr int F_TAIL_BYTES = 256;
static_assert((2 * FSLOTS + 5) * 8 + 16 + 64 <= F_TAIL_BYTES, "tail fits");

// weight gradient
constexpr int TYW = 2;
constexpr int XROWS = TYW + 7;
constexpr int WSLOTS = 4;
constexpr int DSLOTS = 2;
constexpr int W_EPI_WARPS = 4;
constexpr int W_THREADS = 32 * (2 + W_EPI_WARPS);
constexpr uint32_t W_TMEM_COLS = 256;
constexpr int NACC = 9;  // (dz, dx) accumulators

enum Epi { EPI_GELU = 0, EPI_GELU_PRE = 1, EPI_DELTA = 2, EPI_RESID = 3, EPI_DGELU = 4 };

struct ConvParams {
  const __nv_bfloat16* in;          // input activations [Zp][Yp][Hin][Xp][8]
  const __nv_bfloat16* w;           // [27][2][16][8]
  const float* bias;                // [16] or null
  int nx, ny, nz, Xp, Yp, Zp, Hin;
  int nslab, nzc, zchunk, nitems;
  uint32_t slot_bytes, box_bytes;
  __nv_bfloat16* act_out;           // [Zp][Yp][2][Xp][8]
  __nv_bfloat16* pre_out;           // EPI_GELU_PRE
  const __nv_bfloat16* pre_in;      // EPI_DGELU
  float* delta;                     // EPI_DELTA: dense [nz][ny][nx][2]
  float* psi;                       // EPI_RESID: solver field (complex64, 2 ghosts)
  int psi_Nx, psi_Ny;
  float out_scale;
  int* status;
  unsigned long long wait_limit_ns;
};

struct WgradParams {
  const __nv_bfloat16* x;           // layer input [Zp][Yp][2][Xp][8]
  const __nv_bfloat16* dy;          // gradient of the layer output, same layout
  int nx, ny, nz, Xp, Yp, Zp;
  int nslab, nzc, zchunk, nitems;
  uint32_t xslot_bytes, xbox_bytes, dslot_bytes, dbox_bytes;
  float* partials;                  // [gridDim.x][NACC][128][16]
  int* status;
  unsigned long long wait_limit_ns;
};

// GELU in its tanh form (Hendrycks & Gimpel, 2016):
//   gelu(x) = 0.5 x (1 + t),  t = tanh(u),  u = sqrt(2/pi) (x + 0.044715 x^3),
//   gelu'(x) = 0.5 (1 + t) + 0.5 x (1 - t^2) u',  u' = sqrt(2/pi) (1 + 3 * 0.044715 x^2).
// tanh through the hardware tanh.approx.f32 instruction (one MUFU operation,
// relative error about 2^-11, below the bfloat16 rounding of the result).
constexpr float GELU_C = 0.7978845608028654f;  // sqrt(2/pi)
constexpr float GELU_A = 0.044715f;

__device__ __forceinline__ float tanh_approx(float u) {
  float t;
  asm("tanh.approx.f32 %0, %1;" : "=f"(t) : "f"(u));
  return t;
}
__device__ __forceinline__ float gelu(float x) {
  const float t = tanh_approx(GELU_C * fmaf(GELU_A * x, x * x, x));
  const float hx = 0.5f * x;
  return fmaf(hx, t, hx);
}
// Two values at once on the packed FP32x2 pipe: u = x (C + C A x^2),
// gelu = h + h t with h = x / 2, t = tanh(u) (two scalar MUFU operations).
__device__ __forceinline__ float2 gelu2(float2 x) {
  const float2 x2 = __fmul2_rn(x, x);
  const float2 k = __ffma2_rn(make_float2(GELU_C * GELU_A, GELU_C * GELU_A), x2,
                              make_float2(GELU_C, GELU_C));
  const float2 u = __fmul2_rn(x, k);
  const float2 t = make_float2(tanh_approx(u.x), tanh_approx(u.y));
  const float2 h = __fmul2_rn(x, make_float2(0.5f, 0.5f));
  return __ffma2_rn(h, t, h);
}
__device__ __forceinline__ float gelu_grad(float x) {
  const float t = tanh_approx(GELU_C * fmaf(GELU_A * x, x * x, x));
  const float du = GELU_C * fmaf(3.0f * GELU_A * x, x, 1.0f);
  return fmaf(0.5f * x * fmaf(-t, t, 1.0f), du, 0.5f * (1.0f + t));
}

__device__ __forceinline__ size_t act_index(int Xp, int Yp, int x, int y, int z, int h) {
  return ((((size_t)z * Yp + y) * 2 + h) * Xp + x) * 8;
}

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&v);
}

// The interior site (x, y, z) and its periodic ghost images (halo 1), in
// padded coordinates.  Up to three images per axis (n = 1 has both ghosts).
template <typename F>
__device__ __forceinline__ void for_images(int x, int y, int z, int nx, int ny, int nz, F f) {
  const int x1 = x == 0 ? nx + 1 : -1, x2 = x == nx - 1 ? 0 : -1;
  const int y1 = y == 0 ? ny + 1 : -1, y2 = y == ny - 1 ? 0 : -1;
  const int z1 = z == 0 ? nz + 1 : -1, z2 = z == nz - 1 ? 0 : -1;
  if ((x1 & x2 & y1 & y2 & z1 & z2) == -1) {  // interior: no ghost image
    f(x + 1, y + 1, z + 1);
    return;
  }
#pragma unroll
  for (int c = 0; c < 3; c++) {
    const int zp = c == 0 ? z + 1 : (c == 1 ? z1 : z2);
    if (zp < 0) continue;
#pragma unroll
    for (int b = 0; b < 3; b++) {
      const int yp = b == 0 ? y + 1 : (b == 1 ? y1 : y2);
      if (yp < 0) continue;
#pragma unroll
      for (int a = 0; a < 3; a++) {
        const int xp = a == 0 ? x + 1 : (a == 1 ? x1 : x2);
        if (xp < 0) continue;
        f(xp, yp, zp);
      }
    }
  }
}

// 16 channels of one site (two 16-byte records) into a [.][.][2][Xp][8]
// buffer, ghosts included.
__device__ __forceinline__ void store_act16(__nv_bfloat16* buf, int Xp, int Yp, int nx, int ny,
                                            int nz, int x, int y, int z, const float (&a)[16],
                                            bool ghosts) {
  uint4 lo, hi;
  lo.x = pack_bf16x2(a[0], a[1]);   lo.y = pack_bf16x2(a[2], a[3]);
  lo.z = pack_bf16x2(a[4], a[5]);   lo.w = pack_bf16x2(a[6], a[7]);
  hi.x = pack_bf16x2(a[8], a[9]);   hi.y = pack_bf16x2(a[10], a[11]);
  hi.z = pack_bf16x2(a[12], a[13]); hi.w = pack_bf16x2(a[14], a[15]);
  if (!ghosts) {
    *reinterpret_cast<uint4*>(buf + act_index(Xp, Yp, x + 1, y + 1, z + 1, 0)) = lo;
    *reinterpret_cast<uint4*>(buf + act_index(Xp, Yp, x + 1, y + 1, z + 1, 1)) = hi;
    return;
  }
  for_images(x, y, z, nx, ny, nz, [&](int xp, int yp, int zp) {
    *reinterpret_cast<uint4*>(buf + act_index(Xp, Yp, xp, yp, zp, 0)) = lo;
    *reinterpret_cast<uint4*>(buf + act_index(Xp, Yp, xp, yp, zp, 1)) = hi;
  });
}

__device__ __forceinline__ void load_act16(const __nv_bfloat16* buf, int Xp, int Yp, int x,
                                           int y, int z, float (&a)[16]) {
  const uint4 lo = *reinterpret_cast<const uint4*>(buf + act_index(Xp, Yp, x + 1, y + 1, z + 1, 0));
  const uint4 hi = *reinterpret_cast<const uint4*>(buf + act_index(Xp, Yp, x + 1, y + 1, z + 1, 1));
  const uint32_t w[8] = {lo.x, lo.y, lo.z, lo.w, hi.x, hi.y, hi.z, hi.w};
#pragma unroll
  for (int i = 0; i < 8; i++) {
    const __nv_bfloat162 v = *reinterpret_cast<const __nv_bfloat162*>(&w[i]);
    const float2 f = __bfloat1622float2(v);
    a[2 * i] = f.x;
    a[2 * i + 1] = f.y;
  }
}

__device__ __forceinline__ void set_abort(int* status, volatile int* flag, int code) {
  *flag = 1;
  atomicExch(status, code);
}

// --------------------------------------------------------------------------
// Forward / dgrad convolution.

// Global data an epilogue reads besides the accumulators: the stored
// pre-activation (dgrad) or the solver's psi (residual).  Loaded for every
// row of a plane before any of them is computed, so the latencies overlap.
struct EpiAux {
  uint4 lo, hi;
  float2 psi;
};

__device__ __forceinline__ size_t psi_index(const ConvParams& p, int x, int y, int z) {
  return ((size_t)(z + 2) * p.psi_Ny + (y + 2)) * p.psi_Nx + (x + 2);
}

template <int EPI>
__device__ __forceinline__ void epi_load(const ConvParams& p, int x, int y, int z, EpiAux& a) {
  if (EPI == EPI_DGELU) {
    a.lo = *reinterpret_cast<const uint4*>(p.pre_in + act_index(p.Xp, p.Yp, x + 1, y + 1, z + 1, 0));
    a.hi = *reinterpret_cast<const uint4*>(p.pre_in + act_index(p.Xp, p.Yp, x + 1, y + 1, z + 1, 1));
  } else if (EPI == EPI_RESID) {
    a.psi = reinterpret_cast<const float2*>(p.psi)[psi_index(p, x, y, z)];
  }
}

template <int EPI>
__device__ __forceinline__ void conv_epilogue(const ConvParams& p, const float (&acc)[16],
                                              const float* bias, const EpiAux& aux, int x, int y,
                                              int z) {
  if (EPI == EPI_GELU || EPI == EPI_GELU_PRE) {
    float pre[16], a[16];
#pragma unroll
    for (int c = 0; c < 16; c += 2) {
      const float2 v = __fadd2_rn(make_float2(acc[c], acc[c + 1]), make_float2(bias[c], bias[c + 1]));
      const float2 g = gelu2(v);
      pre[c] = v.x;
      pre[c + 1] = v.y;
      a[c] = g.x;
      a[c + 1] = g.y;
    }
    if (EPI == EPI_GELU_PRE) store_act16(p.pre_out, p.Xp, p.Yp, p.nx, p.ny, p.nz, x, y, z, pre, false);
    store_act16(p.act_out, p.Xp, p.Yp, p.nx, p.ny, p.nz, x, y, z, a, true);
  } else if (EPI == EPI_DGELU) {
    float g[16];
    const uint32_t w[8] = {aux.lo.x, aux.lo.y, aux.lo.z, aux.lo.w, aux.hi.x, aux.hi.y, aux.hi.z, aux.hi.w};
#pragma unroll
    for (int i = 0; i < 8; i++) {
      const float2 f = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&w[i]));
      g[2 * i] = acc[2 * i] * gelu_grad(f.x);
      g[2 * i + 1] = acc[2 * i + 1] * gelu_grad(f.y);
    }
    store_act16(p.act_out, p.Xp, p.Yp, p.nx, p.ny, p.nz, x, y, z, g, true);
  } else if (EPI == EPI_DELTA) {
    const size_t s = ((size_t)z * p.ny + y) * p.nx + x;
    reinterpret_cast<float2*>(p.delta)[s] =
        make_float2((acc[0] + bias[0]) * p.out_scale, (acc[1] + bias[1]) * p.out_scale);
  } else {  // EPI_RESID: psi += delta on the solver's field, ghosts (2, periodic) too
    float2 v = aux.psi;
    v.x += (acc[0] + bias[0]) * p.out_scale;
    v.y += (acc[1] + bias[1]) * p.out_scale;
    float2* f = reinterpret_cast<float2*>(p.psi);
    int gx[3] = {x, NO_GHOST, NO_GHOST}, gy[3] = {y, NO_GHOST, NO_GHOST},
        gz[3] = {z, NO_GHOST, NO_GHOST};
    ghost_targets(x, p.nx, 1, gx[1], gx[2]);
    ghost_targets(y, p.ny, 1, gy[1], gy[2]);
    ghost_targets(z, p.nz, 1, gz[1], gz[2]);
#pragma unroll
    for (int c = 0; c < 3; c++) {
      if (gz[c] == NO_GHOST) continue;
#pragma unroll
      for (int b = 0; b < 3; b++) {
        if (gy[b] == NO_GHOST) continue;
#pragma unroll
        for (int a = 0; a < 3; a++) {
          if (gx[a] == NO_GHOST) continue;
          f[psi_index(p, gx[a], gy[b], gz[c])] = v;
        }
      }
    }
  }
}

template <int EPI, int CO>
__global__ void __launch_bounds__(F_THREADS, F_CTAS_PER_SM)
conv_fwd_kernel(const __grid_constant__ ConvParams p) {
  constexpr int CW = OutShape<CO>::CW, NB = OutShape<CO>::NB, WTB = OutShape<CO>::WTB;
  extern __shared__ unsigned char smem_raw[];
  unsigned char* ring = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* wsm = ring + FSLOTS * p.slot_bytes + 4096;  // 4 KB of zeros after the ring
  uint64_t* full = reinterpret_cast<uint64_t*>(wsm + W_TILES * WTB);
  uint64_t* empty = full + FSLOTS;
  uint64_t* accf = empty + FSLOTS;  // MMAs of one input plane done
  uint64_t* acce = accf + 1;        // the finished output plane's slot is drained
  uint64_t* drain = acce + 1;
  uint32_t* tmem_holder = reinterpret_cast<uint32_t*>(drain + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_holder + 1);
  float* bias_s = reinterpret_cast<float*>(tmem_holder + 4);  // [16], 16-byte aligned

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  {  // weights and the zero pad (generic proxy), then make them visible to the tensor core
    const uint4* src = reinterpret_cast<const uint4*>(p.w);
    uint4* dst = reinterpret_cast<uint4*>(wsm);
    for (int i = threadIdx.x; i < W_TILES * WTB / 16; i += blockDim.x) dst[i] = src[i];
    // the whole ring and the pad start at zero: rows a copy leaves
    // untouched (past the grid's last row) and over-reads stay finite
    uint4* z = reinterpret_cast<uint4*>(ring);
    for (int i = threadIdx.x; i < (int)(FSLOTS * p.slot_bytes + 4096) / 16; i += blockDim.x)
      z[i] = make_uint4(0, 0, 0, 0);
  }
  if (threadIdx.x < 16) bias_s[threadIdx.x] = p.bias ? p.bias[threadIdx.x] : 0.0f;
  if (threadIdx.x == 0) {
    for (int s = 0; s < FSLOTS; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    mbar_init(accf, 1);
    mbar_init(acce, 32 * F_EPI_WARPS);
    mbar_init(drain, 1);
    *abort_flag = 0;
    fence_mbar_init();
  }
  fence_proxy_async();
  if (warp == 1) tc::tmem_alloc(smem_u32(tmem_holder), F_TMEM_COLS);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tmem_holder;
  const uint64_t lim = p.wait_limit_ns;
  const uint32_t row_bytes = (uint32_t)p.Xp * 16;
  if (warp >= 2) {  // the whole allocation starts at zero
    const int q = warp & 3, half = (warp - 2) >> 2;
    for (int a = half; a < (int)F_TMEM_COLS / 16; a += 2)
      tc::st_32x32b_x16_zero(tmem + ((uint32_t)(32 * q) << 16) + a * 16);
    tc::wait_st();
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();

  if (warp == 0) {
    if (lane == 0) {
      const size_t row_elems = (size_t)p.Hin * p.Xp * 8;
      const size_t plane_elems = (size_t)p.Yp * row_elems;
      uint32_t g = 0;
      for (int it = blockIdx.x; it < p.nitems && !*abort_flag; it += gridDim.x) {
        const int slab = it % p.nslab, zc = it / p.nslab;
        const int y0 = slab * TYF, z0 = zc * p.zchunk;
        const int nout = min(z0 + p.zchunk, p.nz) - z0;
        for (int pl = 0; pl < nout + 2; pl++, g++) {
          const uint32_t slot = g % FSLOTS, cyc = g / FSLOTS;
          if (cyc > 0 && !mbar_wait_bounded(&empty[slot], (cyc - 1) & 1, lim)) {
            set_abort(p.status, abort_flag, 1);
            break;
          }
          // rows y0 .. y0+TYF+1 (padded) of plane z0+pl: one contiguous range
          const uint32_t bytes = (uint32_t)min(TYF + 2, p.Yp - y0) * (uint32_t)(row_elems * 2);
          mbar_arrive_expect_tx(&full[slot], bytes);
          tc::bulk_load(smem_u32(ring + slot * p.slot_bytes),
                        p.in + (size_t)(z0 + pl) * plane_elems + (size_t)y0 * row_elems, bytes,
                        smem_u32(&full[slot]));
        }
      }
      const uint32_t first = g > FSLOTS ? g - FSLOTS : 0;
      for (uint32_t q = first; q < g; q++)
        if (!mbar_wait_bounded(&full[q % FSLOTS], (q / FSLOTS) & 1, lim)) {
          set_abort(p.status, abort_flag, 1);
          break;
        }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      constexpr int BROW = OSLOTS * CW;  // B rows / D columns per output row
      const uint32_t idesc1 = tc::idesc_bf16_f32(128, OutShape<CO>::n_of(1), false, false);
      const uint32_t idesc2 = tc::idesc_bf16_f32(128, OutShape<CO>::n_of(2), false, false);
      const uint32_t idesc3 = tc::idesc_bf16_f32(128, OutShape<CO>::n_of(3), false, false);
      const uint32_t lbo_a = p.Hin == 2 ? row_bytes : 0;
      const uint32_t ring_s = smem_u32(ring), w_s = smem_u32(wsm);
      const uint64_t bdesc0 = tc::smem_desc(w_s, NB * 16, 128);
      const uint64_t adesc0 = tc::smem_desc(ring_s, lbo_a, 128);
      const uint32_t row_step = (uint32_t)p.Hin * row_bytes;
      uint32_t g = 0, e = 0;  // input planes, steps (one per input plane)
      for (int it = blockIdx.x; it < p.nitems && !*abort_flag; it += gridDim.x) {
        const int slab = it % p.nslab, zc = it / p.nslab;
        const int y0 = slab * TYF, z0 = zc * p.zchunk;
        const int nout = min(z0 + p.zchunk, p.nz) - z0;
        const int nin = min(TYF, p.ny - y0) + 2;  // input rows y0-1 .. y0+nrows
        for (int t = 0; t < nout + 2 && !*abort_flag; t++, g++, e++) {
          const int j = z0 - 1 + t;  // input plane (may be -1: its ghost plane)
          bool ok = mbar_wait_bounded(&full[g % FSLOTS], (g / FSLOTS) & 1, lim);
          if (ok && e > 0) ok = mbar_wait_bounded(acce, (e - 1) & 1, lim);
          if (!ok) {
            set_abort(p.status, abort_flag, 1);
            break;
          }
          tc::fence_after_sync();
          const uint64_t ab = adesc0 + ((g % FSLOTS) * p.slot_bytes >> 4);
          const uint64_t bb = bdesc0 + (uint64_t)(((j + 3) % 3) * 3 * WTB / 16);
#pragma unroll
          for (int i = 0; i < TYF + 2; i++) {
            // input row i feeds slab rows i-2 .. i: keep those inside [0, TYF)
            const int jlo = i < 2 ? 2 - i : 0;
            const int jhi = i > TYF - 1 ? TYF + 1 - i : 2;
            const int cnt = jhi - jlo + 1;
            const uint32_t idesc = cnt == 3 ? idesc3 : (cnt == 2 ? idesc2 : idesc1);
            const uint32_t d = tmem + (uint32_t)((i - 2 + jlo) * BROW);
            const uint64_t b = bb + (uint64_t)(jlo * BROW * 16 / 16);
            if (i < nin) {
#pragma unroll
              for (int dx = 0; dx < 3; dx++)
                tc::mma_bf16(d, ab + ((i * row_step + dx * 16) >> 4), b + (uint64_t)(dx * WTB / 16),
                             idesc, 1u);
            }
          }
          tc::commit(smem_u32(accf));
          tc::commit(smem_u32(&empty[g % FSLOTS]));
        }
      }
      tc::commit(smem_u32(drain));
      if (!mbar_wait_bounded(drain, 0, lim)) set_abort(p.status, abort_flag, 1);
    }
  } else {
    const int q = warp & 3, half = (warp - 2) >> 2;
    const int x = 32 * q + lane;
    const uint32_t tq = tmem + ((uint32_t)(32 * q) << 16);
    uint32_t e = 0;
    for (int it = blockIdx.x; it < p.nitems && !*abort_flag; it += gridDim.x) {
      const int slab = it % p.nslab, zc = it / p.nslab;
      const int y0 = slab * TYF, z0 = zc * p.zchunk;
      const int nout = min(z0 + p.zchunk, p.nz) - z0;
      const int nrows = min(TYF, p.ny - y0);
      bool stop = false;
      for (int t = 0; t < nout + 2; t++, e++) {
        if (!mbar_wait_bounded(accf, e & 1, lim)) {
          set_abort(p.status, abort_flag, 1);
          stop = true;
          break;
        }
        tc::fence_after_sync();
        const int zo = z0 - 2 + t;  // output plane finished by input plane zo + 1
        const bool real = zo >= z0;
        const bool mine = real && x < p.nx;
        const uint32_t so = (uint32_t)((zo + 3) % 3);
        EpiAux aux[EPI_ROWS];
        if (mine) {
#pragma unroll
          for (int k = 0; k < EPI_ROWS; k++)
            if (half + 2 * k < nrows) epi_load<EPI>(p, x, y0 + half + 2 * k, zo, aux[k]);
        }
        float v[EPI_ROWS][16];
        if (real) {
#pragma unroll
          for (int k = 0; k < EPI_ROWS; k++) {
            const int r = half + 2 * k;
            if (r < nrows) {
              if (CW == 16) tc::ld_32x32b_x16(tq + (r * OSLOTS + so) * CW, v[k]);
              else tc::ld_32x32b_x2(tq + (r * OSLOTS + so) * CW, v[k]);
            }
          }
        }
        const bool last = t == nout + 1;
        for (int a = half; a < ACC_ROWS; a += 2) {
#pragma unroll
          for (int ds = 0; ds < 3; ds++) {
            if (ds > 0 && !last) break;  // at the chunk's end: junk of the planes past it
            const uint32_t col = (a * OSLOTS + (so + ds) % 3) * CW;
            if (CW == 16) tc::st_32x32b_x16_zero(tq + col);
            else tc::st_32x32b_x2_zero(tq + col);
          }
        }
        tc::wait_st();
        tc::fence_before_sync();
        mbar_arrive(acce);
        if (mine) {
#pragma unroll
          for (int k = 0; k < EPI_ROWS; k++) {
            const int r = half + 2 * k;
            if (r < nrows) conv_epilogue<EPI>(p, v[k], bias_s, aux[k], x, y0 + r, zo);
          }
        }
      }
      if (stop) break;
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 1) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, F_TMEM_COLS);
  }
}

// --------------------------------------------------------------------------
// Weight gradient.

__global__ void __launch_bounds__(W_THREADS, 1) conv_wgrad_kernel(const __grid_constant__ WgradParams p) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* xring = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* dring = xring + WSLOTS * p.xslot_bytes;
  uint64_t* xfull = reinterpret_cast<uint64_t*>(dring + DSLOTS * p.dslot_bytes);
  uint64_t* xempty = xfull + WSLOTS;
  uint64_t* dfull = xempty + WSLOTS;
  uint64_t* dempty = dfull + DSLOTS;
  uint64_t* drain = dempty + DSLOTS;
  uint32_t* tmem_holder = reinterpret_cast<uint32_t*>(drain + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_holder + 1);
  volatile int* any_flag = abort_flag + 1;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  {  // rings start at zero: rows a copy leaves untouched stay finite
    uint4* z = reinterpret_cast<uint4*>(xring);
    const int n16 = (int)(WSLOTS * p.xslot_bytes + DSLOTS * p.dslot_bytes) / 16;
    for (int i = threadIdx.x; i < n16; i += blockDim.x) z[i] = make_uint4(0, 0, 0, 0);
  }
  fence_proxy_async();
  if (threadIdx.x == 0) {
    for (int s = 0; s < WSLOTS; s++) {
      mbar_init(&xfull[s], 1);
      mbar_init(&xempty[s], 1);
    }
    for (int s = 0; s < DSLOTS; s++) {
      mbar_init(&dfull[s], 1);
      mbar_init(&dempty[s], 1);
    }
    mbar_init(drain, 1);
    *abort_flag = 0;
    *any_flag = 0;
    fence_mbar_init();
  }
  if (warp == 1) tc::tmem_alloc(smem_u32(tmem_holder), W_TMEM_COLS);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tmem_holder;
  const uint64_t lim = p.wait_limit_ns;
  const uint32_t row_bytes = (uint32_t)p.Xp * 16;

  if (warp == 0) {
    if (lane == 0) {
      const size_t row_elems = (size_t)2 * p.Xp * 8;
      const size_t plane_elems = (size_t)p.Yp * row_elems;
      uint32_t gx = 0, gd = 0;
      auto load_x = [&](int y0, int zpad) -> bool {
        const uint32_t slot = gx % WSLOTS, cyc = gx / WSLOTS;
        if (cyc > 0 && !mbar_wait_bounded(&xempty[slot], (cyc - 1) & 1, lim)) return false;
        const uint32_t bytes = (uint32_t)min(XROWS, p.Yp - y0) * (uint32_t)(row_elems * 2);
        mbar_arrive_expect_tx(&xfull[slot], bytes);
        tc::bulk_load(smem_u32(xring + slot * p.xslot_bytes),
                      p.x + (size_t)zpad * plane_elems + (size_t)y0 * row_elems, bytes,
                      smem_u32(&xfull[slot]));
        gx++;
        return true;
      };
      auto load_d = [&](int y0, int zpad) -> bool {
        const uint32_t slot = gd % DSLOTS, cyc = gd / DSLOTS;
        if (cyc > 0 && !mbar_wait_bounded(&dempty[slot], (cyc - 1) & 1, lim)) return false;
        const uint32_t bytes = (uint32_t)min(TYW, p.Yp - (y0 + 1)) * (uint32_t)(row_elems * 2);
        mbar_arrive_expect_tx(&dfull[slot], bytes);
        tc::bulk_load(smem_u32(dring + slot * p.dslot_bytes),
                      p.dy + (size_t)zpad * plane_elems + (size_t)(y0 + 1) * row_elems, bytes,
                      smem_u32(&dfull[slot]));
        gd++;
        return true;
      };
      bool ok = true;
      for (int it = blockIdx.x; it < p.nitems && ok && !*abort_flag; it += gridDim.x) {
        const int slab = it % p.nslab, zc = it / p.nslab;
        const int y0 = slab * TYW, z0 = zc * p.zchunk;
        const int nout = min(z0 + p.zchunk, p.nz) - z0;
        ok = load_x(y0, z0) && load_x(y0, z0 + 1);
        for (int o = 0; o < nout && ok; o++) ok = load_x(y0, z0 + o + 2) && load_d(y0, z0 + o + 1);
      }
      if (!ok) set_abort(p.status, abort_flag, 1);
      const uint32_t fx = gx > WSLOTS ? gx - WSLOTS : 0;
      for (uint32_t q = fx; q < gx; q++)
        if (!mbar_wait_bounded(&xfull[q % WSLOTS], (q / WSLOTS) & 1, lim)) {
          set_abort(p.status, abort_flag, 1);
          break;
        }
      const uint32_t fd = gd > DSLOTS ? gd - DSLOTS : 0;
      for (uint32_t q = fd; q < gd; q++)
        if (!mbar_wait_bounded(&dfull[q % DSLOTS], (q / DSLOTS) & 1, lim)) {
          set_abort(p.status, abort_flag, 1);
          break;
        }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = tc::idesc_bf16_f32(128, 16, true, true);
      const uint32_t xring_s = smem_u32(xring), dring_s = smem_u32(dring);
      uint32_t gx0 = 0, gd0 = 0, xw = 0, dw = 0;
      bool started = false;
      const int nxc = p.nx / 16;
      for (int it = blockIdx.x; it < p.nitems && !*abort_flag; it += gridDim.x) {
        const int slab = it % p.nslab, zc = it / p.nslab;
        const int y0 = slab * TYW, z0 = zc * p.zchunk;
        const int nout = min(z0 + p.zchunk, p.nz) - z0;
        const int nrows = min(TYW, p.ny - y0);
        for (int o = 0; o < nout && !*abort_flag; o++) {
          bool ok = true;
          while (ok && xw < gx0 + o + 3) {
            ok = mbar_wait_bounded(&xfull[xw % WSLOTS], (xw / WSLOTS) & 1, lim);
            if (ok) xw++;
          }
          while (ok && dw < gd0 + o + 1) {
            ok = mbar_wait_bounded(&dfull[dw % DSLOTS], (dw / DSLOTS) & 1, lim);
            if (ok) dw++;
          }
          if (!ok) {
            set_abort(p.status, abort_flag, 1);
            break;
          }
          tc::fence_after_sync();
          uint32_t xb[3];
#pragma unroll
          for (int dz = 0; dz < 3; dz++) xb[dz] = xring_s + ((gx0 + o + dz) % WSLOTS) * p.xslot_bytes;
          const uint32_t db = dring_s + ((gd0 + o) % DSLOTS) * p.dslot_bytes;
          for (int r = 0; r < nrows; r++) {
            for (int xc = 0; xc < nxc; xc++) {
              const uint64_t bdesc = tc::smem_desc(db + (uint32_t)(r * 2) * row_bytes +
                                                       (uint32_t)(1 + 16 * xc) * 16,
                                                   128, row_bytes);
#pragma unroll
              for (int dz = 0; dz < 3; dz++)
#pragma unroll
                for (int dx = 0; dx < 3; dx++) {
                  const uint64_t adesc = tc::smem_desc(
                      xb[dz] + (uint32_t)(r * 2) * row_bytes + (uint32_t)(16 * xc + dx) * 16, 128,
                      row_bytes);
                  tc::mma_bf16(tmem + (dz * 3 + dx) * 16, adesc, bdesc, idesc, started ? 1u : 0u);
                }
              started = true;
            }
          }
          tc::commit(smem_u32(&xempty[(gx0 + o) % WSLOTS]));
          tc::commit(smem_u32(&dempty[(gd0 + o) % DSLOTS]));
        }
        if (*abort_flag) break;
        tc::commit(smem_u32(&xempty[(gx0 + nout) % WSLOTS]));
        tc::commit(smem_u32(&xempty[(gx0 + nout + 1) % WSLOTS]));
        gx0 += nout + 2;
        gd0 += nout;
      }
      if (started) *any_flag = 1;
      tc::commit(smem_u32(drain));
      if (!mbar_wait_bounded(drain, 0, lim)) set_abort(p.status, abort_flag, 1);
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (warp >= 2) {
    const int q = warp & 3;
    const int m = 32 * q + lane;
    float* out = p.partials + (size_t)blockIdx.x * NACC * 128 * 16;
    const bool any = *any_flag && !*abort_flag;
    for (int a = 0; a < NACC; a++) {
      float v[16];
      tc::ld_32x32b_x16(tmem + ((uint32_t)(32 * q) << 16) + a * 16, v);
      float4* o4 = reinterpret_cast<float4*>(out + ((size_t)a * 128 + m) * 16);
#pragma unroll
      for (int i = 0; i < 4; i++)
        o4[i] = any ? make_float4(v[4 * i], v[4 * i + 1], v[4 * i + 2], v[4 * i + 3])
                    : make_float4(0.f, 0.f, 0.f, 0.f);
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 1) {
    tc::fence_after_sync();
    tc::tmem_dealloc(tmem, W_TMEM_COLS);
  }
}

// --------------------------------------------------------------------------
// Element-wise and reduction kernels.

// Solver field (2 ghosts, pitches Nx, Ny; complex of TS) -> first-layer input
// (channels Re, Im, 0, ...; H halves), ghosts included.  Every padded site
// reads its periodic interior source (the solver keeps only the face ghosts
// a star stencil needs, not edges and corners): one block per padded (y, z)
// row, consecutive threads along x.
template <typename TS>
__global__ void pack_input_kernel(const TS* __restrict__ psi, int Nx, int Ny, int nx, int ny,
                                  int nz, __nv_bfloat16* __restrict__ act, int H) {
  const int Xp = nx + 2, Yp = ny + 2;
  const int row = blockIdx.x;  // zp * Yp + yp
  const int yp = row % Yp, zp = row / Yp;
  const int y = yp == 0 ? ny - 1 : (yp == ny + 1 ? 0 : yp - 1);
  const int z = zp == 0 ? nz - 1 : (zp == nz + 1 ? 0 : zp - 1);
  const size_t q0 = ((size_t)(z + 2) * Ny + (y + 2)) * Nx + 2;
  __nv_bfloat16* dst = act + (size_t)row * H * Xp * 8;
  const uint4 zero = make_uint4(0, 0, 0, 0);
  for (int xp = threadIdx.x; xp < Xp; xp += blockDim.x) {
    const int x = xp == 0 ? nx - 1 : (xp == nx + 1 ? 0 : xp - 1);
    const size_t q = q0 + x;
    *reinterpret_cast<uint4*>(dst + (size_t)xp * 8) =
        make_uint4(pack_bf16x2((float)psi[2 * q], (float)psi[2 * q + 1]), 0, 0, 0);
    if (H == 2) *reinterpret_cast<uint4*>(dst + ((size_t)Xp + xp) * 8) = zero;
  }
}

// Loss of one training pair and the gradient with respect to the last
// layer's output: e = u + delta - target, loss = sum |e|^2 / n,
// dL/d(out_c) = 2 e_c out_scale / n into channels 0, 1 of g (others 0).
template <typename TS, typename TT>
__global__ void loss_kernel(const float* __restrict__ delta, const TS* __restrict__ u, int Nx,
                            int Ny, const TT* __restrict__ target, int nx, int ny, int nz,
                            float out_scale, __nv_bfloat16* __restrict__ g,
                            double* __restrict__ partials) {
  __shared__ double red[32];
  const int Xp = nx + 2, Yp = ny + 2;
  const size_t n = (size_t)nx * ny * nz;
  const double inv_n = 1.0 / (double)n;
  double acc = 0.0;
  for (size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x; s < n;
       s += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(s % nx);
    const size_t t = s / nx;
    const int y = (int)(t % ny), z = (int)(t / ny);
    const size_t q = ((size_t)(z + 2) * Ny + (y + 2)) * Nx + (x + 2);
    const double er = (double)u[2 * q] + (double)delta[2 * s] - (double)target[2 * s];
    const double ei = (double)u[2 * q + 1] + (double)delta[2 * s + 1] - (double)target[2 * s + 1];
    acc += er * er + ei * ei;
    float a[16] = {};
    a[0] = (float)(2.0 * er * inv_n * out_scale);
    a[1] = (float)(2.0 * ei * inv_n * out_scale);
    store_act16(g, Xp, Yp, nx, ny, nz, x, y, z, a, true);
  }
  acc = warp_sum(acc);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
    partials[blockIdx.x] = t;
  }
}

// Per-block channel sums of a gradient buffer's interior (bias gradient).
__global__ void channel_sum_kernel(const __nv_bfloat16* __restrict__ g, int nx, int ny, int nz,
                                   float* __restrict__ partials) {
  __shared__ float red[256][17];
  const int Xp = nx + 2, Yp = ny + 2;
  const size_t n = (size_t)nx * ny * nz;
  float acc[16] = {};
  for (size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x; s < n;
       s += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(s % nx);
    const size_t t = s / nx;
    const int y = (int)(t % ny), z = (int)(t / ny);
    float a[16];
    load_act16(g, Xp, Yp, x, y, z, a);
#pragma unroll
    for (int c = 0; c < 16; c++) acc[c] += a[c];
  }
#pragma unroll
  for (int c = 0; c < 16; c++) red[threadIdx.x][c] = acc[c];
  __syncthreads();
  if (threadIdx.x < 16) {
    float t = 0.f;
    for (int i = 0; i < (int)blockDim.x; i++) t += red[i][threadIdx.x];
    partials[blockIdx.x * 16 + threadIdx.x] = t;
  }
}

// dW[tap][co][ci] (fp32) of one layer from the wgrad partials, and db from
// the channel sums.  One thread per weight; fixed summation order.
__global__ void grad_finalize_kernel(const float* __restrict__ wpart, int nwblk,
                                     const float* __restrict__ bpart, int nbblk,
                                     float* __restrict__ dw, float* __restrict__ db) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < NTAP * 16 * 16) {
    const int ci = i % 16, co = (i / 16) % 16, tap = i / 256;
    const int dz = tap / 9, dy = (tap / 3) % 3, dx = tap % 3;
    const int a = dz * 3 + dx, m = dy * 16 + ci;
    float t = 0.f;
    for (int b = 0; b < nwblk; b++) t += wpart[(((size_t)b * NACC + a) * 128 + m) * 16 + co];
    dw[i] = t;
  } else if (i < NTAP * 16 * 16 + 16) {
    const int c = i - NTAP * 16 * 16;
    float t = 0.f;
    for (int b = 0; b < nbblk; b++) t += bpart[b * 16 + c];
    db[c] = t;
  }
}

// Adam (Kingma & Ba) on the masked parameters of all layers.
__global__ void adam_kernel(float* __restrict__ w, const float* __restrict__ g,
                            float* __restrict__ m, float* __restrict__ v,
                            const unsigned char* __restrict__ mask, int n, float lr, float b1,
                            float b2, float eps, float c1, float c2) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n || !mask[i]) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  w[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

// fp32 weights [L][27][16 co][16 ci] -> bf16 B tiles [L][rot][dx][2 halves]
// [144 rows][8] (layout of the forward kernel's stacked B operand), K =
// input channel 8h + c.  The dgrad tiles hold the mirrored tap with co and
// ci exchanged (the adjoint convolution).
__global__ void pack_weights_kernel(const float* __restrict__ w, __nv_bfloat16* __restrict__ wf,
                                    __nv_bfloat16* __restrict__ wt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NLAYER * W_TILES * 2 * NSTACK * 8) return;
  const int c = i % 8, n = (i / 8) % NSTACK, h = (i / (8 * NSTACK)) % 2,
            tile = (i / (16 * NSTACK)) % W_TILES, l = i / (16 * NSTACK * W_TILES);
  const int rot = tile / 3, dx = tile % 3;
  const int co = n % 16, sj = n / 16, s = sj % 3, jrow = sj / 3;
  const int dz = 2 - (((s - rot + 1) % 3 + 3) % 3);
  const int tap = dz * 9 + (2 - jrow) * 3 + dx;
  const int k = 8 * h + c;
  const size_t base = (size_t)l * NTAP * 256;
  wf[i] = __float2bfloat16_rn(w[base + (size_t)tap * 256 + co * 16 + k]);
  wt[i] = __float2bfloat16_rn(w[base + (size_t)(NTAP - 1 - tap) * 256 + k * 16 + co]);
}

// The last layer (2 output channels) in the N = 32 layout of
// conv_fwd_kernel<*, 2>: [rot][dx][2 halves][32 rows][8], row n = (jrow*3 + s)*2
// + co for n < 18, zero rows above.
__global__ void pack_out2_kernel(const float* __restrict__ w, __nv_bfloat16* __restrict__ wf2) {
  constexpr int NB = OutShape<2>::NB;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= W_TILES * 2 * NB * 8) return;
  const int c = i % 8, n = (i / 8) % NB, h = (i / (8 * NB)) % 2, tile = i / (16 * NB);
  const int rot = tile / 3, dx = tile % 3;
  float v = 0.0f;
  if (n < 18) {
    const int co = n % 2, sj = n / 2, s = sj % 3, jrow = sj / 3;
    const int dz = 2 - (((s - rot + 1) % 3 + 3) % 3);
    const int tap = dz * 9 + (2 - jrow) * 3 + dx;
    v = w[(size_t)(NLAYER - 1) * NTAP * 256 + (size_t)tap * 256 + co * 16 + 8 * h + c];
  }
  wf2[i] = __float2bfloat16_rn(v);
}

// 2:1 restriction (2x2x2 average) of a solver field (2 ghosts) to a dense
// complex array of TO on the coarse grid.
template <typename TS, typename TO>
__global__ void restrict_kernel(const TS* __restrict__ f, int Nx, int Ny, int nxc, int nyc,
                                int nzc, TO* __restrict__ out) {
  const size_t n = (size_t)nxc * nyc * nzc;
  for (size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x; s < n;
       s += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(s % nxc);
    const size_t t = s / nxc;
    const int y = (int)(t % nyc), z = (int)(t / nyc);
    double re = 0.0, im = 0.0;
    for (int c = 0; c < 2; c++)
      for (int b = 0; b < 2; b++)
        for (int a = 0; a < 2; a++) {
          const size_t q = ((size_t)(2 * z + c + 2) * Ny + (2 * y + b + 2)) * Nx + (2 * x + a + 2);
          re += (double)f[2 * q];
          im += (double)f[2 * q + 1];
        }
    out[2 * s] = (TO)(0.125 * re);
    out[2 * s + 1] = (TO)(0.125 * im);
  }
}

}  // namespace cnn
}  // namespace gpe
