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
// Forward / dgrad kernel: one CTA per (y-slab of 8 rows, z-chunk) item;
// warp 0 streams input planes (8 + 2 rows, both halves, the full padded x
// extent) into a 4-slot ring with TMA; warp 1 issues, per output row,
// 27 tcgen05.mma (M = 128 sites, N = 16, K = 16) into a TMEM accumulator
// (two buffers of 8 rows x 16 columns); warps 2-9 read the accumulators back
// (tcgen05.ld 32x32b), apply the epilogue and store.
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
constexpr int TYF = 8;
constexpr int FSLOTS = 4;
constexpr int F_EPI_WARPS = 8;
constexpr int F_THREADS = 32 * (2 + F_EPI_WARPS);
constexpr uint32_t F_TMEM_COLS = 256;

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
  CUtensorMap tmap;                 // input activations, box (8, Xp, Hin, TYF+2, 1)
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
  CUtensorMap tmap_x;               // box (8, Xp, 2, XROWS, 1)
  CUtensorMap tmap_dy;              // box (8, Xp, 2, TYW, 1)
  int nx, ny, nz, Xp, Yp, Zp;
  int nslab, nzc, zchunk, nitems;
  uint32_t xslot_bytes, xbox_bytes, dslot_bytes, dbox_bytes;
  float* partials;                  // [gridDim.x][NACC][128][16]
  int* status;
  unsigned long long wait_limit_ns;
};

// GELU from its definition x * Phi(x), Phi the standard normal CDF.
__device__ __forceinline__ float gelu(float x) {
  return 0.5f * x * (1.0f + erff(x * 0.7071067811865476f));
}
__device__ __forceinline__ float gelu_grad(float x) {
  return 0.5f * (1.0f + erff(x * 0.7071067811865476f)) +
         x * 0.3989422804014327f * expf(-0.5f * x * x);
}

__device__ __forceinline__ size_t act_index(int Xp, int Yp, int x, int y, int z, int h) {
  return ((((size_t)z * Yp + y) * 2 + h) * Xp + x) * 8;
}

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
  const __nv_bfloat162 v = __floats2bfloat162_rn(a, b);
  return *reinterpret_cast<const uint32_t*>(&v);
}

// The interior site (x, y, z) and its periodic ghost images (halo 1).
template <typename F>
__device__ __forceinline__ void for_images(int x, int y, int z, int nx, int ny, int nz, F f) {
  int xs[3], ys[3], zs[3];
  int nxs = 0, nys = 0, nzs = 0;
  xs[nxs++] = x + 1;
  if (x == 0) xs[nxs++] = nx + 1;
  if (x == nx - 1) xs[nxs++] = 0;
  ys[nys++] = y + 1;
  if (y == 0) ys[nys++] = ny + 1;
  if (y == ny - 1) ys[nys++] = 0;
  zs[nzs++] = z + 1;
  if (z == 0) zs[nzs++] = nz + 1;
  if (z == nz - 1) zs[nzs++] = 0;
  for (int c = 0; c < nzs; c++)
    for (int b = 0; b < nys; b++)
      for (int a = 0; a < nxs; a++) f(xs[a], ys[b], zs[c]);
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

template <int EPI>
__device__ __forceinline__ void conv_epilogue(const ConvParams& p, const float (&acc)[16], int x,
                                              int y, int z) {
  if (EPI == EPI_GELU || EPI == EPI_GELU_PRE) {
    float pre[16], a[16];
#pragma unroll
    for (int c = 0; c < 16; c++) {
      pre[c] = acc[c] + p.bias[c];
      a[c] = gelu(pre[c]);
    }
    if (EPI == EPI_GELU_PRE) store_act16(p.pre_out, p.Xp, p.Yp, p.nx, p.ny, p.nz, x, y, z, pre, false);
    store_act16(p.act_out, p.Xp, p.Yp, p.nx, p.ny, p.nz, x, y, z, a, true);
  } else if (EPI == EPI_DGELU) {
    float pre[16], g[16];
    load_act16(p.pre_in, p.Xp, p.Yp, x, y, z, pre);
#pragma unroll
    for (int c = 0; c < 16; c++) g[c] = acc[c] * gelu_grad(pre[c]);
    store_act16(p.act_out, p.Xp, p.Yp, p.nx, p.ny, p.nz, x, y, z, g, true);
  } else if (EPI == EPI_DELTA) {
    const size_t s = ((size_t)z * p.ny + y) * p.nx + x;
    reinterpret_cast<float2*>(p.delta)[s] =
        make_float2((acc[0] + p.bias[0]) * p.out_scale, (acc[1] + p.bias[1]) * p.out_scale);
  } else {  // EPI_RESID: psi += delta on the solver's field, ghosts (2, periodic) too
    const float dr = (acc[0] + p.bias[0]) * p.out_scale;
    const float di = (acc[1] + p.bias[1]) * p.out_scale;
    float2* f = reinterpret_cast<float2*>(p.psi);
    const size_t s = ((size_t)(z + 2) * p.psi_Ny + (y + 2)) * p.psi_Nx + (x + 2);
    float2 v = f[s];
    v.x += dr;
    v.y += di;
    int gx[3] = {x, NO_GHOST, NO_GHOST}, gy[3] = {y, NO_GHOST, NO_GHOST},
        gz[3] = {z, NO_GHOST, NO_GHOST};
    ghost_targets(x, p.nx, 1, gx[1], gx[2]);
    ghost_targets(y, p.ny, 1, gy[1], gy[2]);
    ghost_targets(z, p.nz, 1, gz[1], gz[2]);
    for (int c = 0; c < 3; c++) {
      if (gz[c] == NO_GHOST) continue;
      for (int b = 0; b < 3; b++) {
        if (gy[b] == NO_GHOST) continue;
        for (int a = 0; a < 3; a++) {
          if (gx[a] == NO_GHOST) continue;
          f[((size_t)(gz[c] + 2) * p.psi_Ny + (gy[b] + 2)) * p.psi_Nx + (gx[a] + 2)] = v;
        }
      }
    }
  }
}

template <int EPI>
__global__ void __launch_bounds__(F_THREADS, 1) conv_fwd_kernel(const __grid_constant__ ConvParams p) {
  extern __shared__ unsigned char smem_raw[];
  unsigned char* ring = reinterpret_cast<unsigned char*>(
      (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  unsigned char* wsm = ring + FSLOTS * p.slot_bytes + 4096;  // 4 KB of zeros after the ring
  uint64_t* full = reinterpret_cast<uint64_t*>(wsm + NTAP * TAP_BYTES);
  uint64_t* empty = full + FSLOTS;
  uint64_t* accf = empty + FSLOTS;
  uint64_t* acce = accf + 2;
  uint64_t* drain = acce + 2;
  uint32_t* tmem_holder = reinterpret_cast<uint32_t*>(drain + 1);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(tmem_holder + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  {  // weights and the zero pad (generic proxy), then make them visible to the tensor core
    const uint4* src = reinterpret_cast<const uint4*>(p.w);
    uint4* dst = reinterpret_cast<uint4*>(wsm);
    for (int i = threadIdx.x; i < NTAP * TAP_BYTES / 16; i += blockDim.x) dst[i] = src[i];
    uint4* pad = reinterpret_cast<uint4*>(ring + FSLOTS * p.slot_bytes);
    for (int i = threadIdx.x; i < 4096 / 16; i += blockDim.x) pad[i] = make_uint4(0, 0, 0, 0);
    for (int s = 0; s < FSLOTS; s++) {
      uint4* gap = reinterpret_cast<uint4*>(ring + s * p.slot_bytes + p.box_bytes);
      for (int i = threadIdx.x; i < (int)(p.slot_bytes - p.box_bytes) / 16; i += blockDim.x)
        gap[i] = make_uint4(0, 0, 0, 0);
    }
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < FSLOTS; s++) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; b++) {
      mbar_init(&accf[b], 1);
      mbar_init(&acce[b], 32 * F_EPI_WARPS);
    }
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

  if (warp == 0) {
    if (lane == 0) {
      prefetch_tmap(&p.tmap);
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
          mbar_arrive_expect_tx(&full[slot], p.box_bytes);
          tc::tma_load_5d(smem_u32(ring + slot * p.slot_bytes), &p.tmap, 0, 0, 0, y0, z0 + pl,
                          smem_u32(&full[slot]));
        }
      }
      // every load issued must have landed before the CTA exits
      const uint32_t first = g > FSLOTS ? g - FSLOTS : 0;
      for (uint32_t q = first; q < g; q++)
        if (!mbar_wait_bounded(&full[q % FSLOTS], (q / FSLOTS) & 1, lim)) {
          set_abort(p.status, abort_flag, 1);
          break;
        }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      const uint32_t idesc = tc::idesc_bf16_f32(128, 16, false, false);
      const uint32_t lbo_a = p.Hin == 2 ? row_bytes : 0;
      const uint32_t ring_s = smem_u32(ring), w_s = smem_u32(wsm);
      const uint64_t bdesc0 = tc::smem_desc(w_s, 256, 128);
      uint32_t g0 = 0, waited = 0, accn = 0;
      for (int it = blockIdx.x; it < p.nitems && !*abort_flag; it += gridDim.x) {
        const int slab = it % p.nslab, zc = it / p.nslab;
        const int y0 = slab * TYF, z0 = zc * p.zchunk;
        const int nout = min(z0 + p.zchunk, p.nz) - z0;
        const int nrows = min(TYF, p.ny - y0);
        for (int o = 0; o < nout && !*abort_flag; o++) {
          bool ok = true;
          while (waited < g0 + o + 3) {
            if (!mbar_wait_bounded(&full[waited % FSLOTS], (waited / FSLOTS) & 1, lim)) {
              ok = false;
              break;
            }
            waited++;
          }
          const uint32_t buf = accn & 1;
          if (ok && accn >= 2) ok = mbar_wait_bounded(&acce[buf], ((accn >> 1) - 1) & 1, lim);
          if (!ok) {
            set_abort(p.status, abort_flag, 1);
            break;
          }
          tc::fence_after_sync();
          uint32_t pbase[3];
#pragma unroll
          for (int dz = 0; dz < 3; dz++) pbase[dz] = ring_s + ((g0 + o + dz) % FSLOTS) * p.slot_bytes;
          for (int r = 0; r < nrows; r++) {
            const uint32_t d = tmem + (buf * TYF + r) * 16;
#pragma unroll
            for (int dz = 0; dz < 3; dz++)
#pragma unroll
              for (int dy = 0; dy < 3; dy++) {
                const uint32_t rowa = pbase[dz] + (uint32_t)((r + dy) * p.Hin) * row_bytes;
#pragma unroll
                for (int dx = 0; dx < 3; dx++) {
                  const int tap = dz * 9 + dy * 3 + dx;
                  const uint64_t adesc = tc::smem_desc(rowa + dx * 16, lbo_a, 128);
                  tc::mma_bf16(d, adesc, bdesc0 + (uint64_t)(tap * TAP_BYTES / 16), idesc,
                               tap > 0 ? 1u : 0u);
                }
              }
          }
          tc::commit(smem_u32(&accf[buf]));
          tc::commit(smem_u32(&empty[(g0 + o) % FSLOTS]));
          accn++;
        }
        if (*abort_flag) break;
        tc::commit(smem_u32(&empty[(g0 + nout) % FSLOTS]));
        tc::commit(smem_u32(&empty[(g0 + nout + 1) % FSLOTS]));
        g0 += nout + 2;
      }
      tc::commit(smem_u32(drain));
      if (!mbar_wait_bounded(drain, 0, lim)) set_abort(p.status, abort_flag, 1);
    }
  } else {
    const int ew = warp - 2;
    const int q = warp & 3, half = ew >> 2;
    const int x = 32 * q + lane;
    uint32_t accn = 0;
    for (int it = blockIdx.x; it < p.nitems && !*abort_flag; it += gridDim.x) {
      const int slab = it % p.nslab, zc = it / p.nslab;
      const int y0 = slab * TYF, z0 = zc * p.zchunk;
      const int nout = min(z0 + p.zchunk, p.nz) - z0;
      const int nrows = min(TYF, p.ny - y0);
      for (int o = 0; o < nout; o++) {
        const uint32_t buf = accn & 1;
        if (!mbar_wait_bounded(&accf[buf], (accn >> 1) & 1, lim)) {
          set_abort(p.status, abort_flag, 1);
          break;
        }
        tc::fence_after_sync();
        for (int r = half; r < nrows; r += 2) {
          float v[16];
          tc::ld_32x32b_x16(tmem + ((uint32_t)(32 * q) << 16) + (buf * TYF + r) * 16, v);
          if (x < p.nx) conv_epilogue<EPI>(p, v, x, y0 + r, z0 + o);
        }
        tc::fence_before_sync();
        mbar_arrive(&acce[buf]);
        accn++;
      }
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
      prefetch_tmap(&p.tmap_x);
      prefetch_tmap(&p.tmap_dy);
      uint32_t gx = 0, gd = 0;
      auto load_x = [&](int y0, int zpad) -> bool {
        const uint32_t slot = gx % WSLOTS, cyc = gx / WSLOTS;
        if (cyc > 0 && !mbar_wait_bounded(&xempty[slot], (cyc - 1) & 1, lim)) return false;
        mbar_arrive_expect_tx(&xfull[slot], p.xbox_bytes);
        tc::tma_load_5d(smem_u32(xring + slot * p.xslot_bytes), &p.tmap_x, 0, 0, 0, y0, zpad,
                        smem_u32(&xfull[slot]));
        gx++;
        return true;
      };
      auto load_d = [&](int y0, int zpad) -> bool {
        const uint32_t slot = gd % DSLOTS, cyc = gd / DSLOTS;
        if (cyc > 0 && !mbar_wait_bounded(&dempty[slot], (cyc - 1) & 1, lim)) return false;
        mbar_arrive_expect_tx(&dfull[slot], p.dbox_bytes);
        tc::tma_load_5d(smem_u32(dring + slot * p.dslot_bytes), &p.tmap_dy, 0, 0, 0, y0 + 1, zpad,
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
// (channels Re, Im, 0, ...; H halves), ghosts included.
template <typename TS>
__global__ void pack_input_kernel(const TS* __restrict__ psi, int Nx, int Ny, int nx, int ny,
                                  int nz, __nv_bfloat16* __restrict__ act, int H) {
  const int Xp = nx + 2, Yp = ny + 2;
  const size_t n = (size_t)nx * ny * nz;
  for (size_t s = (size_t)blockIdx.x * blockDim.x + threadIdx.x; s < n;
       s += (size_t)gridDim.x * blockDim.x) {
    const int x = (int)(s % nx);
    const size_t t = s / nx;
    const int y = (int)(t % ny), z = (int)(t / ny);
    const size_t q = ((size_t)(z + 2) * Ny + (y + 2)) * Nx + (x + 2);
    uint4 lo = make_uint4(pack_bf16x2((float)psi[2 * q], (float)psi[2 * q + 1]), 0, 0, 0);
    const uint4 zero = make_uint4(0, 0, 0, 0);
    for_images(x, y, z, nx, ny, nz, [&](int xp, int yp, int zp) {
      const size_t b = (((size_t)zp * Yp + yp) * H * Xp) * 8;
      *reinterpret_cast<uint4*>(act + b + (size_t)xp * 8) = lo;
      if (H == 2) *reinterpret_cast<uint4*>(act + b + ((size_t)Xp + xp) * 8) = zero;
    });
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

// fp32 weights [L][27][16 co][16 ci] -> bf16 forward tiles [L][27][2][16][8]
// (K = ci halves) and dgrad tiles (taps mirrored, co <-> ci).
__global__ void pack_weights_kernel(const float* __restrict__ w, __nv_bfloat16* __restrict__ wf,
                                    __nv_bfloat16* __restrict__ wt) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= NLAYER * NTAP * 16 * 16) return;
  const int c = i % 8, n = (i / 8) % 16, h = (i / 128) % 2, tap = (i / 256) % NTAP,
            l = i / (256 * NTAP);
  const size_t base = (size_t)l * NTAP * 256;
  wf[i] = __float2bfloat16_rn(w[base + (size_t)tap * 256 + n * 16 + (8 * h + c)]);
  wt[i] = __float2bfloat16_rn(w[base + (size_t)(NTAP - 1 - tap) * 256 + (8 * h + c) * 16 + n]);
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
