// device_utils.cuh -- PTX wrappers (mbarrier, TMA tile loads), complex pair
// loads/stores and block reductions used by the GPE stage kernels.
//
// TMA: plain tile loads only (cp.async.bulk.tensor ... .tile), never the
// cluster-multicast form; every load's source is this GPU's own memory.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace gpe {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)),
               "r"(count)
               : "memory");
}

// Make barrier initialisation visible to the async (TMA) proxy.
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Order earlier generic-proxy shared-memory accesses before later TMA writes
// into the same buffer.
__device__ __forceinline__ void fence_proxy_async() {
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar,
                                                      uint32_t bytes) {
  asm volatile(
      "mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(
          smem_u32(bar)),
      "r"(bytes)
      : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// Barrier among the first `nthreads` threads (a multiple of 32) of the CTA.
__device__ __forceinline__ void named_barrier_sync(int id, int nthreads) {
  asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

__device__ __forceinline__ uint64_t global_timer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Wait for phase `parity` of an mbarrier, giving up after limit_ns.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar,
                                                  uint32_t parity,
                                                  uint64_t limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_timer_ns();
  while (true) {
    if (mbar_try_wait(bar, parity)) return true;
    if (global_timer_ns() - t0 > limit_ns) return false;
  }
}

// 3-D tiled TMA load global -> shared, completion counted on `bar`.
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map,
                                            uint64_t* bar, int c0, int c1,
                                            int c2) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::"
      "complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2),
      "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void prefetch_tmap(const CUtensorMap* map) {
  asm volatile("prefetch.tensormap [%0];" ::"l"(
                   reinterpret_cast<uint64_t>(map))
               : "memory");
}

// ---------------------------------------------------------------------------
// Two consecutive complex values along x (re0, im0, re1, im1).

template <typename T>
struct Pair {
  T r0, i0, r1, i1;
};

template <typename T>
__device__ __forceinline__ Pair<T> ld_pair(const T* p);
template <>
__device__ __forceinline__ Pair<float> ld_pair<float>(const float* p) {
  const float4 v = *reinterpret_cast<const float4*>(p);
  return {v.x, v.y, v.z, v.w};
}
template <>
__device__ __forceinline__ Pair<double> ld_pair<double>(const double* p) {
  const double2 a = reinterpret_cast<const double2*>(p)[0];
  const double2 b = reinterpret_cast<const double2*>(p)[1];
  return {a.x, a.y, b.x, b.y};
}

template <typename T>
__device__ __forceinline__ void st_pair(T* p, const Pair<T>& v);
template <>
__device__ __forceinline__ void st_pair<float>(float* p, const Pair<float>& v) {
  *reinterpret_cast<float4*>(p) = make_float4(v.r0, v.i0, v.r1, v.i1);
}
template <>
__device__ __forceinline__ void st_pair<double>(double* p,
                                                const Pair<double>& v) {
  reinterpret_cast<double2*>(p)[0] = make_double2(v.r0, v.i0);
  reinterpret_cast<double2*>(p)[1] = make_double2(v.r1, v.i1);
}

template <typename T>
__device__ __forceinline__ void st_one(T* p, T re, T im) {
  p[0] = re;
  p[1] = im;
}
template <>
__device__ __forceinline__ void st_one<float>(float* p, float re, float im) {
  *reinterpret_cast<float2*>(p) = make_float2(re, im);
}
template <>
__device__ __forceinline__ void st_one<double>(double* p, double re,
                                               double im) {
  *reinterpret_cast<double2*>(p) = make_double2(re, im);
}

template <typename TO, typename TI>
__device__ __forceinline__ Pair<TO> cvt_pair(const Pair<TI>& a) {
  return {static_cast<TO>(a.r0), static_cast<TO>(a.i0),
          static_cast<TO>(a.r1), static_cast<TO>(a.i1)};
}

// ---------------------------------------------------------------------------
// Block reductions in FP64 (fixed order => deterministic).

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1)
    v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Ghost targets of interior index i along an axis of n points: the ghost
// positions (-2, -1, n, n+1) whose value is a copy of point i.  Periodic
// (bcs 1): ghost g holds f(g mod n).  Reflective (bcs 2): mirror about the
// end nodes, f(-1)=f(1), f(-2)=f(2), f(n)=f(n-2), f(n+1)=f(n-3).
constexpr int NO_GHOST = -1000000;
__device__ __forceinline__ void ghost_targets(int i, int n, int bcs, int& g0,
                                              int& g1) {
  g0 = NO_GHOST;
  g1 = NO_GHOST;
  int s0, s1, s2, s3;
  if (bcs == 1) {
    s0 = n - 2; s1 = n - 1; s2 = 0; s3 = 1;
  } else {
    s0 = 2; s1 = 1; s2 = n - 2; s3 = n - 3;
  }
  if (s0 == i) { g0 = -2; }
  if (s1 == i) { if (g0 == NO_GHOST) g0 = -1; else g1 = -1; }
  if (s2 == i) { if (g0 == NO_GHOST) g0 = n; else g1 = n; }
  if (s3 == i) { if (g0 == NO_GHOST) g0 = n + 1; else g1 = n + 1; }
}

}  // namespace gpe
