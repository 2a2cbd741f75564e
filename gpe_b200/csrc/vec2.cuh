// vec2.cuh -- two-lane vector arithmetic on one complex value (re, im).
//
// For float the lanes map onto sm_100's packed FP32x2 instructions
// (__fadd2_rn / __fmul2_rn / __ffma2_rn), so a complex add, a real-by-complex
// multiply or a real-weighted accumulate is one instruction; each lane rounds
// exactly like the scalar __fadd_rn / __fmul_rn / __fmaf_rn.  For double the
// same helpers fall back to scalar FP64 operations.
#pragma once

#include <cuda_runtime.h>

namespace gpe {

template <typename TC>
struct VT;
template <>
struct VT<float> {
  using T = float2;
};
template <>
struct VT<double> {
  using T = double2;
};

__device__ __forceinline__ float2 vadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 vmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 vfma(float2 a, float2 b, float2 c) {
  return __ffma2_rn(a, b, c);
}
__device__ __forceinline__ float2 vsplat(float s) { return make_float2(s, s); }
__device__ __forceinline__ float2 vpair(float a, float b) { return make_float2(a, b); }

__device__ __forceinline__ double2 vadd(double2 a, double2 b) {
  return make_double2(a.x + b.x, a.y + b.y);
}
__device__ __forceinline__ double2 vmul(double2 a, double2 b) {
  return make_double2(a.x * b.x, a.y * b.y);
}
__device__ __forceinline__ double2 vfma(double2 a, double2 b, double2 c) {
  return make_double2(fma(a.x, b.x, c.x), fma(a.y, b.y, c.y));
}
__device__ __forceinline__ double2 vsplat(double s) { return make_double2(s, s); }
__device__ __forceinline__ double2 vpair(double a, double b) { return make_double2(a, b); }

// (im, re): with a coefficient pair (-c, c) this forms c * i * v.
template <typename V>
__device__ __forceinline__ V vswap(V a) {
  V r;
  r.x = a.y;
  r.y = a.x;
  return r;
}

// Two consecutive complex values along x, loaded / stored as one 16-byte
// (float) or two 16-byte (double) accesses.
template <typename TC>
struct CPair {
  typename VT<TC>::T a, b;  // site x, site x+1
};

template <typename TS, typename TC>
__device__ __forceinline__ CPair<TC> ld_cpair(const TS* p);

template <>
__device__ __forceinline__ CPair<float> ld_cpair<float, float>(const float* p) {
  const float4 v = *reinterpret_cast<const float4*>(p);
  return {make_float2(v.x, v.y), make_float2(v.z, v.w)};
}
template <>
__device__ __forceinline__ CPair<double> ld_cpair<double, double>(const double* p) {
  const double2 a = reinterpret_cast<const double2*>(p)[0];
  const double2 b = reinterpret_cast<const double2*>(p)[1];
  return {a, b};
}
template <>
__device__ __forceinline__ CPair<double> ld_cpair<float, double>(const float* p) {
  const float4 v = *reinterpret_cast<const float4*>(p);
  return {make_double2(v.x, v.y), make_double2(v.z, v.w)};
}

template <typename TS, typename V>
__device__ __forceinline__ void st_cpair(TS* p, V a, V b);
template <>
__device__ __forceinline__ void st_cpair<float, float2>(float* p, float2 a, float2 b) {
  *reinterpret_cast<float4*>(p) = make_float4(a.x, a.y, b.x, b.y);
}
template <>
__device__ __forceinline__ void st_cpair<double, double2>(double* p, double2 a, double2 b) {
  reinterpret_cast<double2*>(p)[0] = a;
  reinterpret_cast<double2*>(p)[1] = b;
}

template <typename TS, typename V>
__device__ __forceinline__ typename VT<TS>::T cvt_v(V a) {
  typename VT<TS>::T r;
  r.x = (TS)a.x;
  r.y = (TS)a.y;
  return r;
}

template <typename TS, typename V>
__device__ __forceinline__ void st_c1(TS* p, V a) {
  p[0] = (TS)a.x;
  p[1] = (TS)a.y;
}

}  // namespace gpe
