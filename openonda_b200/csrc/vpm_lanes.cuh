// vpm_lanes.cuh -- arithmetic on a "lane" value: one FP64 target (double) or two FP32
// targets packed in a float2 and processed by the sm_100 paired FP32 instructions
// (FFMA2 / FADD2 / FMUL2 via __ffma2_rn, __fadd2_rn, __fmul2_rn).  The pair operators are
// written once against these helpers.
#pragma once

#include <cuda_runtime.h>

#include "vpm_common.cuh"

namespace vpm {

template <class V>
struct LaneTraits;
template <>
struct LaneTraits<double> {
  using Scalar = double;
  static constexpr int kLanes = 1;
};
template <>
struct LaneTraits<float2> {
  using Scalar = float;
  static constexpr int kLanes = 2;
};

// ---- constants ----------------------------------------------------------------------------
template <class V>
__device__ __forceinline__ V splat(double c);
template <>
__device__ __forceinline__ double splat<double>(double c) {
  return c;
}
template <>
__device__ __forceinline__ float2 splat<float2>(double c) {
  return make_float2(float(c), float(c));
}

// ---- packed FP32 arithmetic -------------------------------------------------------------
__device__ __forceinline__ float2 operator+(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 operator-(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 operator-(float2 a, float2 b) { return __fadd2_rn(a, -b); }
__device__ __forceinline__ float2 operator*(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
using ::fma;  // keep the scalar overloads visible next to the packed one

// ---- reciprocal square root ---------------------------------------------------------------
// FP32: the hardware approximation (PTX rsqrt.approx.ftz.f32; the argument x = r^2 + s^2 is
// never below the smallest squared core, so flushing denormals changes nothing), optionally
// refined by one Newton-Raphson step y <- y + y (1/2 - x y^2 / 2).  FP64: CUDA's rsqrt().
__device__ __forceinline__ float rsqrt_approx(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// 1/x for the lane: hardware approximation in FP32 (second MUFU op), exact division in FP64.
__device__ __forceinline__ float2 rcp_lane(float2 x) {
  return make_float2(rcp_approx(x.x), rcp_approx(x.y));
}
__device__ __forceinline__ double rcp_lane(double x) { return 1.0 / x; }

template <bool REFINE>
__device__ __forceinline__ float rsqrt_lane(float x) {
  float y = rsqrt_approx(x);
  if constexpr (REFINE) {
    const float hx = 0.5f * x;
    const float e = fmaf(-(hx * y), y, 0.5f);
    y = fmaf(y, e, y);
  }
  return y;
}
template <bool REFINE>
__device__ __forceinline__ float2 rsqrt_lane(float2 x) {
  if constexpr (REFINE) {
    const float2 y = make_float2(rsqrt_approx(x.x), rsqrt_approx(x.y));
    const float2 hx = __fmul2_rn(x, make_float2(0.5f, 0.5f));
    const float2 e = __ffma2_rn(-__fmul2_rn(hx, y), y, make_float2(0.5f, 0.5f));
    return __ffma2_rn(y, e, y);
  } else {
    return make_float2(rsqrt_approx(x.x), rsqrt_approx(x.y));
  }
}
template <bool REFINE>
__device__ __forceinline__ double rsqrt_lane(double x) {
  return rsqrt(x);
}

// ---- per-lane selections --------------------------------------------------------------------
// acc + v * w where a > thr, acc unchanged elsewhere: a skipped pair adds nothing even when
// its terms are not finite, as with the reference's branch (ParticlesPhysicsCuda.py:80, 332).
__device__ __forceinline__ double fma_if_gt(double a, double thr, double v, double w,
                                            double acc) {
  return a > thr ? fma(v, w, acc) : acc;
}
__device__ __forceinline__ float2 fma_if_gt(float2 a, double thr, float2 v, float2 w,
                                            float2 acc) {
  const float t = float(thr);
  const float2 r = fma(v, w, acc);
  return make_float2(a.x > t ? r.x : acc.x, a.y > t ? r.y : acc.y);
}
// v except in the lanes whose target index equals j
__device__ __forceinline__ double zero_if_self(double v, const int64_t* i, int64_t j) {
  return i[0] == j ? 0.0 : v;
}
__device__ __forceinline__ float2 zero_if_self(float2 v, const int64_t* i, int64_t j) {
  return make_float2(i[0] == j ? 0.f : v.x, i[1] == j ? 0.f : v.y);
}

// ---- lane <-> FP64 --------------------------------------------------------------------------
__device__ __forceinline__ double lane_get(double v, int) { return v; }
__device__ __forceinline__ double lane_get(float2 v, int k) { return double(k ? v.y : v.x); }
__device__ __forceinline__ void lane_zero(double& v) { v = 0.0; }
__device__ __forceinline__ void lane_zero(float2& v) { v = make_float2(0.f, 0.f); }

// Scalar value of a stored record element ({v, v} pairs hold the same value twice).
__host__ __device__ __forceinline__ double elem(double v) { return v; }
__host__ __device__ __forceinline__ double elem(float2 v) { return double(v.x); }

}  // namespace vpm
