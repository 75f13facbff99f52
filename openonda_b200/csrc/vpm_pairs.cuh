// vpm_pairs.cuh -- per-pair operators of the VPM all-pairs sums.
//
// Each operator adds one source particle's contribution to the partial sums of one "lane"
// of targets: one FP64 target (V = double) or two FP32 targets (V = float2, paired FP32
// instructions).  All kernels of the reference are written in the sigma-symmetric rsqrt
// form
//     x = r^2 + s^2,  y = x^(-1/2)
// where s is the pair core (sigma_i + sigma_j)/2 for self sums and sigma_j for probes:
//
//   q(rho)/sigma^3 = (rho^2 + 2.5)/((rho^2 + 1)^2.5 sigma^3) = (x + 1.5 s^2) y^5
//   stretching f2  = 3 (rho^2 + 3.5)/(sigma^5 (rho^2 + 1)^3.5) = 3 (x + 2.5 s^2) y^7
//   PSE kernel     = 105 nu sigma^3/(sigma^5 (rho^2 + 1)^4.5)  = 105 nu s^7 y^9
//   zeta kernel    = 7.5/((rho^2 + 1)^3.5 sigma^3)             = 7.5 s^4 y^7
//   enstrophy      = (r^2 + 3.2 s^2)/(r^2 + s^2)^1.5            = (x + 2.2 s^2) y^3
//   kinetic energy = [2 rho/sqrt(rho^2+1) P1 + rho^3/(rho^2+1)^1.5 ((r^.a_i)(r^.a_j) - P1)]/|r|
//                  = P1 (y + s^2 y^3) + y^3 (r.a_i)(r.a_j),  P1 = a_i.a_j
//
// Target-only factors (1/4pi, 105 nu_i, 7.5, 3, the sign, a_i x ...) are applied once per
// target in the finalize pass.  The stretching term a_i x a_j is summed as
//   sum_j g (a_i x a_j) = a_i x sum_j g (a_j - a_i),
// which is exact in exact arithmetic, vanishes identically for j == i and keeps the
// partial sum small when neighbouring strengths are nearly parallel.  In the stretching-only
// operator the triple product a_i . (r x a_j) is evaluated as r . (d x a_i) with
// d = a_j - a_i (equal since a_i . (r x a_i) = 0; same cost there); the fused operator
// reuses the velocity's r x a_j instead, which measured equally accurate and is cheaper.
//
// References (OpenONDA/solvers/VPM/ParticlesPhysicsCuda.py):
//   OpVel      get_selfinduced_velocity_kernel      :133-191
//   OpVelAt    get_induced_velocity_at_kernel       :39-97
//   OpVortAt   get_vorticity_field_at_kernel_simplified :291-346
//   OpStretch  get_strength_gradients_kernel        :375-445
//   OpPse      get_strength_gradients_PSE_kernel    :478-530
//   OpKe       get_total_kinetic_energy_kernel      :563-642
//   OpEns      get_total_enstrophy_kernel_simple    :867-920
//   OpLesStep  OpVelStretch + OpVortAt (particles as probes) + OpEns on one state
//   (helicity, :673-750, is  -a_i . sum_j g (r x a_j), i.e. a by-product of OpVel)
#pragma once

#include "vpm_lanes.cuh"

namespace vpm {

// Stretching sums on ring-shaped fields cancel between near neighbours, so their FP32 partials
// are folded into FP64 every 16 sources instead of 32 (error on the 8192-particle ring
// 1.95e-6 -> 1.23e-6 relative against FP64).
#ifndef VPM_STRETCH_WINDOW
#define VPM_STRETCH_WINDOW 16
#endif

template <class V>
struct Src {
  V x, y, z, s, ax, ay, az, nu;
};

template <class V>
__device__ __forceinline__ Src<V> load_src(const Rec<V>& r);

template <>
__device__ __forceinline__ Src<float2> load_src<float2>(const Rec<float2>& r) {
  const float4* p = reinterpret_cast<const float4*>(&r);
  const float4 a = p[0], b = p[1], c = p[2], d = p[3];
  return Src<float2>{make_float2(a.x, a.y), make_float2(a.z, a.w), make_float2(b.x, b.y),
                     make_float2(b.z, b.w), make_float2(c.x, c.y), make_float2(c.z, c.w),
                     make_float2(d.x, d.y), make_float2(d.z, d.w)};
}

template <>
__device__ __forceinline__ Src<double> load_src<double>(const Rec<double>& r) {
  const double2* p = reinterpret_cast<const double2*>(&r);
  const double2 a = p[0], b = p[1], c = p[2], d = p[3];
  return Src<double>{a.x, a.y, b.x, b.y, c.x, c.y, d.x, d.y};
}

// Per-lane target registers shared by all operators.
template <class V>
struct Tgt {
  V x, y, z, hs;   // position, half core
  V ax, ay, az;    // strength
  V sc, s2c, s4c;  // core, core^2, core^4 (the pair core when all cores are equal)
};

// `r` points at the lane's records: one for FP64, two (lane 0, lane 1) for FP32.
__device__ __forceinline__ Tgt<double> make_tgt(const Rec<double>* const* r) {
  const Rec<double>& a = *r[0];
  const double s2 = a.s * a.s;
  return Tgt<double>{a.x, a.y, a.z, 0.5 * a.s, a.ax, a.ay, a.az, a.s, s2, s2 * s2};
}
__device__ __forceinline__ Tgt<float2> make_tgt(const Rec<float2>* const* r) {
  const Rec<float2>& a = *r[0];
  const Rec<float2>& b = *r[1];
  const float2 sc = make_float2(a.s.x, b.s.x);
  const float2 s2 = sc * sc;
  return Tgt<float2>{make_float2(a.x.x, b.x.x),   make_float2(a.y.x, b.y.x),
                     make_float2(a.z.x, b.z.x),   make_float2(0.5f * a.s.x, 0.5f * b.s.x),
                     make_float2(a.ax.x, b.ax.x), make_float2(a.ay.x, b.ay.x),
                     make_float2(a.az.x, b.az.x), sc, s2, s2 * s2};
}

// Pair core s = (sigma_i + sigma_j)/2 and s^2.  UC ("uniform core"): the caller guarantees
// that every particle has the same core, so s = sigma_i exactly (0.5 s + 0.5 s rounds to s)
// and s^2 is a per-target constant: two lane-ops fewer per pair, same values.
template <bool UC, class V>
__device__ __forceinline__ void pair_core(const Tgt<V>& t, const Src<V>& s, V& sg, V& s2) {
  if constexpr (UC) {
    sg = t.sc;
    s2 = t.s2c;
  } else {
    sg = fma(s.s, splat<V>(0.5), t.hs);
    s2 = sg * sg;
  }
}

// Record/lane plumbing shared by the operators on the standard 64-byte record.
template <class V>
struct PairOpBase {
  static constexpr int kR = 0;  // targets per thread: 0 = the precision's default
  // FP32 sources per FP64 carry fold of the one-sided sweep: 0 = the sweep's default (32)
  static constexpr int kWindow = 0;
  using Record = Rec<V>;
  using SrcT = Src<V>;
  using TgtT = Tgt<V>;
  __device__ __forceinline__ static SrcT load(const Record& r) { return load_src<V>(r); }
  __device__ __forceinline__ static TgtT target(const Record* const* r) { return make_tgt(r); }
};

// ---- self-induced velocity: U += g (r x a_j) ------------------------------------------
template <class V, bool REFINE, bool UC = false>
struct OpVel : PairOpBase<V> {
  static constexpr int NV = 3;
  __device__ __forceinline__ static void pair(const Tgt<V>& t, V* acc, const Src<V>& s,
                                              const int64_t*, int64_t) {
    const V rx = t.x - s.x, ry = t.y - s.y, rz = t.z - s.z;
    V sg, s2;
    pair_core<UC>(t, s, sg, s2);
    const V x = fma(rx, rx, fma(ry, ry, fma(rz, rz, s2)));
    const V y = rsqrt_lane<REFINE>(x);
    const V y2 = y * y;
    const V y5 = (y2 * y2) * y;
    const V g = fma(splat<V>(1.5), s2, x) * y5;
    const V cx = fma(ry, s.az, -(rz * s.ay));
    const V cy = fma(rz, s.ax, -(rx * s.az));
    const V cz = fma(rx, s.ay, -(ry * s.ax));
    acc[0] = fma(g, cx, acc[0]);
    acc[1] = fma(g, cy, acc[1]);
    acc[2] = fma(g, cz, acc[2]);
  }
};

// ---- probe velocity: source core sigma_j, pairs with r^2 <= 1e-8 skipped ----------------
template <class V, bool REFINE>
struct OpVelAt : PairOpBase<V> {
  static constexpr int NV = 3;
  __device__ __forceinline__ static void pair(const Tgt<V>& t, V* acc, const Src<V>& s,
                                              const int64_t*, int64_t) {
    const V rx = t.x - s.x, ry = t.y - s.y, rz = t.z - s.z;
    const V r2 = fma(rx, rx, fma(ry, ry, rz * rz));
    const V s2 = s.s * s.s;
    const V y = rsqrt_lane<REFINE>(r2 + s2);
    const V y2 = y * y;
    const V y5 = (y2 * y2) * y;
    const V g = fma(splat<V>(2.5), s2, r2) * y5;
    const V cx = fma(ry, s.az, -(rz * s.ay));
    const V cy = fma(rz, s.ax, -(rx * s.az));
    const V cz = fma(rx, s.ay, -(ry * s.ax));
    acc[0] = fma_if_gt(r2, kRefEps, g, cx, acc[0]);
    acc[1] = fma_if_gt(r2, kRefEps, g, cy, acc[1]);
    acc[2] = fma_if_gt(r2, kRefEps, g, cz, acc[2]);
  }
};

// ---- probe vorticity (zeta kernel only): W += s^4 y^7 a_j, r^2 <= 1e-8 skipped ----------
template <class V, bool REFINE>
struct OpVortAt : PairOpBase<V> {
  static constexpr int NV = 3;
  __device__ __forceinline__ static void pair(const Tgt<V>& t, V* acc, const Src<V>& s,
                                              const int64_t*, int64_t) {
    const V rx = t.x - s.x, ry = t.y - s.y, rz = t.z - s.z;
    const V r2 = fma(rx, rx, fma(ry, ry, rz * rz));
    const V s2 = s.s * s.s;
    const V y = rsqrt_lane<REFINE>(r2 + s2);
    const V y2 = y * y;
    const V y3 = y2 * y;
    const V y7 = (y3 * y3) * y;
    const V k = (s2 * s2) * y7;
    acc[0] = fma_if_gt(r2, kRefEps, k, s.ax, acc[0]);
    acc[1] = fma_if_gt(r2, kRefEps, k, s.ay, acc[1]);
    acc[2] = fma_if_gt(r2, kRefEps, k, s.az, acc[2]);
  }
};

// ---- LES test filter: the vorticity filter sum with two more particle fields -------------
// The least-squares dynamic coefficient needs, at the test-filter width, the vorticity and
// the filtered fields (|u|^2 v, sigma^2 |w|^2 v): one probe-style sweep of the particles over
// themselves with the zeta kernel of the source core (here 2 sigma_j), pairs with
// r^2 <= 1e-8 skipped as in OpVortAt.  Record: position, core, strength and the two fields,
// 80 bytes in both precisions.
template <class E>
struct alignas(16) RecF {
  E x, y, z, s;
  E ax, ay, az, f1;
  E f2, pad;
};
static_assert(sizeof(RecF<double>) == 80 && sizeof(RecF<float2>) == 80, "RecF is 80 B");

template <class V>
struct SrcF {
  V x, y, z, s, ax, ay, az, f1, f2;
};
template <class V>
struct TgtF {
  V x, y, z;
};

__device__ __forceinline__ SrcF<double> load_srcf(const RecF<double>& r) {
  const double2* p = reinterpret_cast<const double2*>(&r);
  const double2 a = p[0], b = p[1], c = p[2], d = p[3], e = p[4];
  return SrcF<double>{a.x, a.y, b.x, b.y, c.x, c.y, d.x, d.y, e.x};
}
__device__ __forceinline__ SrcF<float2> load_srcf(const RecF<float2>& r) {
  const float4* p = reinterpret_cast<const float4*>(&r);
  const float4 a = p[0], b = p[1], c = p[2], d = p[3], e = p[4];
  return SrcF<float2>{make_float2(a.x, a.y), make_float2(a.z, a.w), make_float2(b.x, b.y),
                      make_float2(b.z, b.w), make_float2(c.x, c.y), make_float2(c.z, c.w),
                      make_float2(d.x, d.y), make_float2(d.z, d.w), make_float2(e.x, e.y)};
}
__device__ __forceinline__ TgtF<double> make_tgtf(const RecF<double>* const* r) {
  return TgtF<double>{r[0]->x, r[0]->y, r[0]->z};
}
__device__ __forceinline__ TgtF<float2> make_tgtf(const RecF<float2>* const* r) {
  return TgtF<float2>{make_float2(r[0]->x.x, r[1]->x.x), make_float2(r[0]->y.x, r[1]->y.x),
                      make_float2(r[0]->z.x, r[1]->z.x)};
}

template <class V, bool REFINE>
struct OpTestFilter {
  static constexpr int NV = 5;
  static constexpr int kR = 0;
  static constexpr int kWindow = 0;
  using Record = RecF<V>;
  using SrcT = SrcF<V>;
  using TgtT = TgtF<V>;
  __device__ __forceinline__ static SrcT load(const Record& r) { return load_srcf(r); }
  __device__ __forceinline__ static TgtT target(const Record* const* r) { return make_tgtf(r); }
  __device__ __forceinline__ static void pair(const TgtT& t, V* acc, const SrcT& s,
                                              const int64_t*, int64_t) {
    const V rx = t.x - s.x, ry = t.y - s.y, rz = t.z - s.z;
    const V r2 = fma(rx, rx, fma(ry, ry, rz * rz));
    const V s2 = s.s * s.s;
    const V y = rsqrt_lane<REFINE>(r2 + s2);
    const V y2 = y * y;
    const V y3 = y2 * y;
    const V y7 = (y3 * y3) * y;
    const V k = (s2 * s2) * y7;
    acc[0] = fma_if_gt(r2, kRefEps, k, s.ax, acc[0]);
    acc[1] = fma_if_gt(r2, kRefEps, k, s.ay, acc[1]);
    acc[2] = fma_if_gt(r2, kRefEps, k, s.az, acc[2]);
    acc[3] = fma_if_gt(r2, kRefEps, k, s.f1, acc[3]);
    acc[4] = fma_if_gt(r2, kRefEps, k, s.f2, acc[4]);
  }
};

// ---- stretching (transpose scheme): A += g (a_j - a_i),  B += f (r . (d x a_i)) r -------
template <class V, bool REFINE, bool UC = false>
struct OpStretch : PairOpBase<V> {
  static constexpr int NV = 6;
  static constexpr int kWindow = VPM_STRETCH_WINDOW;
  __device__ __forceinline__ static void pair(const Tgt<V>& t, V* acc, const Src<V>& s,
                                              const int64_t*, int64_t) {
    const V rx = t.x - s.x, ry = t.y - s.y, rz = t.z - s.z;
    V sg, s2;
    pair_core<UC>(t, s, sg, s2);
    const V x = fma(rx, rx, fma(ry, ry, fma(rz, rz, s2)));
    const V y = rsqrt_lane<REFINE>(x);
    const V y2 = y * y;
    const V y5 = (y2 * y2) * y;
    const V t1 = fma(splat<V>(1.5), s2, x);
    const V g = t1 * y5;
    const V f = (t1 + s2) * (y5 * y2);
    const V dx = s.ax - t.ax, dy = s.ay - t.ay, dz = s.az - t.az;
    acc[0] = fma(g, dx, acc[0]);
    acc[1] = fma(g, dy, acc[1]);
    acc[2] = fma(g, dz, acc[2]);
    const V wx = fma(dy, t.az, -(dz * t.ay));
    const V wy = fma(dz, t.ax, -(dx * t.az));
    const V wz = fma(dx, t.ay, -(dy * t.ax));
    const V h = f * fma(rx, wx, fma(ry, wy, rz * wz));
    acc[3] = fma(h, rx, acc[3]);
    acc[4] = fma(h, ry, acc[4]);
    acc[5] = fma(h, rz, acc[5]);
  }
};

// ---- fused velocity + stretching: U (3), A (3), B (3) ----------------------------------
#ifndef VPM_Y2_RCP
#define VPM_Y2_RCP 0
#endif
template <class V, bool REFINE, bool UC = false>
struct OpVelStretch : PairOpBase<V> {
  static constexpr int NV = 9;
  static constexpr int kWindow = VPM_STRETCH_WINDOW;
  __device__ __forceinline__ static void pair(const Tgt<V>& t, V* acc, const Src<V>& s,
                                              const int64_t*, int64_t) {
    const V rx = t.x - s.x, ry = t.y - s.y, rz = t.z - s.z;
    V sg, s2;
    pair_core<UC>(t, s, sg, s2);
    const V x = fma(rx, rx, fma(ry, ry, fma(rz, rz, s2)));
    const V y = rsqrt_lane<REFINE>(x);
#if VPM_Y2_RCP
    const V y2 = (LaneTraits<V>::kLanes == 2) ? rcp_lane(x) : y * y;
#else
    const V y2 = y * y;
#endif
    const V y5 = (y2 * y2) * y;
    const V t1 = fma(splat<V>(1.5), s2, x);
    const V g = t1 * y5;
    const V f = (t1 + s2) * (y5 * y2);
    const V cx = fma(ry, s.az, -(rz * s.ay));
    const V cy = fma(rz, s.ax, -(rx * s.az));
    const V cz = fma(rx, s.ay, -(ry * s.ax));
    acc[0] = fma(g, cx, acc[0]);
    acc[1] = fma(g, cy, acc[1]);
    acc[2] = fma(g, cz, acc[2]);
    acc[3] = fma(g, s.ax - t.ax, acc[3]);
    acc[4] = fma(g, s.ay - t.ay, acc[4]);
    acc[5] = fma(g, s.az - t.az, acc[5]);
    const V h = f * fma(t.ax, cx, fma(t.ay, cy, t.az * cz));
    acc[6] = fma(h, rx, acc[6]);
    acc[7] = fma(h, ry, acc[7]);
    acc[8] = fma(h, rz, acc[8]);
  }
};

// ---- LES step sweep: velocity + stretching + both dynamic-LES filter sums ------------------
// The LES time step needs, on the same (x, alpha, sigma), the velocity and stretching
// (vpmModule.py:704, :753), the particle vorticity (:640, get_vorticity_field_at with the
// particles as probes: source core sigma_j, r^2 <= 1e-8 skipped) and the enstrophy filter sum
// (:644, pair core, all pairs).  One sweep gives all 15 sums:
//   U, A, B as OpVelStretch;  W += s_j^4 y_j^7 a_j  (y_j = (r^2 + s_j^2)^-1/2);
//   E += (x + 2.2 s^2) y^3 a_j.
// Per pair 56 FP32 lane-ops and 2 MUFU (counts beside the statements): 39 for velocity and
// stretching (one more than OpVelStretch, since r^2 is formed on its own for the vorticity),
// 11 for the vorticity, 6 for the enstrophy, plus the vorticity's r^2 test (compare and
// selects, ALU pipe); three separate sweeps cost 38 + ~20 + ~15.  Uniform cores: 52.  15 sums per target do not fit four targets per thread in registers, so
// this operator runs two (one packed lane).
#ifndef VPM_LES_R
#define VPM_LES_R 2
#endif
template <class V, bool REFINE, bool UC = false>
struct OpLesStep : PairOpBase<V> {
  static constexpr int kR = VPM_LES_R;
  static constexpr int NV = 15;
  static constexpr int kWindow = VPM_STRETCH_WINDOW;
  __device__ __forceinline__ static void pair(const Tgt<V>& t, V* acc, const Src<V>& s,
                                              const int64_t*, int64_t) {
    const V rx = t.x - s.x, ry = t.y - s.y, rz = t.z - s.z;  // 3
    V sg, s2;
    pair_core<UC>(t, s, sg, s2);                               // 2 (0 with UC)
    const V r2 = fma(rx, rx, fma(ry, ry, rz * rz));            // 3
    const V x = r2 + s2;                                       // 1
    const V y = rsqrt_lane<REFINE>(x);
    const V y2 = y * y;                                        // 1
    const V y5 = (y2 * y2) * y;                                // 2
    const V t1 = fma(splat<V>(1.5), s2, x);                    // 1
    const V g = t1 * y5;                                       // 1
    const V f = (t1 + s2) * (y5 * y2);                         // 3
    const V cx = fma(ry, s.az, -(rz * s.ay));                  // 6
    const V cy = fma(rz, s.ax, -(rx * s.az));
    const V cz = fma(rx, s.ay, -(ry * s.ax));
    acc[0] = fma(g, cx, acc[0]);                               // 3
    acc[1] = fma(g, cy, acc[1]);
    acc[2] = fma(g, cz, acc[2]);
    acc[3] = fma(g, s.ax - t.ax, acc[3]);                      // 6
    acc[4] = fma(g, s.ay - t.ay, acc[4]);
    acc[5] = fma(g, s.az - t.az, acc[5]);
    const V h = f * fma(t.ax, cx, fma(t.ay, cy, t.az * cz));   // 4
    acc[6] = fma(h, rx, acc[6]);                               // 3
    acc[7] = fma(h, ry, acc[7]);
    acc[8] = fma(h, rz, acc[8]);
    // vorticity filter sum (source core)
    const V sj2 = UC ? t.s2c : s.s * s.s;                      // 1 (0 with UC)
    const V yv = rsqrt_lane<REFINE>(r2 + sj2);                 // 1
    const V yv2 = yv * yv;                                     // 4
    const V yv3 = yv2 * yv;
    const V yv7 = (yv3 * yv3) * yv;
    const V sj4 = UC ? t.s4c : sj2 * sj2;                      // 1 (0 with UC)
    const V kv = sj4 * yv7;                                    // 1
    acc[9] = fma_if_gt(r2, kRefEps, kv, s.ax, acc[9]);         // 3 (+ compare, selects)
    acc[10] = fma_if_gt(r2, kRefEps, kv, s.ay, acc[10]);
    acc[11] = fma_if_gt(r2, kRefEps, kv, s.az, acc[11]);
    // enstrophy filter sum (pair core)
    const V ke = fma(splat<V>(2.2), s2, x) * (y2 * y);         // 3
    acc[12] = fma(ke, s.ax, acc[12]);                          // 3
    acc[13] = fma(ke, s.ay, acc[13]);
    acc[14] = fma(ke, s.az, acc[14]);
  }
};

// ---- PSE diffusion: P += s^7 y^9 (a_j - a_i)  (nu_i applied in finalize) -----------------
template <class V, bool REFINE, bool UC = false>
struct OpPse : PairOpBase<V> {
  static constexpr int NV = 3;
  __device__ __forceinline__ static void pair(const Tgt<V>& t, V* acc, const Src<V>& s,
                                              const int64_t*, int64_t) {
    const V rx = t.x - s.x, ry = t.y - s.y, rz = t.z - s.z;
    V sg, s2;
    pair_core<UC>(t, s, sg, s2);
    const V x = fma(rx, rx, fma(ry, ry, fma(rz, rz, s2)));
    const V y = rsqrt_lane<REFINE>(x);
    const V z = sg * y;  // <= 1
    const V z2 = z * z;
    const V z4 = z2 * z2;
    const V z7 = (z4 * z2) * z;
    const V k = z7 * (y * y);
    acc[0] = fma(k, s.ax - t.ax, acc[0]);
    acc[1] = fma(k, s.ay - t.ay, acc[1]);
    acc[2] = fma(k, s.az - t.az, acc[2]);
  }
};

// ---- enstrophy filter sum (all pairs incl. i == j): V += (x + 2.2 s^2) y^3 a_j ---------
template <class V, bool REFINE, bool UC = false>
struct OpEns : PairOpBase<V> {
  static constexpr int NV = 3;
  __device__ __forceinline__ static void pair(const Tgt<V>& t, V* acc, const Src<V>& s,
                                              const int64_t*, int64_t) {
    const V rx = t.x - s.x, ry = t.y - s.y, rz = t.z - s.z;
    V sg, s2;
    pair_core<UC>(t, s, sg, s2);
    const V x = fma(rx, rx, fma(ry, ry, fma(rz, rz, s2)));
    const V y = rsqrt_lane<REFINE>(x);
    const V y3 = (y * y) * y;
    const V k = fma(splat<V>(2.2), s2, x) * y3;
    acc[0] = fma(k, s.ax, acc[0]);
    acc[1] = fma(k, s.ay, acc[1]);
    acc[2] = fma(k, s.az, acc[2]);
  }
};

// ---- kinetic energy (j != i): K += (y + s^2 y^3) a_j + y^3 (r . a_j) r ------------------
template <class V, bool REFINE, bool UC = false>
struct OpKe : PairOpBase<V> {
  static constexpr int NV = 3;
  __device__ __forceinline__ static void pair(const Tgt<V>& t, V* acc, const Src<V>& s,
                                              const int64_t* i, int64_t j) {
    const V rx = t.x - s.x, ry = t.y - s.y, rz = t.z - s.z;
    V sg, s2;
    pair_core<UC>(t, s, sg, s2);
    const V x = fma(rx, rx, fma(ry, ry, fma(rz, rz, s2)));
    const V y = rsqrt_lane<REFINE>(x);
    const V y3 = (y * y) * y;
    const V w = zero_if_self(fma(s2, y3, y), i, j);
    const V q = y3 * fma(rx, s.ax, fma(ry, s.ay, rz * s.az));
    acc[0] = fma(q, rx, fma(w, s.ax, acc[0]));
    acc[1] = fma(q, ry, fma(w, s.ay, acc[1]));
    acc[2] = fma(q, rz, fma(w, s.az, acc[2]));
  }
};

}  // namespace vpm
