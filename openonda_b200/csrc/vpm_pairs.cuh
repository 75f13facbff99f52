// vpm_pairs.cuh -- per-pair operators of the VPM all-pairs sums.
//
// Each operator adds one source particle's contribution to one target's partial sums.
// All kernels of the reference are written here in the sigma-symmetric rsqrt form
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
// partial sum small when neighbouring strengths are nearly parallel.
//
// References (OpenONDA/solvers/VPM/ParticlesPhysicsCuda.py):
//   OpVel      get_selfinduced_velocity_kernel      :133-191
//   OpVelAt    get_induced_velocity_at_kernel       :39-97
//   OpVortAt   get_vorticity_field_at_kernel_simplified :291-346
//   OpStretch  get_strength_gradients_kernel        :375-445
//   OpPse      get_strength_gradients_PSE_kernel    :478-530
//   OpKe       get_total_kinetic_energy_kernel      :563-642
//   OpEns      get_total_enstrophy_kernel_simple    :867-920
//   (helicity, :673-750, is  -a_i . sum_j g (r x a_j), i.e. a by-product of OpVel)
#pragma once

#include "vpm_common.cuh"

namespace vpm {

template <class T>
struct Src {
  T x, y, z, s, ax, ay, az, nu;
};

template <class T>
__device__ __forceinline__ Src<T> load_src(const Rec<T>& r);

template <>
__device__ __forceinline__ Src<float> load_src<float>(const Rec<float>& r) {
  const float4* p = reinterpret_cast<const float4*>(&r);
  const float4 a = p[0], b = p[1];
  return Src<float>{a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
}

template <>
__device__ __forceinline__ Src<double> load_src<double>(const Rec<double>& r) {
  const double2* p = reinterpret_cast<const double2*>(&r);
  const double2 a = p[0], b = p[1], c = p[2], d = p[3];
  return Src<double>{a.x, a.y, b.x, b.y, c.x, c.y, d.x, d.y};
}

// Per-target registers shared by all operators.
template <class T>
struct Tgt {
  T x, y, z, hs;   // position, half core
  T ax, ay, az;    // strength
};

template <class T>
__device__ __forceinline__ Tgt<T> make_tgt(const Rec<T>& r) {
  return Tgt<T>{r.x, r.y, r.z, T(0.5) * r.s, r.ax, r.ay, r.az};
}

// ---- self-induced velocity: U += g (r x a_j) ------------------------------------------
template <class T, bool REFINE>
struct OpVel {
  static constexpr int NV = 3;
  static constexpr bool EXCLUDE_SELF = false;
  __device__ __forceinline__ static void pair(const Tgt<T>& t, T* acc, const Src<T>& s,
                                              int64_t, int64_t) {
    const T rx = t.x - s.x, ry = t.y - s.y, rz = t.z - s.z;
    const T sg = fma(s.s, T(0.5), t.hs);
    const T s2 = sg * sg;
    const T x = fma(rx, rx, fma(ry, ry, fma(rz, rz, s2)));
    const T y = rsqrt_t<REFINE>(x);
    const T y2 = y * y;
    const T y5 = (y2 * y2) * y;
    const T g = fma(T(1.5), s2, x) * y5;
    const T cx = fma(ry, s.az, -(rz * s.ay));
    const T cy = fma(rz, s.ax, -(rx * s.az));
    const T cz = fma(rx, s.ay, -(ry * s.ax));
    acc[0] = fma(g, cx, acc[0]);
    acc[1] = fma(g, cy, acc[1]);
    acc[2] = fma(g, cz, acc[2]);
  }
};

// ---- probe velocity: source core sigma_j, pairs with r^2 <= 1e-8 skipped ----------------
template <class T, bool REFINE>
struct OpVelAt {
  static constexpr int NV = 3;
  static constexpr bool EXCLUDE_SELF = false;
  __device__ __forceinline__ static void pair(const Tgt<T>& t, T* acc, const Src<T>& s,
                                              int64_t, int64_t) {
    const T rx = t.x - s.x, ry = t.y - s.y, rz = t.z - s.z;
    const T r2 = fma(rx, rx, fma(ry, ry, rz * rz));
    const T s2 = s.s * s.s;
    const T y = rsqrt_t<REFINE>(r2 + s2);
    const T y2 = y * y;
    const T y5 = (y2 * y2) * y;
    T g = fma(T(2.5), s2, r2) * y5;
    g = (r2 > T(kRefEps)) ? g : T(0);
    const T cx = fma(ry, s.az, -(rz * s.ay));
    const T cy = fma(rz, s.ax, -(rx * s.az));
    const T cz = fma(rx, s.ay, -(ry * s.ax));
    acc[0] = fma(g, cx, acc[0]);
    acc[1] = fma(g, cy, acc[1]);
    acc[2] = fma(g, cz, acc[2]);
  }
};

// ---- probe vorticity (zeta kernel only): W += s^4 y^7 a_j, r^2 <= 1e-8 skipped ----------
template <class T, bool REFINE>
struct OpVortAt {
  static constexpr int NV = 3;
  static constexpr bool EXCLUDE_SELF = false;
  __device__ __forceinline__ static void pair(const Tgt<T>& t, T* acc, const Src<T>& s,
                                              int64_t, int64_t) {
    const T rx = t.x - s.x, ry = t.y - s.y, rz = t.z - s.z;
    const T r2 = fma(rx, rx, fma(ry, ry, rz * rz));
    const T s2 = s.s * s.s;
    const T y = rsqrt_t<REFINE>(r2 + s2);
    const T y2 = y * y;
    const T y3 = y2 * y;
    const T y7 = (y3 * y3) * y;
    T k = (s2 * s2) * y7;
    k = (r2 > T(kRefEps)) ? k : T(0);
    acc[0] = fma(k, s.ax, acc[0]);
    acc[1] = fma(k, s.ay, acc[1]);
    acc[2] = fma(k, s.az, acc[2]);
  }
};

// ---- stretching (transpose scheme): A += g (a_j - a_i),  B += f (a_i . (r x a_j)) r -----
template <class T, bool REFINE>
struct OpStretch {
  static constexpr int NV = 6;
  static constexpr bool EXCLUDE_SELF = false;
  __device__ __forceinline__ static void pair(const Tgt<T>& t, T* acc, const Src<T>& s,
                                              int64_t, int64_t) {
    const T rx = t.x - s.x, ry = t.y - s.y, rz = t.z - s.z;
    const T sg = fma(s.s, T(0.5), t.hs);
    const T s2 = sg * sg;
    const T x = fma(rx, rx, fma(ry, ry, fma(rz, rz, s2)));
    const T y = rsqrt_t<REFINE>(x);
    const T y2 = y * y;
    const T y5 = (y2 * y2) * y;
    const T t1 = fma(T(1.5), s2, x);
    const T g = t1 * y5;
    const T f = (t1 + s2) * (y5 * y2);
    const T cx = fma(ry, s.az, -(rz * s.ay));
    const T cy = fma(rz, s.ax, -(rx * s.az));
    const T cz = fma(rx, s.ay, -(ry * s.ax));
    acc[0] = fma(g, s.ax - t.ax, acc[0]);
    acc[1] = fma(g, s.ay - t.ay, acc[1]);
    acc[2] = fma(g, s.az - t.az, acc[2]);
    const T h = f * fma(t.ax, cx, fma(t.ay, cy, t.az * cz));
    acc[3] = fma(h, rx, acc[3]);
    acc[4] = fma(h, ry, acc[4]);
    acc[5] = fma(h, rz, acc[5]);
  }
};

// ---- fused velocity + stretching: U (3), A (3), B (3) ----------------------------------
template <class T, bool REFINE>
struct OpVelStretch {
  static constexpr int NV = 9;
  static constexpr bool EXCLUDE_SELF = false;
  __device__ __forceinline__ static void pair(const Tgt<T>& t, T* acc, const Src<T>& s,
                                              int64_t, int64_t) {
    const T rx = t.x - s.x, ry = t.y - s.y, rz = t.z - s.z;
    const T sg = fma(s.s, T(0.5), t.hs);
    const T s2 = sg * sg;
    const T x = fma(rx, rx, fma(ry, ry, fma(rz, rz, s2)));
    const T y = rsqrt_t<REFINE>(x);
    const T y2 = y * y;
    const T y5 = (y2 * y2) * y;
    const T t1 = fma(T(1.5), s2, x);
    const T g = t1 * y5;
    const T f = (t1 + s2) * (y5 * y2);
    const T cx = fma(ry, s.az, -(rz * s.ay));
    const T cy = fma(rz, s.ax, -(rx * s.az));
    const T cz = fma(rx, s.ay, -(ry * s.ax));
    acc[0] = fma(g, cx, acc[0]);
    acc[1] = fma(g, cy, acc[1]);
    acc[2] = fma(g, cz, acc[2]);
    acc[3] = fma(g, s.ax - t.ax, acc[3]);
    acc[4] = fma(g, s.ay - t.ay, acc[4]);
    acc[5] = fma(g, s.az - t.az, acc[5]);
    const T h = f * fma(t.ax, cx, fma(t.ay, cy, t.az * cz));
    acc[6] = fma(h, rx, acc[6]);
    acc[7] = fma(h, ry, acc[7]);
    acc[8] = fma(h, rz, acc[8]);
  }
};

// ---- PSE diffusion: P += s^7 y^9 (a_j - a_i)  (nu_i applied in finalize) -----------------
template <class T, bool REFINE>
struct OpPse {
  static constexpr int NV = 3;
  static constexpr bool EXCLUDE_SELF = false;
  __device__ __forceinline__ static void pair(const Tgt<T>& t, T* acc, const Src<T>& s,
                                              int64_t, int64_t) {
    const T rx = t.x - s.x, ry = t.y - s.y, rz = t.z - s.z;
    const T sg = fma(s.s, T(0.5), t.hs);
    const T s2 = sg * sg;
    const T x = fma(rx, rx, fma(ry, ry, fma(rz, rz, s2)));
    const T y = rsqrt_t<REFINE>(x);
    const T z = sg * y;  // <= 1
    const T z2 = z * z;
    const T z4 = z2 * z2;
    const T z7 = (z4 * z2) * z;
    const T k = z7 * (y * y);
    acc[0] = fma(k, s.ax - t.ax, acc[0]);
    acc[1] = fma(k, s.ay - t.ay, acc[1]);
    acc[2] = fma(k, s.az - t.az, acc[2]);
  }
};

// ---- enstrophy filter sum (all pairs incl. i == j): V += (x + 2.2 s^2) y^3 a_j ---------
template <class T, bool REFINE>
struct OpEns {
  static constexpr int NV = 3;
  static constexpr bool EXCLUDE_SELF = false;
  __device__ __forceinline__ static void pair(const Tgt<T>& t, T* acc, const Src<T>& s,
                                              int64_t, int64_t) {
    const T rx = t.x - s.x, ry = t.y - s.y, rz = t.z - s.z;
    const T sg = fma(s.s, T(0.5), t.hs);
    const T s2 = sg * sg;
    const T x = fma(rx, rx, fma(ry, ry, fma(rz, rz, s2)));
    const T y = rsqrt_t<REFINE>(x);
    const T y3 = (y * y) * y;
    const T k = fma(T(2.2), s2, x) * y3;
    acc[0] = fma(k, s.ax, acc[0]);
    acc[1] = fma(k, s.ay, acc[1]);
    acc[2] = fma(k, s.az, acc[2]);
  }
};

// ---- kinetic energy (j != i): K += (y + s^2 y^3) a_j + y^3 (r . a_j) r ------------------
template <class T, bool REFINE>
struct OpKe {
  static constexpr int NV = 3;
  static constexpr bool EXCLUDE_SELF = true;
  __device__ __forceinline__ static void pair(const Tgt<T>& t, T* acc, const Src<T>& s,
                                              int64_t i, int64_t j) {
    const T rx = t.x - s.x, ry = t.y - s.y, rz = t.z - s.z;
    const T sg = fma(s.s, T(0.5), t.hs);
    const T s2 = sg * sg;
    const T x = fma(rx, rx, fma(ry, ry, fma(rz, rz, s2)));
    const T y = rsqrt_t<REFINE>(x);
    const T y3 = (y * y) * y;
    T w = fma(s2, y3, y);
    w = (i == j) ? T(0) : w;
    const T q = y3 * fma(rx, s.ax, fma(ry, s.ay, rz * s.az));
    acc[0] = fma(q, rx, fma(w, s.ax, acc[0]));
    acc[1] = fma(q, ry, fma(w, s.ay, acc[1]));
    acc[2] = fma(q, rz, fma(w, s.az, acc[2]));
  }
};

}  // namespace vpm
