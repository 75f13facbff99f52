// vpm_adjoint.cuh -- hand-written adjoint (vector-Jacobian products) of the VPM right-hand
// side and of the kinetic-energy loss.  No counterpart in the reference (it has no adjoint).
//
// Right-hand side of the coupled ODE dx/dt = u, da/dt = S + P (GPU semantics of
// ParticlesPhysicsCuda.py):
//   u_i = -(1/4pi) sum_j g (r_ij x a_j)                                 (:133-191)
//   S_i =  (1/4pi) sum_j [g (a_i x a_j) + f (a_i . (r_ij x a_j)) r_ij]   (:375-445)
//   P_i =  (105 nu_i/4pi) sum_j k (a_j - a_i)                           (:478-530)
// with x = r^2 + s^2, y = x^(-1/2), g = (x + 1.5 s^2) y^5, f = 3 (x + 2.5 s^2) y^7,
// k = s^7 y^9, s = (sigma_i + sigma_j)/2.  Derivatives used (at fixed s, resp. fixed r^2):
//   dg/dr^2 = -f/2,                    dg/ds = -7.5 s^3 y^7
//   df/dr^2 = -7.5 (x + 3.5 s^2) y^9,  df/ds = -52.5 s^3 y^9
//   dk/dr^2 = -4.5 s^7 y^11,           dk/ds = s^6 y^11 (7 r^2 - 2 s^2)
//
// Given cotangents (ubar, sbar) of (u, S + P), the sweep returns (xbar, abar, sigmabar, nubar).
// Cotangents enter the packed record pre-scaled: u' = -ubar/(4pi), s' = sbar/(4pi), and
// nu' = 105 nu, so the pair terms carry no constant factors.
//
// Symmetric gather: the thread owning particle k visits every partner l once and adds the
// contributions of the pair to k in both roles -- k as target i (l as source j) and k as
// source j (l as target i) -- sharing the scalar kernel values, which depend only on r^2 and
// s.  No atomics; results are deterministic.  With r = x_k - x_l, w = a_l x a_k,
// ds = s'_k - s'_l, dp = ds . r, d = r . w, E = u'_k.(r x a_l) - u'_l.(r x a_k) - ds . w,
// D = d dp, Q = nu'_k s'_k.(a_l - a_k) + nu'_l s'_l.(a_k - a_l), K = k:
//   xbar_k   += (2 dg/dr^2 E + 2 df/dr^2 D + 2 dk/dr^2 Q) r + f dp w + f d ds
//               + g (a_l x u'_k - a_k x u'_l)
//   abar_k   += g (a_l x ds + r x u'_l) + f dp (r x a_l) + k (nu'_l s'_l - nu'_k s'_k)
//   dL/ds    += dg/ds E + df/ds D + dk/ds Q          (sigmabar_k = 1/2 of the sum)
//   nubar'_k += k s'_k . (a_l - a_k)
// The g-weighted cross products are factored per target: sum_l g a_l = G_a and
// sum_l g u'_l = G_u are accumulated and crossed with a_k, u'_k, s'_k in the finalize pass.
// The pair l == k is excluded by zeroing y (the forward sums skip j == i).
#pragma once

#include "vpm_pairs.cuh"

namespace vpm {

// Wide record: state, pre-scaled cotangents and the per-particle product m = a x s'
// (160 bytes for both element types; m is formed in FP64 by the pack kernel).
template <class E>
struct alignas(16) RecG {
  E x, y, z, s;
  E ax, ay, az, nu;    // nu holds 105 * nu
  E ux, uy, uz, mx;    // -ubar / (4 pi); m = a x s'
  E gx, gy, gz, my;    // sbar / (4 pi)
  E mz, pad0, pad1, pad2;
};
static_assert(sizeof(RecG<double>) == 160 && sizeof(RecG<float2>) == 160, "RecG is 160 B");

template <class V>
struct SrcG {
  V x, y, z, s, ax, ay, az, nu, ux, uy, uz, gx, gy, gz, mx, my, mz;
};

template <class V>
struct TgtG {
  V x, y, z, hs, ax, ay, az, nu, ux, uy, uz, gx, gy, gz;
};

__device__ __forceinline__ SrcG<double> load_srcg(const RecG<double>& r) {
  const double2* p = reinterpret_cast<const double2*>(&r);
  const double2 a = p[0], b = p[1], c = p[2], d = p[3], e = p[4], f = p[5], g = p[6], h = p[7],
                i = p[8];
  return SrcG<double>{a.x, a.y, b.x, b.y, c.x, c.y, d.x, d.y, e.x, e.y, f.x,
                      g.x, g.y, h.x, f.y, h.y, i.x};
}
__device__ __forceinline__ SrcG<float2> load_srcg(const RecG<float2>& r) {
  const float4* p = reinterpret_cast<const float4*>(&r);
  const float4 a = p[0], b = p[1], c = p[2], d = p[3], e = p[4], f = p[5], g = p[6], h = p[7],
               i = p[8];
  return SrcG<float2>{make_float2(a.x, a.y), make_float2(a.z, a.w), make_float2(b.x, b.y),
                      make_float2(b.z, b.w), make_float2(c.x, c.y), make_float2(c.z, c.w),
                      make_float2(d.x, d.y), make_float2(d.z, d.w), make_float2(e.x, e.y),
                      make_float2(e.z, e.w), make_float2(f.x, f.y), make_float2(g.x, g.y),
                      make_float2(g.z, g.w), make_float2(h.x, h.y), make_float2(f.z, f.w),
                      make_float2(h.z, h.w), make_float2(i.x, i.y)};
}

__device__ __forceinline__ TgtG<double> make_tgtg(const RecG<double>* const* r) {
  const RecG<double>& a = *r[0];
  return TgtG<double>{a.x, a.y, a.z, 0.5 * a.s, a.ax, a.ay, a.az,
                      a.nu, a.ux, a.uy, a.uz, a.gx, a.gy, a.gz};
}
__device__ __forceinline__ TgtG<float2> make_tgtg(const RecG<float2>* const* r) {
  const RecG<float2>& a = *r[0];
  const RecG<float2>& b = *r[1];
  return TgtG<float2>{make_float2(a.x.x, b.x.x),   make_float2(a.y.x, b.y.x),
                      make_float2(a.z.x, b.z.x),   make_float2(0.5f * a.s.x, 0.5f * b.s.x),
                      make_float2(a.ax.x, b.ax.x), make_float2(a.ay.x, b.ay.x),
                      make_float2(a.az.x, b.az.x), make_float2(a.nu.x, b.nu.x),
                      make_float2(a.ux.x, b.ux.x), make_float2(a.uy.x, b.uy.x),
                      make_float2(a.uz.x, b.uz.x), make_float2(a.gx.x, b.gx.x),
                      make_float2(a.gy.x, b.gy.x), make_float2(a.gz.x, b.gz.x)};
}

// Partial values of the adjoint sweep.
enum VjpSlot {
  VJ_X = 0,   // xbar (3)
  VJ_A = 3,   // abar (3)
  VJ_S = 6,   // dL/ds
  VJ_NU = 7,  // dL/dnu'
  VJ_GA = 8,  // sum g a_l (3)
  VJ_GU = 11, // sum g u'_l (3)
  VJ_K = 14,  // sum k        (PSE only)
  VJ_KS = 15  // sum k nu'_l s'_l (3, PSE only)
};

template <class V, bool REFINE, bool PSE>
struct OpRhsVjp {
  static constexpr int NV = PSE ? 18 : 14;
  static constexpr int kR = 2;  // register-heavy: one FP32 lane (two targets) per thread
  static constexpr int kWindow = 0;  // the sweep's default FP32 window
  using Record = RecG<V>;
  using SrcT = SrcG<V>;
  using TgtT = TgtG<V>;
  __device__ __forceinline__ static SrcT load(const Record& r) { return load_srcg(r); }
  __device__ __forceinline__ static TgtT target(const Record* const* r) { return make_tgtg(r); }

  __device__ __forceinline__ static void pair(const TgtT& t, V* acc, const SrcT& s,
                                              const int64_t* i, int64_t j) {
    const V rx = t.x - s.x, ry = t.y - s.y, rz = t.z - s.z;
    const V sg = fma(s.s, splat<V>(0.5), t.hs);
    const V s2 = sg * sg;
    const V x = fma(rx, rx, fma(ry, ry, fma(rz, rz, s2)));
    const V y = zero_if_self(rsqrt_lane<REFINE>(x), i, j);
    const V y2 = y * y;
    const V y5 = (y2 * y2) * y;
    const V y7 = y5 * y2;
    const V y9 = y7 * y2;
    const V s3 = s2 * sg;
    const V t1 = fma(splat<V>(1.5), s2, x);
    const V g = t1 * y5;
    const V t2 = t1 + s2;
    const V f = splat<V>(3.0) * (t2 * y7);
    const V m2gr = f;                                          // -2 dg/dr^2
    const V gs = splat<V>(-7.5) * (s3 * y7);                   // dg/ds
    const V f2r = splat<V>(-15.0) * ((t2 + s2) * y9);          // 2 df/dr^2
    const V fs = splat<V>(-52.5) * (s3 * y9);                  // df/ds

    // cross products
    const V clx = fma(ry, s.az, -(rz * s.ay));  // r x a_l
    const V cly = fma(rz, s.ax, -(rx * s.az));
    const V clz = fma(rx, s.ay, -(ry * s.ax));
    const V ckx = fma(ry, t.az, -(rz * t.ay));  // r x a_k
    const V cky = fma(rz, t.ax, -(rx * t.az));
    const V ckz = fma(rx, t.ay, -(ry * t.ax));
    const V wx = fma(s.ay, t.az, -(s.az * t.ay));  // w = a_l x a_k
    const V wy = fma(s.az, t.ax, -(s.ax * t.az));
    const V wz = fma(s.ax, t.ay, -(s.ay * t.ax));
    const V dsx = t.gx - s.gx, dsy = t.gy - s.gy, dsz = t.gz - s.gz;
    const V eT = fma(t.ux, clx, fma(t.uy, cly, t.uz * clz));
    const V eS = fma(s.ux, ckx, fma(s.uy, cky, s.uz * ckz));
    const V dsw = fma(dsx, wx, fma(dsy, wy, dsz * wz));
    const V E = (eT - eS) - dsw;
    const V d = fma(rx, wx, fma(ry, wy, rz * wz));
    const V dp = fma(dsx, rx, fma(dsy, ry, dsz * rz));
    const V D = d * dp;
    V cr = fma(f2r, D, -(m2gr * E));  // 2 dg/dr^2 E + 2 df/dr^2 D
    V sd = fma(gs, E, fs * D);
    if constexpr (PSE) {
      const V z = sg * y;
      const V z2 = z * z;
      const V z6 = (z2 * z2) * z2;
      const V k = (z6 * z) * y2;                      // s^7 y^9
      const V k2r = splat<V>(-9.0) * (k * y2);        // 2 dk/dr^2
      const V r2 = x - s2;
      const V ks = (z6 * y2) * y2 * y * fma(splat<V>(7.0), r2, splat<V>(-2.0) * s2);  // dk/ds
      const V ddx = s.ax - t.ax, ddy = s.ay - t.ay, ddz = s.az - t.az;  // a_l - a_k
      const V qT = fma(t.gx, ddx, fma(t.gy, ddy, t.gz * ddz));
      const V qS = fma(s.gx, ddx, fma(s.gy, ddy, s.gz * ddz));
      const V Q = fma(t.nu, qT, -(s.nu * qS));
      cr = fma(k2r, Q, cr);
      sd = fma(ks, Q, sd);
      acc[VJ_NU] = fma(k, qT, acc[VJ_NU]);
      acc[VJ_K] = acc[VJ_K] + k;
      const V kn = k * s.nu;
      acc[VJ_KS + 0] = fma(kn, s.gx, acc[VJ_KS + 0]);
      acc[VJ_KS + 1] = fma(kn, s.gy, acc[VJ_KS + 1]);
      acc[VJ_KS + 2] = fma(kn, s.gz, acc[VJ_KS + 2]);
    }
    const V fdp = f * dp;
    const V fd = f * d;
    acc[VJ_X + 0] = fma(cr, rx, fma(fdp, wx, fma(fd, dsx, acc[VJ_X + 0])));
    acc[VJ_X + 1] = fma(cr, ry, fma(fdp, wy, fma(fd, dsy, acc[VJ_X + 1])));
    acc[VJ_X + 2] = fma(cr, rz, fma(fdp, wz, fma(fd, dsz, acc[VJ_X + 2])));
    acc[VJ_S] = acc[VJ_S] + sd;
    acc[VJ_GA + 0] = fma(g, s.ax, acc[VJ_GA + 0]);
    acc[VJ_GA + 1] = fma(g, s.ay, acc[VJ_GA + 1]);
    acc[VJ_GA + 2] = fma(g, s.az, acc[VJ_GA + 2]);
    acc[VJ_GU + 0] = fma(g, s.ux, acc[VJ_GU + 0]);
    acc[VJ_GU + 1] = fma(g, s.uy, acc[VJ_GU + 1]);
    acc[VJ_GU + 2] = fma(g, s.uz, acc[VJ_GU + 2]);
    // abar: g (r x u'_l - a_l x s'_l) + f dp (r x a_l); the G_a x s'_k part is in finalize
    const V nx = fma(ry, s.uz, -(rz * s.uy)) - s.mx;  // m_l = a_l x s'_l from the record
    const V ny = fma(rz, s.ux, -(rx * s.uz)) - s.my;
    const V nz = fma(rx, s.uy, -(ry * s.ux)) - s.mz;
    acc[VJ_A + 0] = fma(g, nx, fma(fdp, clx, acc[VJ_A + 0]));
    acc[VJ_A + 1] = fma(g, ny, fma(fdp, cly, acc[VJ_A + 1]));
    acc[VJ_A + 2] = fma(g, nz, fma(fdp, clz, acc[VJ_A + 2]));
  }
};

// Gradient of the kinetic energy E = (1/16pi) sum_{i != j} h_ij,
// h = P1 (y + s^2 y^3) + y^3 (r.a_i)(r.a_j), P1 = a_i.a_j  (ParticlesPhysicsCuda.py:563-642).
// h is symmetric in (i, j), so dE/dz_k = (2/16pi) sum_{l != k} dh(k,l)/dz_k:
//   abar  += w a_l + y^3 (r.a_l) r,                      w = y + s^2 y^3
//   xbar  += 2 dh/dr^2 r + y^3 ((r.a_l) a_k + (r.a_k) a_l)
//   dh/ds += P1 (s y^3 - 3 s^3 y^5) - 3 s y^5 (r.a_k)(r.a_l)
// with dh/dr^2 = -P1 (y^3/2 + 1.5 s^2 y^5) - 1.5 y^5 (r.a_k)(r.a_l).
template <class V, bool REFINE>
struct OpKeGrad : PairOpBase<V> {
  static constexpr int NV = 7;
  __device__ __forceinline__ static void pair(const Tgt<V>& t, V* acc, const Src<V>& s,
                                              const int64_t* i, int64_t j) {
    const V rx = t.x - s.x, ry = t.y - s.y, rz = t.z - s.z;
    const V sg = fma(s.s, splat<V>(0.5), t.hs);
    const V s2 = sg * sg;
    const V x = fma(rx, rx, fma(ry, ry, fma(rz, rz, s2)));
    const V y = zero_if_self(rsqrt_lane<REFINE>(x), i, j);
    const V y2 = y * y;
    const V y3 = y2 * y;
    const V y5 = y3 * y2;
    const V w = fma(s2, y3, y);
    const V p1 = fma(t.ax, s.ax, fma(t.ay, s.ay, t.az * s.az));
    const V rl = fma(rx, s.ax, fma(ry, s.ay, rz * s.az));
    const V rk = fma(rx, t.ax, fma(ry, t.ay, rz * t.az));
    const V rr = rk * rl;
    const V q = y3 * rl;
    acc[3] = fma(q, rx, fma(w, s.ax, acc[3]));
    acc[4] = fma(q, ry, fma(w, s.ay, acc[4]));
    acc[5] = fma(q, rz, fma(w, s.az, acc[5]));
    // 2 dh/dr^2 = -P1 (y^3 + 3 s^2 y^5) - 3 y^5 rr
    const V h2r = -fma(p1, fma(splat<V>(3.0) * s2, y5, y3), splat<V>(3.0) * (y5 * rr));
    const V yk = y3 * rk;
    acc[0] = fma(h2r, rx, fma(q, t.ax, fma(yk, s.ax, acc[0])));
    acc[1] = fma(h2r, ry, fma(q, t.ay, fma(yk, s.ay, acc[1])));
    acc[2] = fma(h2r, rz, fma(q, t.az, fma(yk, s.az, acc[2])));
    // dh/ds = s [P1 (y^3 - 3 s^2 y^5) - 3 y^5 rr]
    const V hs = sg * fma(p1, fma(splat<V>(-3.0) * s2, y5, y3), splat<V>(-3.0) * (y5 * rr));
    acc[6] = acc[6] + hs;
  }
};

}  // namespace vpm
