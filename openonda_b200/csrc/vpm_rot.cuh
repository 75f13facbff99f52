// vpm_rot.cuh -- both-sides sweeps of the self sums (FP32-compensated: fused velocity +
// stretching, velocity, PSE, the LES step sums, the adjoint of (u, S); FP64: the fused,
// velocity and PSE sums), with the source side carried around the warp in registers.
//
// The pair terms of (i <- j) and (j <- i) share r^2, the core, the rsqrt and the kernel
// values.  Seen from particle j, with r = x_i - x_j as computed for target i:
//   U_j += -g (r x a_i),   A_j += -g (a_j - a_i),   B_j += -h r,   h = f a_i . (r x a_j),
//   P_j += -k (a_j - a_i)   (PSE; nu_j is applied per particle in the finalize),
// so one evaluation of an unordered pair costs 53 FP32 lane-ops instead of 2 x 38 for the
// fused sum, 31 instead of 2 x 22 for the velocity, 24 instead of 2 x 21 for PSE, 69-82
// instead of 2 x 52-56 for the four LES step sums and about 128 instead of 2 x 100 for the
// adjoint.
//
// Warp layout: each lane holds 2 kP targets (kP packed FP32x2 lanes: 3 for the fused,
// velocity and PSE sums, 2 for the LES sums and the adjoint, 1 for the adjoint with PSE) and
// one source of the current batch of 32 (read from L2, the next batch prefetched).  In 32
// steps every lane meets every source of the batch: after each step the sources and their
// source-side accumulators move one lane down (__shfl_sync), so after the 32nd step each
// source is back in its lane with its sums over the warp's 64 kP targets.  Warp shuffles are
// the second-scarcest resource here; six targets per lane keep them at 25 per 384 ordered
// pairs for the fused sum.  The source-side sums are then added over the CTA's warps in FP64
// (fixed order) and added into the accumulator of the source particle with a non-returning
// atomic.
//
// Tile-pair schedule: particles form nt tiles of T = 64 kP WARPS.  A CTA owns one tile pair
// (I, J), I < J.  Diagonal pair q of a launch is J - I = k (accumulator sets 2q / 2q+1 for
// the target / source side) together with J - I = nt - k (sets 2q+1 / 2q, on row ranges
// disjoint from the first diagonal's): every accumulator element has one writer per launch
// and the launches run in stream order, so the atomic additions happen in a fixed order and
// the result is deterministic.  A launch runs m
// consecutive diagonal pairs (m chosen so that its m * nt CTAs fill whole waves); launch 0
// runs the diagonal tiles (I, I) one-sided, each in kRotDiagSplit CTAs that take a part of the
// tile's sources each and add into sets 0 .. kRotDiagSplit - 1.  The finalize pass sums the
// max(2m, kRotDiagSplit) sets in order.
//
// Accumulation (FP32 kernel): target side in FP32 over windows of 16 to 64 steps per value
// (kTgtWindow, kTgtWindowShort, kTgtWindowLong), folded into FP64 carries held in shared
// memory; source side in FP32 over windows of kSrcWindow steps (each half of the packed
// accumulator sums kSrcWindow kP terms), the windows of a batch added in FP32 in shared
// memory, then both halves in FP64 across warps and tile pairs.  The FP64 kernel
// (rot64_sweep_kernel, at the end) keeps every sum in FP64 registers.
#pragma once

#include "vpm_adjoint.cuh"
#include "vpm_sweep.cuh"

namespace vpm {

// Build parameters: warps per CTA; resident CTAs per SM the registers are sized for (fused
// sum VPM_ROT_MINB and a second build VPM_ROT_MINB_ALT, three-sum operators VPM_ROT3_MINB,
// LES step VPM_ROT15_MINB, whose 77 KB of shared memory allow two, adjoint VPM_ROTG_MINB and
// VPM_ROTGP_MINB); unroll of the 32 steps; packed target lanes per thread (VPM_ROT_P,
// VPM_ROT3_P, VPM_ROTG_P, VPM_ROTGP_P; the LES operator holds two).
#ifndef VPM_ROT_WARPS
#define VPM_ROT_WARPS 4
#endif
#ifndef VPM_ROT_MINB
#define VPM_ROT_MINB 3
#endif
#ifndef VPM_ROT_MINB_ALT
#define VPM_ROT_MINB_ALT 2
#endif
#ifndef VPM_ROT3_MINB
#define VPM_ROT3_MINB 3
#endif
#ifndef VPM_ROT_P
#define VPM_ROT_P 3
#endif
#ifndef VPM_ROT3_P
#define VPM_ROT3_P 3
#endif
#ifndef VPM_ROT15_MINB
#define VPM_ROT15_MINB 2
#endif
#ifndef VPM_ROT_UNROLL
#define VPM_ROT_UNROLL 8
#endif
#ifndef VPM_ROT15_UNROLL
#define VPM_ROT15_UNROLL 2
#endif
#ifndef VPM_ROTG_P
#define VPM_ROTG_P 2
#endif
#ifndef VPM_ROTG_MINB
#define VPM_ROTG_MINB 2
#endif
#ifndef VPM_ROTG_UNROLL
#define VPM_ROTG_UNROLL 2
#endif
#ifndef VPM_ROTGP_P
#define VPM_ROTGP_P 1
#endif
#ifndef VPM_ROTGP_MINB
#define VPM_ROTGP_MINB 2
#endif
#ifndef VPM_ROTGP_UNROLL
#define VPM_ROTGP_UNROLL 2
#endif

constexpr int kRotWarps = VPM_ROT_WARPS;
// The diagonal tiles (one launch of their own) split their sources into this many parts, one
// CTA each, so that the launch fills more of the GPU; part h adds into accumulator set h.
constexpr int kRotDiagSplit = 4;
constexpr int kRotThreads = 32 * kRotWarps;
constexpr float kRotFar = 1e15f;  // position of the padding sources: every kernel underflows

struct RotArgs {
  const void* rec;  // packed records of all n particles (the operator's record type)
  int64_t n;
  int nt;       // tiles of the operator's rot_tile particles
  int k0;       // first diagonal of this launch (0 = the diagonal tiles)
  double* acc;  // accumulators [sets][NV][n]
  int set0 = 0;   // the diagonal tiles' launch: its first accumulator set
  int tile0 = 0;  // the diagonal tiles' launch: its first tile (a part of a sweep)
};

// Particles per tile: kP packed FP32x2 target lanes (2 kP targets) per thread.
template <class Op>
__host__ __device__ constexpr int rot_tile() {
  return 64 * Op::kP * kRotWarps;
}

// Source-side window (Op::kSrcWindow steps): at the end of a window each lane adds the packed
// FP32 sums of the source it holds into that source's slot in shared memory and starts again
// from zero, so no FP32 sum runs over more than kSrcWindow * kP terms.  The stretching sums
// (fused, LES step) take short windows for accuracy; velocity, PSE and the adjoint, whose
// errors are far inside their bars, take one window per batch.
#ifndef VPM_ROT_SRC_WINDOW
#define VPM_ROT_SRC_WINDOW 8
#endif
#ifndef VPM_ROT3_SRC_WINDOW
#define VPM_ROT3_SRC_WINDOW 32
#endif
#ifndef VPM_ROTG_SRC_WINDOW
#define VPM_ROTG_SRC_WINDOW 32
#endif
#ifndef VPM_ROT_TGT_WINDOW
#define VPM_ROT_TGT_WINDOW 32
#endif
// Target-side windows per value in the fused and LES operators.  The stretching term
// g (a_j - a_i) (values 3-5) has the FP32 partial sums that cancel most: its error sets the
// stretching error and grows with the window, so it folds every 16 steps.  The other values
// (velocity, the stretching term f (r . (a_i x (r x a_j))) r, vorticity, the enstrophy filter
// sum) fold every 64 steps, so a 64-step span has as many folds as with 32-step windows for
// all.  On the leapfrogging rings (N = 131072, 50 steps) the stretching error went from
// 1.5-1.9e-6 to 0.9-1.2e-6 and the velocity error from 0.8-0.9e-7 to 1.2-1.4e-7, at the
// same sweep time; on the dynamic-LES ring (N = 2^20) the LES step's stretching error from
// 1.65e-6 to 1.48e-6 and its vorticity error from 2.9e-7 to 3.8e-7.
#ifndef VPM_ROT_STRETCH_TGT_WINDOW
#define VPM_ROT_STRETCH_TGT_WINDOW 16
#endif
#ifndef VPM_ROT_LONG_TGT_WINDOW
#define VPM_ROT_LONG_TGT_WINDOW 64
#endif

// Dynamic shared memory of one CTA: the target-side FP64 carries [NV][T], then the
// source-side sums of the first kSymFrom values, [kJBufs][kSymFrom][warps * 32].
template <class Op>
constexpr size_t rot_smem_bytes() {
  if constexpr (Op::kFP64) {
    // FP64 kernel: the warps' source-side sums of a batch only, [kSymFrom][warps * 32]
    return size_t(Op::kSymFrom) * kRotWarps * 32 * sizeof(double);
  } else {
    return size_t(rot_tile<Op>()) * Op::NV * sizeof(double) +
           size_t(Op::kJBufs) * Op::kSymFrom * kRotWarps * 32 * sizeof(float2);
  }
}

// The source a lane holds on the standard 64-byte record: position, core, strength.
struct RotSrc {
  float x, y, z, s, ax, ay, az;
};

// Rotation policy of the operators on the standard record (Rec<float2>): four targets per
// lane; the source's position, strength and (for general cores) core move around the warp.
template <class OneSidedOp, bool UC>
struct RotStd {
  using V = float2;
  using Record = Rec<float2>;
  using OneSided = OneSidedOp;
  using TgtT = Tgt<float2>;
  using SrcT = Src<float2>;
  using Lane = RotSrc;
  static constexpr int kP = 2;
  static constexpr bool kSrcCore = !UC;  // the pair core needs the source's sigma

  // Source j of the packed records (j < n), or a padding source far away with no strength.
  __device__ __forceinline__ static Lane load_lane(const Record* rec, int64_t j, int64_t n) {
    if (j < n) {
      const float4* p = reinterpret_cast<const float4*>(rec + j);
      const float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2), d = __ldg(p + 3);
      return Lane{a.x, a.z, b.x, b.z, c.x, c.z, d.x};
    }
    return Lane{kRotFar, kRotFar, kRotFar, 1.f, 0.f, 0.f, 0.f};
  }
  // lane l takes what lane src_lane held
  __device__ __forceinline__ static void shuffle(Lane& c, int src_lane) {
    c.x = __shfl_sync(0xffffffffu, c.x, src_lane);
    c.y = __shfl_sync(0xffffffffu, c.y, src_lane);
    c.z = __shfl_sync(0xffffffffu, c.z, src_lane);
    if constexpr (kSrcCore) c.s = __shfl_sync(0xffffffffu, c.s, src_lane);
    c.ax = __shfl_sync(0xffffffffu, c.ax, src_lane);
    c.ay = __shfl_sync(0xffffffffu, c.ay, src_lane);
    c.az = __shfl_sync(0xffffffffu, c.az, src_lane);
  }
  __device__ __forceinline__ static SrcT broadcast(const Lane& c) {
    return SrcT{make_float2(c.x, c.x),   make_float2(c.y, c.y),   make_float2(c.z, c.z),
                make_float2(c.s, c.s),   make_float2(c.ax, c.ax), make_float2(c.ay, c.ay),
                make_float2(c.az, c.az), make_float2(0.f, 0.f)};
  }
  __device__ __forceinline__ static TgtT target(const Record* const* r) { return make_tgt(r); }
  // Uniform cores: every record carries the same core, so the target's core, core^2 and
  // core^4 come from one record for all of a thread's packed lanes (one register pair each
  // instead of one per lane; the values are the same bits as the lanes' own)
  static constexpr bool kFP64 = false;  // the FP32 kernel (rot_sweep_kernel)
  static constexpr bool kCustomDiag = false;  // the diagonal tiles take OneSided::pair
  static constexpr bool kUniformCore = UC;
  __device__ __forceinline__ static void uniform_core(TgtT& t, const Record* rec) {
    const float sc = rec[0].s.x, s2 = sc * sc;
    t.sc = make_float2(sc, sc);
    t.s2c = make_float2(s2, s2);
    t.s4c = make_float2(s2 * s2, s2 * s2);
  }
  // one-sided pair of the diagonal tiles; these operators need no index for the pair i == j
  // (it adds nothing, except the enstrophy filter sum, which includes it as the reference does)
  __device__ __forceinline__ static void diag(const TgtT& t, V* acc, const SrcT& s,
                                              const int64_t*, int64_t) {
    OneSided::pair(t, acc, s, nullptr, 0);
  }
  // every source-side sum is carried and stored
  __device__ __forceinline__ static constexpr bool carried(int) { return true; }
  // values folded into the FP64 carries every kTgtWindowShort steps instead of every
  // kTgtWindow (0: none), and values folded every kTgtWindowLong steps (whole batches; 0: none)
  static constexpr int kTgtWindowShort = 0;
  __device__ __forceinline__ static constexpr bool short_fold(int) { return false; }
  static constexpr int kTgtWindowLong = 0;
  __device__ __forceinline__ static constexpr bool long_fold(int) { return false; }
};

// Fused velocity + stretching, both sides of the pair (FP32x2 lanes).  Built for 3 and for 2
// resident CTAs per SM (MINB); the planner takes the one whose launches fill the waves better.
template <bool REFINE, bool UC, int MINB = VPM_ROT_MINB, int P = VPM_ROT_P>
struct OpVelStretchBoth : RotStd<OpVelStretch<float2, REFINE, UC>, UC> {
  using V = float2;
  static constexpr int NV = 9;
  static constexpr int kP = P;
  static constexpr int kMinBlocks = MINB;
  static constexpr int kUnroll = VPM_ROT_UNROLL;
  static constexpr int kSrcWindow = VPM_ROT_SRC_WINDOW;
  static constexpr int kTgtWindow = VPM_ROT_TGT_WINDOW;
  static constexpr int kTgtWindowShort = VPM_ROT_STRETCH_TGT_WINDOW;
  static constexpr int kTgtWindowLong = VPM_ROT_LONG_TGT_WINDOW;
  static constexpr int kSymFrom = NV;  // every sum has a source side
  static constexpr int kJBufs = 2;     // double-buffered source-side sums
  __device__ __forceinline__ static constexpr bool short_fold(int v) { return v >= 3 && v < 6; }
  __device__ __forceinline__ static constexpr bool long_fold(int v) { return v < 3 || v >= 6; }
  // one unordered pair for both particles, in any lane type (float2 here; double in the FP64
  // operator below)
  template <class W>
  __device__ __forceinline__ static void pair2(const Tgt<W>& t, W* acc, W* jv,
                                               const Src<W>& s) {
    using V = W;
    const V rx = t.x - s.x, ry = t.y - s.y, rz = t.z - s.z;
    V sg, s2;
    pair_core<UC>(t, s, sg, s2);
    const V x = fma(rx, rx, fma(ry, ry, fma(rz, rz, s2)));
    const V y = rsqrt_lane<REFINE>(x);
    const V y2 = y * y;
    V g, f;
    if constexpr (UC) {
      // (x + 1.5 s^2) y^5 = y^3 (1 + 1.5 s^2 y^2) and (x + 2.5 s^2) y^7 = y^5 (1 + 2.5 s^2 y^2),
      // with 1.5 s^2 and 2.5 s^2 loop-invariant: one op fewer per pair
      const V y3 = y2 * y;
      g = y3 * fma(splat<V>(1.5f) * s2, y2, splat<V>(1.f));
      f = (y3 * y2) * fma(splat<V>(2.5f) * s2, y2, splat<V>(1.f));
    } else {
      const V y5 = (y2 * y2) * y;
      const V t1 = fma(splat<V>(1.5), s2, x);
      g = t1 * y5;
      f = (t1 + s2) * (y5 * y2);
    }
    const V cx = fma(ry, s.az, -(rz * s.ay));
    const V cy = fma(rz, s.ax, -(rx * s.az));
    const V cz = fma(rx, s.ay, -(ry * s.ax));
    acc[0] = fma(g, cx, acc[0]);
    acc[1] = fma(g, cy, acc[1]);
    acc[2] = fma(g, cz, acc[2]);
    const V dx = s.ax - t.ax, dy = s.ay - t.ay, dz = s.az - t.az;
    acc[3] = fma(g, dx, acc[3]);
    acc[4] = fma(g, dy, acc[4]);
    acc[5] = fma(g, dz, acc[5]);
    const V h = f * fma(t.ax, cx, fma(t.ay, cy, t.az * cz));
    acc[6] = fma(h, rx, acc[6]);
    acc[7] = fma(h, ry, acc[7]);
    acc[8] = fma(h, rz, acc[8]);
    // source side, accumulated with the opposite sign (negated when it is stored)
    const V ex = fma(ry, t.az, -(rz * t.ay));  // r x a_i
    const V ey = fma(rz, t.ax, -(rx * t.az));
    const V ez = fma(rx, t.ay, -(ry * t.ax));
    jv[0] = fma(g, ex, jv[0]);
    jv[1] = fma(g, ey, jv[1]);
    jv[2] = fma(g, ez, jv[2]);
    jv[3] = fma(g, dx, jv[3]);
    jv[4] = fma(g, dy, jv[4]);
    jv[5] = fma(g, dz, jv[5]);
    jv[6] = fma(h, rx, jv[6]);
    jv[7] = fma(h, ry, jv[7]);
    jv[8] = fma(h, rz, jv[8]);
  }
};

// Self-induced velocity, both sides of the pair (FP32x2 lanes): U_j += -g (r x a_i).
template <bool REFINE, bool UC>
struct OpVelBoth : RotStd<OpVel<float2, REFINE, UC>, UC> {
  using V = float2;
  static constexpr int NV = 3;
  static constexpr int kP = VPM_ROT3_P;
  static constexpr int kMinBlocks = VPM_ROT3_MINB;
  static constexpr int kUnroll = VPM_ROT_UNROLL;
  static constexpr int kSrcWindow = VPM_ROT3_SRC_WINDOW;
  static constexpr int kTgtWindow = 32;
  static constexpr int kSymFrom = NV;
  static constexpr int kJBufs = 2;
  template <class W>
  __device__ __forceinline__ static void pair2(const Tgt<W>& t, W* acc, W* jv,
                                               const Src<W>& s) {
    using V = W;
    const V rx = t.x - s.x, ry = t.y - s.y, rz = t.z - s.z;
    V sg, s2;
    pair_core<UC>(t, s, sg, s2);
    const V x = fma(rx, rx, fma(ry, ry, fma(rz, rz, s2)));
    const V y = rsqrt_lane<REFINE>(x);
    const V y2 = y * y;
    V g;
    if constexpr (UC) {
      g = (y2 * y) * fma(splat<V>(1.5f) * s2, y2, splat<V>(1.f));  // y^3 (1 + 1.5 s^2 y^2)
    } else {
      const V y5 = (y2 * y2) * y;
      g = fma(splat<V>(1.5), s2, x) * y5;
    }
    const V cx = fma(ry, s.az, -(rz * s.ay));  // r x a_j
    const V cy = fma(rz, s.ax, -(rx * s.az));
    const V cz = fma(rx, s.ay, -(ry * s.ax));
    acc[0] = fma(g, cx, acc[0]);
    acc[1] = fma(g, cy, acc[1]);
    acc[2] = fma(g, cz, acc[2]);
    // source side, accumulated with the opposite sign (negated when it is stored)
    const V ex = fma(ry, t.az, -(rz * t.ay));  // r x a_i
    const V ey = fma(rz, t.ax, -(rx * t.az));
    const V ez = fma(rx, t.ay, -(ry * t.ax));
    jv[0] = fma(g, ex, jv[0]);
    jv[1] = fma(g, ey, jv[1]);
    jv[2] = fma(g, ez, jv[2]);
  }
};

// PSE diffusion, both sides of the pair (FP32x2 lanes): the kernel value k is symmetric and
// the exchange antisymmetric, P_j += -k (a_j - a_i); nu of each particle is applied by the
// finalize.
template <bool REFINE, bool UC>
struct OpPseBoth : RotStd<OpPse<float2, REFINE, UC>, UC> {
  using V = float2;
  static constexpr int NV = 3;
  static constexpr int kP = VPM_ROT3_P;
  static constexpr int kMinBlocks = VPM_ROT3_MINB;
  static constexpr int kUnroll = VPM_ROT_UNROLL;
  static constexpr int kSrcWindow = VPM_ROT3_SRC_WINDOW;
  static constexpr int kTgtWindow = 32;
  static constexpr int kSymFrom = NV;
  static constexpr int kJBufs = 2;
  template <class W>
  __device__ __forceinline__ static void pair2(const Tgt<W>& t, W* acc, W* jv,
                                               const Src<W>& s) {
    using V = W;
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
    const V dx = s.ax - t.ax, dy = s.ay - t.ay, dz = s.az - t.az;
    acc[0] = fma(k, dx, acc[0]);
    acc[1] = fma(k, dy, acc[1]);
    acc[2] = fma(k, dz, acc[2]);
    jv[0] = fma(k, dx, jv[0]);  // negated when it is stored
    jv[1] = fma(k, dy, jv[1]);
    jv[2] = fma(k, dz, jv[2]);
  }
};

// The four sums of a dynamic-LES step (OpLesStep), both sides of the pair (FP32x2 lanes):
// velocity and stretching as OpVelStretchBoth; the vorticity filter sum uses the core of the
// particle that is summed over, so target i takes s_j^4 (r^2 + s_j^2)^-7/2 a_j and particle
// j takes s_i^4 (r^2 + s_i^2)^-7/2 a_i (one rsqrt each; with uniform cores both equal the
// pair core's y and need none); the enstrophy filter sum (x + 2.2 s^2) y^3 is symmetric.
// The vorticity sum is symmetric, so its source-side terms enter negated (the stored value is
// negated once more).  Pairs with r^2 <= 1e-8 add no vorticity.  Only the scalar
// sum_i a_i . E_i of the enstrophy filter sum is wanted, so each target carries the one sum
// sum_j ke (a_i . a_j) (value 12) in place of the three components of E_i.  65 FP32 lane-ops
// per unordered pair with uniform cores, about 80 without (one-sided: 2 x 52, 2 x 56).  Two
// CTAs per SM, step loop unrolled 2.
// v where a > thr, else 0 (per packed lane)
__device__ __forceinline__ float2 keep_if_gt(float2 a, double thr, float2 v) {
  const float t = float(thr);
  return make_float2(a.x > t ? v.x : 0.f, a.y > t ? v.y : 0.f);
}
__device__ __forceinline__ double keep_if_gt(double a, double thr, double v) {
  return a > thr ? v : 0.0;
}

template <bool REFINE, bool UC>
struct OpLesStepBoth : RotStd<OpLesStep<float2, REFINE, UC>, UC> {
  using V = float2;
  using OneSided = OpLesStep<float2, REFINE, UC>;
  static constexpr int NV = 13;
  static constexpr int kMinBlocks = VPM_ROT15_MINB;
  static constexpr int kUnroll = VPM_ROT15_UNROLL;
  static constexpr int kSrcWindow = VPM_ROT_SRC_WINDOW;
  static constexpr int kTgtWindow = VPM_ROT_TGT_WINDOW;
  static constexpr int kTgtWindowShort = VPM_ROT_STRETCH_TGT_WINDOW;
  static constexpr int kTgtWindowLong = VPM_ROT_LONG_TGT_WINDOW;
  __device__ __forceinline__ static constexpr bool short_fold(int v) { return v >= 3 && v < 6; }
  __device__ __forceinline__ static constexpr bool long_fold(int v) { return v < 3 || v >= 6; }
  // value 12 (enstrophy filter sum) is taken once per unordered pair, target side only
  static constexpr int kSymFrom = 12;
  // three resident CTAs fit the shared memory only with one buffer of source-side sums
  static constexpr int kJBufs = VPM_ROT15_MINB >= 3 ? 1 : 2;
  __device__ __forceinline__ static constexpr bool carried(int v) { return v < kSymFrom; }
  static constexpr bool kCustomDiag = true;  // the FP64 kernel calls diag<double>
  template <class W>
  __device__ __forceinline__ static void pair2(const Tgt<W>& t, W* acc, W* jv,
                                               const Src<W>& s) {
    using V = W;
    const V rx = t.x - s.x, ry = t.y - s.y, rz = t.z - s.z;
    V sg, s2;
    pair_core<UC>(t, s, sg, s2);
    const V r2 = fma(rx, rx, fma(ry, ry, rz * rz));
    const V x = r2 + s2;
    const V y = rsqrt_lane<REFINE>(x);
    const V y2 = y * y;
    const V y3 = y2 * y;
    const V y5 = y3 * y2;
    // (the y^3 (1 + 1.5 s^2 y^2) form of the other operators measured slower here)
    const V y7 = y5 * y2;
    const V t1 = fma(splat<V>(1.5), s2, x);
    const V g = t1 * y5;
    const V f = (t1 + s2) * y7;
    const V cx = fma(ry, s.az, -(rz * s.ay));  // r x a_j
    const V cy = fma(rz, s.ax, -(rx * s.az));
    const V cz = fma(rx, s.ay, -(ry * s.ax));
    acc[0] = fma(g, cx, acc[0]);
    acc[1] = fma(g, cy, acc[1]);
    acc[2] = fma(g, cz, acc[2]);
    const V dx = s.ax - t.ax, dy = s.ay - t.ay, dz = s.az - t.az;
    acc[3] = fma(g, dx, acc[3]);
    acc[4] = fma(g, dy, acc[4]);
    acc[5] = fma(g, dz, acc[5]);
    const V h = f * fma(t.ax, cx, fma(t.ay, cy, t.az * cz));
    acc[6] = fma(h, rx, acc[6]);
    acc[7] = fma(h, ry, acc[7]);
    acc[8] = fma(h, rz, acc[8]);
    const V ex = fma(ry, t.az, -(rz * t.ay));  // r x a_i
    const V ey = fma(rz, t.ax, -(rx * t.az));
    const V ez = fma(rx, t.ay, -(ry * t.ax));
    jv[0] = fma(g, ex, jv[0]);
    jv[1] = fma(g, ey, jv[1]);
    jv[2] = fma(g, ez, jv[2]);
    jv[3] = fma(g, dx, jv[3]);
    jv[4] = fma(g, dy, jv[4]);
    jv[5] = fma(g, dz, jv[5]);
    jv[6] = fma(h, rx, jv[6]);
    jv[7] = fma(h, ry, jv[7]);
    jv[8] = fma(h, rz, jv[8]);
    // vorticity filter sums: kernel values zeroed for r^2 <= 1e-8
    V ki, kj;
    if constexpr (UC) {
      ki = t.s4c * y7;
      kj = ki;
    } else {
      const V sj2 = s.s * s.s;
      const V yi = rsqrt_lane<REFINE>(r2 + sj2);  // source core: target i's sum
      const V yi2 = yi * yi;
      const V yi3 = yi2 * yi;
      ki = (sj2 * sj2) * ((yi3 * yi3) * yi);
      const V yj = rsqrt_lane<REFINE>(r2 + t.s2c);  // target core: particle j's sum
      const V yj2 = yj * yj;
      const V yj3 = yj2 * yj;
      kj = t.s4c * ((yj3 * yj3) * yj);
    }
    ki = keep_if_gt(r2, kRefEps, ki);
    kj = keep_if_gt(r2, kRefEps, kj);
    acc[9] = fma(ki, s.ax, acc[9]);
    acc[10] = fma(ki, s.ay, acc[10]);
    acc[11] = fma(ki, s.az, acc[11]);
    jv[9] = fma(-kj, t.ax, jv[9]);
    jv[10] = fma(-kj, t.ay, jv[10]);
    jv[11] = fma(-kj, t.az, jv[11]);
    // enstrophy filter sum (pair core): the pair term ke (a_i . a_j) is symmetric, so target
    // i takes the pair once and the finalize doubles it; particle j takes nothing (the
    // diagonal tiles, visited one-sided, are folded at half weight)
    const V ke = fma(splat<V>(2.2), s2, x) * y3;
    acc[12] = fma(ke, fma(t.ax, s.ax, fma(t.ay, s.ay, t.az * s.az)), acc[12]);
  }
  // one-sided pair of the diagonal tiles: the one-sided operator's 15 sums, its enstrophy
  // components E_i dotted with a_i into value 12 (any lane type)
  template <class W>
  __device__ __forceinline__ static void diag(const Tgt<W>& t, W* acc, const Src<W>& s,
                                              const int64_t*, int64_t) {
    using V = W;
    using One = OpLesStep<W, REFINE, UC>;
    V full[One::NV];
    static_assert(One::NV == 15, "velocity, stretching, vorticity, 3 enstrophy sums");
#pragma unroll
    for (int v = 0; v < 12; ++v) full[v] = acc[v];
    full[12] = full[13] = full[14] = splat<V>(0.0);
    One::pair(t, full, s, nullptr, 0);
#pragma unroll
    for (int v = 0; v < 12; ++v) acc[v] = full[v];
    acc[12] = fma(t.ax, full[12], fma(t.ay, full[13], fma(t.az, full[14], acc[12])));
  }
};

// Adjoint of the right-hand side (u, S [+ P]) (OpRhsVjp), both sides of the pair, on the
// 160-byte adjoint record.  The gather form of OpRhsVjp already visits each pair in both
// roles for its target k; the scalars it builds (E, D, the kernel derivatives) are symmetric
// under k <-> l, so seen from particle l (r -> -r, w -> -w, ds -> -ds, dp unchanged):
//   xbar_l  += -(cr r + f dp w + f d ds)                   (minus the target's term)
//   abar_l  += -(g (r x u'_k + m_k) + f dp (r x a_k))
//   dL/ds_l += sd,   G_a(l) += g a_k,   G_u(l) += g u'_k
// (the G_a, G_u cross products and G_a x s'_l are applied by the same finalize pass).  About
// 128 FP32 lane-ops per unordered pair against 2 x 100 for the gather.  The source lane
// carries 16 values (position, core, strength, u', s', m); slot VJ_NU stays empty.
// With PSE the exchange scalar Q = nu'_k s'_k.(a_l - a_k) + nu'_l s'_l.(a_k - a_l) is
// symmetric too, and particle l takes dL/dnu'_l += k s'_l.(a_k - a_l), sum k and
// sum k nu'_k s'_k; the lane carries nu' as a 17th value.  The 18 sums fit two targets per
// lane (VPM_ROTGP_P).
template <bool REFINE, bool PSE>
struct OpRhsVjpBoth {
  using V = float2;
  using Record = RecG<float2>;
  using OneSided = OpRhsVjp<float2, REFINE, PSE>;
  struct TgtT : TgtG<float2> {
    float2 mx, my, mz;  // m_k = a_k x s'_k
  };
  using SrcT = SrcG<float2>;
  struct Lane {
    float x, y, z, s, ax, ay, az, ux, uy, uz, gx, gy, gz, mx, my, mz, nu;  // nu: 105 nu
  };
  static constexpr int kLaneValues = PSE ? 17 : 16;  // values that move around the warp
  static constexpr int NV = OneSided::NV;
  static constexpr int kP = PSE ? VPM_ROTGP_P : VPM_ROTG_P;
  static constexpr int kMinBlocks = PSE ? VPM_ROTGP_MINB : VPM_ROTG_MINB;
  static constexpr int kUnroll = PSE ? VPM_ROTGP_UNROLL : VPM_ROTG_UNROLL;
  static constexpr int kSrcWindow = VPM_ROTG_SRC_WINDOW;
  static constexpr int kTgtWindow = 32;
  static constexpr int kTgtWindowShort = 0;
  __device__ __forceinline__ static constexpr bool short_fold(int) { return false; }
  static constexpr int kTgtWindowLong = 0;
  __device__ __forceinline__ static constexpr bool long_fold(int) { return false; }
  static constexpr int kSymFrom = NV;
  static constexpr int kJBufs = 2;
  static constexpr bool kFP64 = false;
  static constexpr bool kUniformCore = false;
  __device__ __forceinline__ static void uniform_core(TgtT&, const Record*) {}

  __device__ __forceinline__ static Lane load_lane(const Record* rec, int64_t j, int64_t n) {
    if (j < n) {
      const float4* p = reinterpret_cast<const float4*>(rec + j);
      const float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2), d = __ldg(p + 3),
                   e = __ldg(p + 4), f = __ldg(p + 5), g = __ldg(p + 6), h = __ldg(p + 7),
                   i = __ldg(p + 8);
      return Lane{a.x, a.z, b.x, b.z, c.x, c.z, d.x, e.x, e.z,
                  f.x, g.x, g.z, h.x, f.z, h.z, i.x, d.z};
    }
    return Lane{kRotFar, kRotFar, kRotFar, 1.f, 0.f, 0.f, 0.f, 0.f, 0.f,
                0.f,     0.f,     0.f,     0.f, 0.f, 0.f, 0.f, 0.f};
  }
  __device__ __forceinline__ static void shuffle(Lane& c, int src_lane) {
    float* v = reinterpret_cast<float*>(&c);
#pragma unroll
    for (int q = 0; q < kLaneValues; ++q) v[q] = __shfl_sync(0xffffffffu, v[q], src_lane);
  }
  __device__ __forceinline__ static SrcT broadcast(const Lane& c) {
    const auto b = [](float v) { return make_float2(v, v); };
    return SrcT{b(c.x),  b(c.y),  b(c.z),  b(c.s),  b(c.ax), b(c.ay),
                b(c.az), b(PSE ? c.nu : 0.f),       b(c.ux), b(c.uy), b(c.uz),
                b(c.gx), b(c.gy), b(c.gz), b(c.mx), b(c.my), b(c.mz)};
  }
  __device__ __forceinline__ static TgtT target(const Record* const* r) {
    TgtT t;
    static_cast<TgtG<float2>&>(t) = make_tgtg(r);
    t.mx = make_float2(r[0]->mx.x, r[1]->mx.x);
    t.my = make_float2(r[0]->my.x, r[1]->my.x);
    t.mz = make_float2(r[0]->mz.x, r[1]->mz.x);
    return t;
  }
  // diagonal tiles: the gather operator, with the pair k == l excluded by index
  __device__ __forceinline__ static void diag(const TgtT& t, V* acc, const SrcT& s,
                                              const int64_t* ti, int64_t j) {
    OneSided::pair(t, acc, s, ti, j);
  }
  __device__ __forceinline__ static constexpr bool carried(int v) { return PSE || v != VJ_NU; }

  __device__ __forceinline__ static void pair2(const TgtT& t, V* acc, V* jv, const SrcT& s) {
    const V rx = t.x - s.x, ry = t.y - s.y, rz = t.z - s.z;
    const V sg = fma(s.s, splat<V>(0.5), t.hs);
    const V s2 = sg * sg;
    const V x = fma(rx, rx, fma(ry, ry, fma(rz, rz, s2)));
    const V y = rsqrt_lane<REFINE>(x);
    const V y2 = y * y;
    const V y5 = (y2 * y2) * y;
    const V y7 = y5 * y2;
    const V y9 = y7 * y2;
    const V s3 = s2 * sg;
    const V t1 = fma(splat<V>(1.5), s2, x);
    const V g = t1 * y5;
    const V t2 = t1 + s2;
    const V f = splat<V>(3.0) * (t2 * y7);
    const V gs = splat<V>(-7.5) * (s3 * y7);           // dg/ds
    const V f2r = splat<V>(-15.0) * ((t2 + s2) * y9);  // 2 df/dr^2
    const V fs = splat<V>(-52.5) * (s3 * y9);          // df/ds
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
    V cr = fma(f2r, D, -(f * E));  // 2 dg/dr^2 E + 2 df/dr^2 D  (-2 dg/dr^2 = f)
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
      // source side (negated when stored): k s'_l.(a_k - a_l) = -k qS, sum k, sum k nu'_k s'_k
      jv[VJ_NU] = fma(k, qS, jv[VJ_NU]);
      jv[VJ_K] = jv[VJ_K] - k;
      const V knt = k * t.nu;
      jv[VJ_KS + 0] = fma(-knt, t.gx, jv[VJ_KS + 0]);
      jv[VJ_KS + 1] = fma(-knt, t.gy, jv[VJ_KS + 1]);
      jv[VJ_KS + 2] = fma(-knt, t.gz, jv[VJ_KS + 2]);
    }
    const V fdp = f * dp;
    const V fd = f * d;
    const V px = fma(cr, rx, fma(fdp, wx, fd * dsx));
    const V py = fma(cr, ry, fma(fdp, wy, fd * dsy));
    const V pz = fma(cr, rz, fma(fdp, wz, fd * dsz));
    acc[VJ_X + 0] = acc[VJ_X + 0] + px;
    acc[VJ_X + 1] = acc[VJ_X + 1] + py;
    acc[VJ_X + 2] = acc[VJ_X + 2] + pz;
    acc[VJ_S] = acc[VJ_S] + sd;
    acc[VJ_GA + 0] = fma(g, s.ax, acc[VJ_GA + 0]);
    acc[VJ_GA + 1] = fma(g, s.ay, acc[VJ_GA + 1]);
    acc[VJ_GA + 2] = fma(g, s.az, acc[VJ_GA + 2]);
    acc[VJ_GU + 0] = fma(g, s.ux, acc[VJ_GU + 0]);
    acc[VJ_GU + 1] = fma(g, s.uy, acc[VJ_GU + 1]);
    acc[VJ_GU + 2] = fma(g, s.uz, acc[VJ_GU + 2]);
    const V nx = fma(ry, s.uz, -(rz * s.uy)) - s.mx;  // r x u'_l - m_l
    const V ny = fma(rz, s.ux, -(rx * s.uz)) - s.my;
    const V nz = fma(rx, s.uy, -(ry * s.ux)) - s.mz;
    acc[VJ_A + 0] = fma(g, nx, fma(fdp, clx, acc[VJ_A + 0]));
    acc[VJ_A + 1] = fma(g, ny, fma(fdp, cly, acc[VJ_A + 1]));
    acc[VJ_A + 2] = fma(g, nz, fma(fdp, clz, acc[VJ_A + 2]));
    // source side, every sum with the opposite sign (negated when it is stored)
    jv[VJ_X + 0] = jv[VJ_X + 0] + px;
    jv[VJ_X + 1] = jv[VJ_X + 1] + py;
    jv[VJ_X + 2] = jv[VJ_X + 2] + pz;
    jv[VJ_S] = jv[VJ_S] - sd;
    jv[VJ_GA + 0] = fma(-g, t.ax, jv[VJ_GA + 0]);
    jv[VJ_GA + 1] = fma(-g, t.ay, jv[VJ_GA + 1]);
    jv[VJ_GA + 2] = fma(-g, t.az, jv[VJ_GA + 2]);
    jv[VJ_GU + 0] = fma(-g, t.ux, jv[VJ_GU + 0]);
    jv[VJ_GU + 1] = fma(-g, t.uy, jv[VJ_GU + 1]);
    jv[VJ_GU + 2] = fma(-g, t.uz, jv[VJ_GU + 2]);
    const V qx = fma(ry, t.uz, -(rz * t.uy)) + t.mx;  // r x u'_k + m_k
    const V qy = fma(rz, t.ux, -(rx * t.uz)) + t.my;
    const V qz = fma(rx, t.uy, -(ry * t.ux)) + t.mz;
    jv[VJ_A + 0] = fma(g, qx, fma(fdp, ckx, jv[VJ_A + 0]));
    jv[VJ_A + 1] = fma(g, qy, fma(fdp, cky, jv[VJ_A + 1]));
    jv[VJ_A + 2] = fma(g, qz, fma(fdp, ckz, jv[VJ_A + 2]));
  }
};

// The tile pair of this CTA: tiles I (targets) and J (sources), the accumulator sets its
// target and source sides add into, and (DIAG) the part h of the diagonal tile's sources.
// False for the CTAs past the middle diagonal's nt - k tile pairs.
//
// Two sets per diagonal pair: the first diagonal's target rows [0, nt - k) and the second's
// source rows [nt - k, nt) share set 2q; the first's source rows [k, nt) and the second's
// target rows [0, k) share set 2q + 1.  The row ranges in a set are disjoint and each tile
// appears once per role, so every element still has one writer per launch.
template <bool DIAG>
__device__ __forceinline__ bool rot_block_pair(const RotArgs& a, int& I, int& J, int& set_i,
                                               int& set_j, int& h) {
  h = 0;
  if (DIAG) {
    const int t = blockIdx.x / kRotDiagSplit;
    h = blockIdx.x - t * kRotDiagSplit;
    I = J = a.tile0 + t;
    set_i = a.set0 + h;  // each part into its own set: one writer per element
    set_j = a.set0 + h;
    return true;
  }
  const int q = blockIdx.x / a.nt, r = blockIdx.x - q * a.nt;
  const int k = a.k0 + q, n1 = a.nt - k;
  if (r < n1) {
    I = r;
    J = r + k;
    set_i = 2 * q;
    set_j = 2 * q + 1;
    return true;
  }
  if (n1 > k) {
    I = r - n1;
    J = I + n1;
    set_i = 2 * q + 1;
    set_j = 2 * q;
    return true;
  }
  return false;  // k == nt - k: the diagonal has only nt - k tile pairs
}

template <class Op, bool DIAG>
__global__ void __launch_bounds__(kRotThreads, Op::kMinBlocks)
rot_sweep_kernel(const RotArgs a) {
  using Record = typename Op::Record;
  using Lane = typename Op::Lane;
  constexpr int NV = Op::NV;
  constexpr int P = Op::kP;
  constexpr int T = rot_tile<Op>();
  constexpr int WT = kRotWarps * 32;  // source slots of a batch: [warp][source lane]
  constexpr int SW = Op::kSrcWindow;
  constexpr int TW = Op::kTgtWindow;
  static_assert(32 % SW == 0, "the source window divides the 32 steps of a batch");
  static_assert(32 % TW == 0 && TW % SW == 0, "target windows are whole source windows");
  constexpr int TWS = Op::kTgtWindowShort;
  static_assert(TWS == 0 || (TW % TWS == 0 && TWS % SW == 0),
                "short target windows divide the target window and are whole source windows");
  constexpr int TWL = Op::kTgtWindowLong;
  static_assert(TWL == 0 || TWL % 32 == 0, "long target windows are whole batches");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  double* car = reinterpret_cast<double*>(smem_raw);  // [NV][T]
  // [2][NV][WT]: each warp's packed source-side sums of the current batch, per source
  constexpr int NJ = Op::kSymFrom;  // values with a source side: the first NJ
  float2* jbuf = reinterpret_cast<float2*>(smem_raw + size_t(T) * NV * sizeof(double));
  const Record* rec = static_cast<const Record*>(a.rec);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  int I, J, set_i, set_j, h;
  if (!rot_block_pair<DIAG>(a, I, J, set_i, set_j, h)) return;
  // sources: the whole tile J, or (DIAG) part h of the diagonal tile
  constexpr int TS = DIAG ? T / kRotDiagSplit : T;
  static_assert(TS % 32 == 0, "source ranges are whole batches");
  const int64_t i0 = int64_t(I) * T, j0 = int64_t(J) * T + int64_t(h) * TS;
  const int cnt = int((a.n - j0 < TS) ? (a.n - j0 > 0 ? a.n - j0 : 0) : TS);

  for (int q = tid; q < T * NV; q += kRotThreads) car[q] = 0.0;

  // this lane's targets: packed lane p holds warp * 64P + 64p + lane + {0, 32}
  int lt[2 * P];
  typename Op::TgtT tg[P];
#pragma unroll
  for (int p = 0; p < P; ++p) {
    lt[2 * p] = warp * 64 * P + p * 64 + lane;
    lt[2 * p + 1] = lt[2 * p] + 32;
    const int64_t t0 = i0 + lt[2 * p], t1 = i0 + lt[2 * p + 1];
    // targets past n (a copy of the last record) occur only in the diagonal tiles: a tile
    // pair has I < J <= nt - 1, so its target tile is whole; the diagonal tiles are one-sided,
    // so those copies add to no source, and their own sums are never stored
    const Record* recs[2] = {rec + (t0 < a.n ? t0 : a.n - 1), rec + (t1 < a.n ? t1 : a.n - 1)};
    tg[p] = Op::target(recs);
    if constexpr (Op::kUniformCore) Op::uniform_core(tg[p], rec);
  }
  float2 acc[P][NV];
#pragma unroll
  for (int p = 0; p < P; ++p)
#pragma unroll
    for (int v = 0; v < NV; ++v) acc[p][v] = make_float2(0.f, 0.f);
  __syncthreads();  // carries zeroed

  // target side: the FP32 window sums of the values take(v) selects into the FP64 carries
  // (each thread its own rows), and those sums start again from zero
  auto fold_targets = [&](auto take) {
#pragma unroll
    for (int p = 0; p < P; ++p) {
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        if (!take(v)) continue;
        if (DIAG && v >= NJ) {
          // a symmetric sum taken once per unordered pair elsewhere: the diagonal tiles
          // visit every ordered pair, so they count half (the finalize doubles the sum)
          car[v * T + lt[2 * p]] += 0.5 * double(acc[p][v].x);
          car[v * T + lt[2 * p + 1]] += 0.5 * double(acc[p][v].y);
        } else {
          car[v * T + lt[2 * p]] += double(acc[p][v].x);
          car[v * T + lt[2 * p + 1]] += double(acc[p][v].y);
        }
        acc[p][v] = make_float2(0.f, 0.f);
      }
    }
  };

  const int nb = (cnt + 31) / 32;
  Lane nxt = Op::load_lane(rec, j0 + lane, j0 + cnt);
  for (int b = 0; b < nb; ++b) {
    Lane cur = nxt;  // the source this lane holds at step 0
    if (b + 1 < nb) nxt = Op::load_lane(rec, j0 + (b + 1) * 32 + lane, j0 + cnt);
    float2 jv[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) jv[v] = make_float2(0.f, 0.f);
    float2* jb = jbuf + (b % Op::kJBufs) * (NJ * WT);
    const int src_lane = (lane + 1) & 31;
    for (int w = 0; w < 32 / SW; ++w) {
#pragma unroll Op::kUnroll
      for (int st = 0; st < SW; ++st) {
        const int step = w * SW + st;
        const typename Op::SrcT src = Op::broadcast(cur);
#pragma unroll
        for (int p = 0; p < P; ++p) {
          if constexpr (DIAG) {
            // at this step the lane holds source b * 32 + ((lane + step) mod 32) of the tile
            const int64_t ti[2] = {i0 + lt[2 * p], i0 + lt[2 * p + 1]};
            Op::diag(tg[p], acc[p], src, ti, j0 + b * 32 + ((lane + step) & 31));
          } else {
            Op::pair2(tg[p], acc[p], jv, src);
          }
        }
        // pass the source one lane down (lane l now holds what lane l+1 held); its sums move
        // with it, except after a window's last step, where they are stored instead
        Op::shuffle(cur, src_lane);
        if constexpr (!DIAG) {
          if (st != SW - 1) {
#pragma unroll
            for (int v = 0; v < NV; ++v) {
              if (Op::carried(v)) {
                jv[v].x = __shfl_sync(0xffffffffu, jv[v].x, src_lane);
                jv[v].y = __shfl_sync(0xffffffffu, jv[v].y, src_lane);
              }
            }
          }
        }
      }
      if constexpr (!DIAG) {
        // end of a window: the lane holds the sums of the source it met at the window's last
        // step, (lane + step) mod 32; add them into that source's slot (the lanes of a warp
        // hold distinct sources) and start the next window from zero
        const int slot = warp * 32 + ((lane + (w + 1) * SW - 1) & 31);
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          if (Op::carried(v)) {
            float2* e = jb + v * WT + slot;
            *e = (w == 0) ? jv[v] : (*e + jv[v]);
            jv[v] = make_float2(0.f, 0.f);
          }
        }
      }
      const int done = (w + 1) * SW;  // steps of this batch done
      const bool at_full = done % TW == 0;
      const bool at_short = TWS > 0 && done % (TWS > 0 ? TWS : 1) == 0;
      const bool at_long = TWL > 0 && (b * 32 + done) % (TWL > 0 ? TWL : 1) == 0;
      if (at_full || at_short || at_long)
        fold_targets([&](int v) {
          return (TWL > 0 && Op::long_fold(v))    ? at_long
                 : (TWS > 0 && Op::short_fold(v)) ? at_short
                                                  : at_full;
        });
    }
    if constexpr (!DIAG) {
      __syncthreads();  // the batch's source-side sums are complete
      const int nsrc = (cnt - b * 32 < 32) ? cnt - b * 32 : 32;
      for (int q = tid; q < 32 * NJ; q += kRotThreads) {
        const int v = q >> 5, jj = q & 31;  // consecutive threads: consecutive sources
        if (jj >= nsrc || !Op::carried(v)) continue;
        // both packed halves of every warp's sum, in FP64, in a fixed order
        double sum = 0.0;
#pragma unroll
        for (int w = 0; w < kRotWarps; ++w) {
          const float2 e = jb[v * WT + w * 32 + jj];
          sum += double(e.x);
          sum += double(e.y);
        }
        // the only writer of this element in this launch, so the fire-and-forget reduction
        // adds in a fixed order (launch order) and the thread does not wait for the load
        atomicAdd(&a.acc[(int64_t(set_j) * NV + v) * a.n + (j0 + b * 32 + jj)], -sum);
      }
      // one buffer: every thread has read it before the next batch writes it
      if constexpr (Op::kJBufs == 1) __syncthreads();
    }
  }
  // long windows span batches: what the last one left
  if constexpr (TWL > 0) fold_targets([](int v) { return Op::long_fold(v); });
  __syncthreads();
  for (int q = tid; q < T * NV; q += kRotThreads) {
    const int v = q / T, t = q - v * T;
    if (i0 + t < a.n) atomicAdd(&a.acc[(int64_t(set_i) * NV + v) * a.n + (i0 + t)], car[q]);
  }
}

// ---- FP64: the fused sum on the both-sides schedule ------------------------------------------
// The exact (FP64) form of the fused velocity + stretching sum (and of the velocity and PSE
// sums) with each unordered pair evaluated once for both particles: the pair terms are the
// FP32 operators' pair2 in double
// (CUDA's rsqrt(double), as the one-sided FP64 sweep), and they differ from the one-sided
// sweep's only in rounding (the triple product a_i . (r x a_j) in place of
// r . ((a_j - a_i) x a_i)); the sums are FP64 throughout, so there are no windows and no
// carries: each lane keeps R = 2 kP targets' sums in registers, and the source's sums travel
// with it around the warp for the 32 steps of a batch.  Tiles, sets and launches are the
// FP32 schedule's (rot_tile, rot_block_pair, the RotSweep planner).
#ifndef VPM_ROT64_P
#define VPM_ROT64_P 2  // R = 4 FP64 targets per lane, 512-particle tiles
#endif
#ifndef VPM_ROT64_MINB
#define VPM_ROT64_MINB 2
#endif

// Both32: the FP32 both-sides operator whose pair2 (a template in the lane type) gives the
// pair terms; OneSided64: the one-sided FP64 operator of the diagonal tiles.
template <class Both32, class OneSided64, bool UC, int MINB = VPM_ROT64_MINB,
          int P = VPM_ROT64_P>
struct OpBoth64 {
  using V = double;
  using Record = Rec<double>;
  using OneSided = OneSided64;
  using TgtT = Tgt<double>;
  using SrcT = Src<double>;
  static constexpr bool kFP64 = true;
  static constexpr int NV = Both32::NV;
  static constexpr int kP = P;  // rot_tile: 64 kP warps = 32 R warps
  static constexpr int kMinBlocks = MINB;
  // values from kSymFrom on are taken once per unordered pair on the target side only
  static constexpr int kSymFrom = Both32::kSymFrom;
  static constexpr bool kUniformCore = UC;
  __device__ __forceinline__ static SrcT load(const Record* rec, int64_t j, int64_t n) {
    if (j < n) return load_src<double>(rec[j]);
    // far and without strength: r^2 = 1e220 stays finite and y^3 = 1e-330 underflows to 0,
    // so the pair adds exactly nothing on either side
    return SrcT{1e110, 1e110, 1e110, 1.0, 0.0, 0.0, 0.0, 0.0};
  }
  __device__ __forceinline__ static void shuffle(SrcT& c, int src_lane) {
    c.x = __shfl_sync(0xffffffffu, c.x, src_lane);
    c.y = __shfl_sync(0xffffffffu, c.y, src_lane);
    c.z = __shfl_sync(0xffffffffu, c.z, src_lane);
    if constexpr (!UC) c.s = __shfl_sync(0xffffffffu, c.s, src_lane);
    c.ax = __shfl_sync(0xffffffffu, c.ax, src_lane);
    c.ay = __shfl_sync(0xffffffffu, c.ay, src_lane);
    c.az = __shfl_sync(0xffffffffu, c.az, src_lane);
  }
  __device__ __forceinline__ static void uniform_core(TgtT& t, const Record* rec) {
    const double sc = rec[0].s, s2 = sc * sc;
    t.sc = sc;
    t.s2c = s2;
    t.s4c = s2 * s2;
  }
  __device__ __forceinline__ static void pair2(const TgtT& t, double* acc, double* jv,
                                               const SrcT& s) {
    Both32::pair2(t, acc, jv, s);
  }
  __device__ __forceinline__ static void diag(const TgtT& t, double* acc, const SrcT& s) {
    if constexpr (Both32::kCustomDiag)
      Both32::diag(t, acc, s, nullptr, 0);
    else
      OneSided::pair(t, acc, s, nullptr, 0);
  }
};
template <bool UC>
using OpVelStretchBoth64 =
    OpBoth64<OpVelStretchBoth<false, UC>, OpVelStretch<double, false, UC>, UC>;
// the three-sum operators fit three CTAs per SM
template <bool UC>
using OpVelBoth64 = OpBoth64<OpVelBoth<false, UC>, OpVel<double, false, UC>, UC, 3>;
template <bool UC>
using OpPseBoth64 = OpBoth64<OpPseBoth<false, UC>, OpPse<double, false, UC>, UC, 3>;
// the LES step's 13 sums: two FP64 targets per lane (256-particle tiles)
template <bool UC>
using OpLesStepBoth64 =
    OpBoth64<OpLesStepBoth<false, UC>, OpLesStep<double, false, UC>, UC, 2, 1>;

template <class Op, bool DIAG>
__global__ void __launch_bounds__(kRotThreads, Op::kMinBlocks)
rot64_sweep_kernel(const RotArgs a) {
  using Record = typename Op::Record;
  constexpr int NV = Op::NV;
  constexpr int R = 2 * Op::kP;  // targets per lane
  constexpr int T = rot_tile<Op>();
  constexpr int WT = kRotWarps * 32;
  static_assert(T == R * WT, "a tile is the CTA's lanes times their targets");
  constexpr int NJ = Op::kSymFrom;  // values with a source side: the first NJ
  extern __shared__ __align__(128) unsigned char smem_raw[];
  double* jbuf = reinterpret_cast<double*>(smem_raw);  // [NJ][WT]
  const Record* rec = static_cast<const Record*>(a.rec);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  int I, J, set_i, set_j, h;
  if (!rot_block_pair<DIAG>(a, I, J, set_i, set_j, h)) return;
  constexpr int TS = DIAG ? T / kRotDiagSplit : T;
  static_assert(TS % 32 == 0, "source ranges are whole batches");
  const int64_t i0 = int64_t(I) * T, j0 = int64_t(J) * T + int64_t(h) * TS;
  const int cnt = int((a.n - j0 < TS) ? (a.n - j0 > 0 ? a.n - j0 : 0) : TS);

  // this lane's targets: warp * 32 R + 32 r + lane
  typename Op::TgtT tg[R];
  int64_t ti[R];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    ti[r] = i0 + warp * 32 * R + r * 32 + lane;
    // past n only in the (one-sided) diagonal tiles, as in rot_sweep_kernel
    const Record* rp = rec + (ti[r] < a.n ? ti[r] : a.n - 1);
    tg[r] = make_tgt(&rp);
    if constexpr (Op::kUniformCore) Op::uniform_core(tg[r], rec);
  }
  double acc[R][NV];
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int v = 0; v < NV; ++v) acc[r][v] = 0.0;

  const int nb = (cnt + 31) / 32;
  const int src_lane = (lane + 1) & 31;
  typename Op::SrcT nxt = Op::load(rec, j0 + lane, j0 + cnt);
  for (int b = 0; b < nb; ++b) {
    typename Op::SrcT cur = nxt;  // the source this lane holds at step 0
    if (b + 1 < nb) nxt = Op::load(rec, j0 + (b + 1) * 32 + lane, j0 + cnt);
    double jv[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) jv[v] = 0.0;
#pragma unroll 2
    for (int st = 0; st < 32; ++st) {
#pragma unroll
      for (int r = 0; r < R; ++r) {
        if constexpr (DIAG)
          Op::diag(tg[r], acc[r], cur);
        else
          Op::pair2(tg[r], acc[r], jv, cur);
      }
      // the source and its sums one lane down; after 32 steps both are back in their lane
      Op::shuffle(cur, src_lane);
      if constexpr (!DIAG) {
#pragma unroll
        for (int v = 0; v < NJ; ++v) jv[v] = __shfl_sync(0xffffffffu, jv[v], src_lane);
      }
    }
    if constexpr (!DIAG) {
      // the warps' sums of source b * 32 + lane, added over the warps in a fixed order
#pragma unroll
      for (int v = 0; v < NJ; ++v) jbuf[v * WT + warp * 32 + lane] = jv[v];
      __syncthreads();
      const int nsrc = (cnt - b * 32 < 32) ? cnt - b * 32 : 32;
      for (int q = tid; q < 32 * NJ; q += kRotThreads) {
        const int v = q >> 5, jj = q & 31;
        if (jj >= nsrc) continue;
        double sum = 0.0;
#pragma unroll
        for (int w = 0; w < kRotWarps; ++w) sum += jbuf[v * WT + w * 32 + jj];
        // the only writer of this element in this launch (non-returning, fixed order)
        atomicAdd(&a.acc[(int64_t(set_j) * NV + v) * a.n + (j0 + b * 32 + jj)], -sum);
      }
      __syncthreads();  // jbuf is read before the next batch writes it
    }
  }
#pragma unroll
  for (int r = 0; r < R; ++r) {
    if (ti[r] < a.n) {
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        // a symmetric sum taken once per unordered pair elsewhere: the diagonal tiles visit
        // every ordered pair, so they count half (the finalize doubles the sum)
        const double w = (DIAG && v >= NJ) ? 0.5 * acc[r][v] : acc[r][v];
        atomicAdd(&a.acc[(int64_t(set_i) * NV + v) * a.n + ti[r]], w);
      }
    }
  }
}

}  // namespace vpm
