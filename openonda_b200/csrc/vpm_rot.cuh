// vpm_rot.cuh -- both-sides sweeps of the FP32-compensated self sums (fused velocity +
// stretching, velocity, PSE, the LES step sums), with the source side carried around the warp
// in registers.
//
// The pair terms of (i <- j) and (j <- i) share r^2, the core, the rsqrt and the kernel
// values.  Seen from particle j, with r = x_i - x_j as computed for target i:
//   U_j += -g (r x a_i),   A_j += -g (a_j - a_i),   B_j += -h r,   h = f a_i . (r x a_j),
//   P_j += -k (a_j - a_i)   (PSE; nu_j is applied per particle in the finalize),
// so one evaluation of an unordered pair costs 53 FP32 lane-ops instead of 2 x 38 for the
// fused sum, 31 instead of 2 x 22 for the velocity, 24 instead of 2 x 21 for PSE and 69-82
// instead of 2 x 52-56 for the four LES step sums.
//
// Warp layout: each lane holds four targets (two packed FP32x2 lanes) and one source of the
// current batch of 32 (read from L2, the next batch prefetched).  In 32 steps every lane meets
// every source of the batch: after each step the sources and their source-side accumulators
// move one lane down (__shfl_sync), so after the 32nd step each source is back in its lane
// with its sums over the warp's 128 targets.  Warp shuffles are the second-scarcest resource
// here (about one per two clocks per SM); four targets per lane keep them at 25 per 256
// ordered pairs for the fused sum.  The source-side sums are then added over the CTA's warps
// in FP64 (fixed order) and added into the accumulator of the source particle with a
// non-returning atomic.
//
// Tile-pair schedule: particles form nt tiles of T = 128 * WARPS.  A CTA owns one tile pair
// (I, J), I < J.  Diagonal pair q of a launch is J - I = k (accumulator sets 4q / 4q+1 for
// the target / source side) together with J - I = nt - k (sets 4q+2 / 4q+3): every
// accumulator element has one writer per launch and the launches run in stream order, so the
// atomic additions happen in a fixed order and the result is deterministic.  A launch runs m
// consecutive diagonal pairs (m chosen so that its m * nt CTAs fill whole waves); launch 0
// runs the diagonal tiles (I, I) one-sided into set 0.  The finalize pass sums the 4m sets in
// order.
//
// Accumulation: target side in FP32 per batch of 32 sources, folded into FP64 carries held in
// shared memory; source side in FP32 over the warp's 128 targets (each half of the packed
// accumulator sums 64 terms), then FP64 across warps and tile pairs.
#pragma once

#include "vpm_sweep.cuh"

namespace vpm {

// Build parameters: warps per CTA, resident CTAs per SM the registers are sized for (fused
// sum VPM_ROT_MINB, three-sum operators VPM_ROT3_MINB, LES step VPM_ROT15_MINB: its 77 KB of
// shared memory allow two), unroll of the 32 steps.
#ifndef VPM_ROT_WARPS
#define VPM_ROT_WARPS 4
#endif
#ifndef VPM_ROT_MINB
#define VPM_ROT_MINB 3
#endif
#ifndef VPM_ROT3_MINB
#define VPM_ROT3_MINB 3
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

// Fused velocity + stretching, both sides of the pair (FP32x2 lanes).
template <bool REFINE, bool UC>
struct OpVelStretchBoth {
  using V = float2;
  using OneSided = OpVelStretch<float2, REFINE, UC>;
  static constexpr int NV = 9;
  static constexpr bool kSrcCore = !UC;  // the pair core needs the source's sigma
  static constexpr int kMinBlocks = VPM_ROT_MINB;
  static constexpr int kUnroll = VPM_ROT_UNROLL;
  __device__ __forceinline__ static void pair2(const Tgt<V>& t, V* acc, V* jv,
                                               const Src<V>& s) {
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
struct OpVelBoth {
  using V = float2;
  using OneSided = OpVel<float2, REFINE, UC>;
  static constexpr int NV = 3;
  static constexpr bool kSrcCore = !UC;
  static constexpr int kMinBlocks = VPM_ROT3_MINB;
  static constexpr int kUnroll = VPM_ROT_UNROLL;
  __device__ __forceinline__ static void pair2(const Tgt<V>& t, V* acc, V* jv,
                                               const Src<V>& s) {
    const V rx = t.x - s.x, ry = t.y - s.y, rz = t.z - s.z;
    V sg, s2;
    pair_core<UC>(t, s, sg, s2);
    const V x = fma(rx, rx, fma(ry, ry, fma(rz, rz, s2)));
    const V y = rsqrt_lane<REFINE>(x);
    const V y2 = y * y;
    const V y5 = (y2 * y2) * y;
    const V g = fma(splat<V>(1.5), s2, x) * y5;
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
struct OpPseBoth {
  using V = float2;
  using OneSided = OpPse<float2, REFINE, UC>;
  static constexpr int NV = 3;
  static constexpr bool kSrcCore = !UC;
  static constexpr int kMinBlocks = VPM_ROT3_MINB;
  static constexpr int kUnroll = VPM_ROT_UNROLL;
  __device__ __forceinline__ static void pair2(const Tgt<V>& t, V* acc, V* jv,
                                               const Src<V>& s) {
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
// Vorticity and enstrophy are symmetric sums, so their source-side terms enter negated (the
// stored value is negated once more).  Pairs with r^2 <= 1e-8 add no vorticity.  69 FP32
// lane-ops per unordered pair with uniform cores, about 82 without (one-sided: 2 x 52,
// 2 x 56).  255 registers per thread: two CTAs per SM, step loop unrolled 2.
template <bool REFINE, bool UC>
struct OpLesStepBoth {
  using V = float2;
  using OneSided = OpLesStep<float2, REFINE, UC>;
  static constexpr int NV = 15;
  static constexpr bool kSrcCore = !UC;
  static constexpr int kMinBlocks = VPM_ROT15_MINB;
  static constexpr int kUnroll = VPM_ROT15_UNROLL;
  __device__ __forceinline__ static void pair2(const Tgt<V>& t, V* acc, V* jv,
                                               const Src<V>& s) {
    const V rx = t.x - s.x, ry = t.y - s.y, rz = t.z - s.z;
    V sg, s2;
    pair_core<UC>(t, s, sg, s2);
    const V r2 = fma(rx, rx, fma(ry, ry, rz * rz));
    const V x = r2 + s2;
    const V y = rsqrt_lane<REFINE>(x);
    const V y2 = y * y;
    const V y3 = y2 * y;
    const V y5 = y3 * y2;
    const V t1 = fma(splat<V>(1.5), s2, x);
    const V g = t1 * y5;
    const V f = (t1 + s2) * (y5 * y2);
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
    const float eps = float(kRefEps);
    V ki, kj;
    if constexpr (UC) {
      const V y7 = (y3 * y3) * y;
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
    ki = make_float2(r2.x > eps ? ki.x : 0.f, r2.y > eps ? ki.y : 0.f);
    kj = make_float2(r2.x > eps ? kj.x : 0.f, r2.y > eps ? kj.y : 0.f);
    acc[9] = fma(ki, s.ax, acc[9]);
    acc[10] = fma(ki, s.ay, acc[10]);
    acc[11] = fma(ki, s.az, acc[11]);
    jv[9] = fma(-kj, t.ax, jv[9]);
    jv[10] = fma(-kj, t.ay, jv[10]);
    jv[11] = fma(-kj, t.az, jv[11]);
    // enstrophy filter sum (pair core)
    const V ke = fma(splat<V>(2.2), s2, x) * y3;
    acc[12] = fma(ke, s.ax, acc[12]);
    acc[13] = fma(ke, s.ay, acc[13]);
    acc[14] = fma(ke, s.az, acc[14]);
    jv[12] = fma(-ke, t.ax, jv[12]);
    jv[13] = fma(-ke, t.ay, jv[13]);
    jv[14] = fma(-ke, t.az, jv[14]);
  }
};

struct RotArgs {
  const Rec<float2>* rec;  // packed records of all n particles
  int64_t n;
  int nt;       // tiles of kRotTile particles
  int k0;       // first diagonal of this launch (0 = the diagonal tiles)
  double* acc;  // accumulators [sets][NV][n]
};

constexpr int kRotWarps = VPM_ROT_WARPS;
constexpr int kRotThreads = 32 * kRotWarps;
constexpr int kRotTile = 128 * kRotWarps;  // four targets per lane (two packed FP32x2 lanes)
constexpr float kRotFar = 1e15f;           // position of the padding sources: g, f underflow

constexpr size_t rot_smem_bytes(int nv) {
  return size_t(kRotTile) * nv * sizeof(double) +          // target-side FP64 carries
         size_t(2) * kRotWarps * 32 * nv * sizeof(float);  // source-side sums, double-buffered
}

struct RotSrc {
  float x, y, z, s, ax, ay, az;
};

// Source j of the packed records (j < n), or a padding source far away with no strength.
__device__ __forceinline__ RotSrc rot_load_src(const Rec<float2>* rec, int64_t j, int64_t n) {
  if (j < n) {
    const float4* p = reinterpret_cast<const float4*>(rec + j);
    const float4 a = __ldg(p), b = __ldg(p + 1), c = __ldg(p + 2), d = __ldg(p + 3);
    return RotSrc{a.x, a.z, b.x, b.z, c.x, c.z, d.x};
  }
  return RotSrc{kRotFar, kRotFar, kRotFar, 1.f, 0.f, 0.f, 0.f};
}

template <class Op, bool DIAG>
__global__ void __launch_bounds__(kRotThreads, Op::kMinBlocks)
rot_sweep_kernel(const RotArgs a) {
  constexpr int NV = Op::NV;
  constexpr int T = kRotTile;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  double* car = reinterpret_cast<double*>(smem_raw);  // [NV][T]
  float* jbuf = reinterpret_cast<float*>(smem_raw + size_t(T) * NV * sizeof(double));

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  int I, J, set_i, set_j;
  if (DIAG) {
    I = J = blockIdx.x;
    set_i = 0;
    set_j = 0;
  } else {
    const int q = blockIdx.x / a.nt, r = blockIdx.x - q * a.nt;
    const int k = a.k0 + q, n1 = a.nt - k;
    if (r < n1) {
      I = r;
      J = r + k;
      set_i = 4 * q;
      set_j = 4 * q + 1;
    } else if (n1 > k) {
      I = r - n1;
      J = I + n1;
      set_i = 4 * q + 2;
      set_j = 4 * q + 3;
    } else {
      return;  // k == nt - k: the diagonal has only nt - k tile pairs
    }
  }
  const int64_t i0 = int64_t(I) * T, j0 = int64_t(J) * T;
  const int cnt = int((a.n - j0 < T) ? (a.n - j0) : T);

  for (int q = tid; q < T * NV; q += kRotThreads) car[q] = 0.0;

  // this lane's four targets: warp*128 + lane + {0, 32} (first packed lane) and + {64, 96}
  int lt[4];
  typename Op::OneSided::TgtT tg[2];
#pragma unroll
  for (int p = 0; p < 2; ++p) {
    lt[2 * p] = warp * 128 + p * 64 + lane;
    lt[2 * p + 1] = lt[2 * p] + 32;
    const int64_t t0 = i0 + lt[2 * p], t1 = i0 + lt[2 * p + 1];
    const Rec<float2>* recs[2] = {a.rec + (t0 < a.n ? t0 : a.n - 1),
                                  a.rec + (t1 < a.n ? t1 : a.n - 1)};
    tg[p] = make_tgt(recs);
  }
  float2 acc[2][NV];
#pragma unroll
  for (int p = 0; p < 2; ++p)
#pragma unroll
    for (int v = 0; v < NV; ++v) acc[p][v] = make_float2(0.f, 0.f);
  __syncthreads();  // carries zeroed

  const int nb = (cnt + 31) / 32;
  RotSrc nxt = rot_load_src(a.rec, j0 + lane, j0 + cnt);
  for (int b = 0; b < nb; ++b) {
    RotSrc cur = nxt;  // the source this lane holds at step 0
    if (b + 1 < nb) nxt = rot_load_src(a.rec, j0 + (b + 1) * 32 + lane, j0 + cnt);
    float2 jv[NV];
#pragma unroll
    for (int v = 0; v < NV; ++v) jv[v] = make_float2(0.f, 0.f);
    const int src_lane = (lane + 1) & 31;
#pragma unroll Op::kUnroll
    for (int step = 0; step < 32; ++step) {
      const Src<float2> src{make_float2(cur.x, cur.x),   make_float2(cur.y, cur.y),
                            make_float2(cur.z, cur.z),   make_float2(cur.s, cur.s),
                            make_float2(cur.ax, cur.ax), make_float2(cur.ay, cur.ay),
                            make_float2(cur.az, cur.az), make_float2(0.f, 0.f)};
#pragma unroll
      for (int p = 0; p < 2; ++p) {
        if constexpr (DIAG)
          Op::OneSided::pair(tg[p], acc[p], src, nullptr, 0);
        else
          Op::pair2(tg[p], acc[p], jv, src);
      }
      // pass the source (and its sums) one lane down: lane l now holds what lane l+1 held
      cur.x = __shfl_sync(0xffffffffu, cur.x, src_lane);
      cur.y = __shfl_sync(0xffffffffu, cur.y, src_lane);
      cur.z = __shfl_sync(0xffffffffu, cur.z, src_lane);
      if constexpr (Op::kSrcCore) cur.s = __shfl_sync(0xffffffffu, cur.s, src_lane);
      cur.ax = __shfl_sync(0xffffffffu, cur.ax, src_lane);
      cur.ay = __shfl_sync(0xffffffffu, cur.ay, src_lane);
      cur.az = __shfl_sync(0xffffffffu, cur.az, src_lane);
      if constexpr (!DIAG) {
#pragma unroll
        for (int v = 0; v < NV; ++v) {
          jv[v].x = __shfl_sync(0xffffffffu, jv[v].x, src_lane);
          jv[v].y = __shfl_sync(0xffffffffu, jv[v].y, src_lane);
        }
      }
    }
    // target side: this batch's FP32 sums into the FP64 carries (each thread its own rows)
#pragma unroll
    for (int p = 0; p < 2; ++p) {
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        car[v * T + lt[2 * p]] += double(acc[p][v].x);
        car[v * T + lt[2 * p + 1]] += double(acc[p][v].y);
        acc[p][v] = make_float2(0.f, 0.f);
      }
    }
    if constexpr (!DIAG) {
      // after 32 steps lane l holds the sums of source b*32 + l again
      float* jb = jbuf + (b & 1) * (kRotWarps * 32 * NV);
#pragma unroll
      for (int v = 0; v < NV; ++v) jb[(warp * 32 + lane) * NV + v] = jv[v].x + jv[v].y;
      __syncthreads();  // one barrier per batch; jbuf is double-buffered
      const int nsrc = (cnt - b * 32 < 32) ? cnt - b * 32 : 32;
      for (int q = tid; q < nsrc * NV; q += kRotThreads) {
        const int jj = q / NV, v = q - jj * NV;
        double sum = 0.0;
#pragma unroll
        for (int w = 0; w < kRotWarps; ++w) sum += double(jb[(w * 32 + jj) * NV + v]);
        // the only writer of this element in this launch, so the fire-and-forget reduction
        // adds in a fixed order (launch order) and the thread does not wait for the load
        atomicAdd(&a.acc[(int64_t(set_j) * NV + v) * a.n + (j0 + b * 32 + jj)], -sum);
      }
    }
  }
  __syncthreads();
  for (int q = tid; q < T * NV; q += kRotThreads) {
    const int v = q / T, t = q - v * T;
    if (i0 + t < a.n) atomicAdd(&a.acc[(int64_t(set_i) * NV + v) * a.n + (i0 + t)], car[q]);
  }
}

}  // namespace vpm
