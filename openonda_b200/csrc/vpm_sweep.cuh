// vpm_sweep.cuh -- the tiled all-pairs sweep (one kernel template for every operator).
//
// Grid: blockIdx.x = a block of THREADS*R targets, blockIdx.y = one contiguous chunk of
// sources (a "split").  Each thread owns R targets (i = base + r*THREADS + tid) in
// registers.  Source records stream through shared memory in tiles of TILE records:
// one elected thread issues a bulk-async (TMA) copy per tile into a STAGES-deep ring,
// completion is signalled on an mbarrier, and all warps read the tile by broadcast.
//
// Accumulation: in FP64 the partial sums accumulate directly in double.  In FP32 each
// target keeps an FP32 accumulator for a window of CW consecutive sources (32; 16 for the
// stretching operators) and folds it into an FP64 carry at the end of every window (one DADD
// per value per window), so rounding grows only over CW terms and the long sum over N
// sources runs in FP64.  FP32
// targets are processed two at a time with the paired FP32 instructions of sm_100.
//
// Each (split, value, target) partial is written as FP64 to
// partial[(split * NV + v) * m + i]; a finalize pass sums the splits in split order, so
// the result does not depend on scheduling.
#pragma once

#include "vpm_pairs.cuh"

namespace vpm {

#ifndef VPM_CARRY_WINDOW
#define VPM_CARRY_WINDOW 32
#endif
constexpr int kCarryWindow = VPM_CARRY_WINDOW;

template <class R>
struct SweepArgs {
  const R* tgt;
  int64_t m;
  int64_t tgt_offset;  // global index of tgt[0] among the sources (self-pair exclusion)
  const R* src;
  int64_t n;
  int64_t chunk;  // sources per split (multiple of kCarryWindow unless it is the last)
  double* partial;
};

// V = double: R FP64 targets per thread.  V = float2: R FP32 targets per thread as R/2
// packed lanes; FP32 partials are folded into per-target FP64 carries every window.
#ifndef VPM_SMEM_CARRY
#define VPM_SMEM_CARRY 0
#endif
#ifndef VPM_SRC_UNROLL
#define VPM_SRC_UNROLL 2
#endif
constexpr int kSrcUnroll = VPM_SRC_UNROLL;

// Dynamic shared memory of one block: the source-tile ring, then (FP32 with shared-memory
// carries) the FP64 carries laid out [value][target][thread] for conflict-free access.
template <class V, class Rec_, int NV, int R, int THREADS, int TILE, int STAGES>
constexpr size_t sweep_smem_bytes() {
  return size_t(STAGES) * TILE * sizeof(Rec_) +
         ((LaneTraits<V>::kLanes == 2 && VPM_SMEM_CARRY) ? size_t(NV) * R * THREADS * 8 : 0);
}

template <class Op, class V, int R, int THREADS, int TILE, int STAGES, int MINB>
__global__ void __launch_bounds__(THREADS, MINB)
sweep_kernel(const SweepArgs<typename Op::Record> a) {
  using RecT = typename Op::Record;
  constexpr int NV = Op::NV;
  constexpr int L = LaneTraits<V>::kLanes;
  constexpr int P = R / L;
  constexpr bool kCarry = (L == 2);
  constexpr int CW = Op::kWindow ? Op::kWindow : kCarryWindow;  // sources per FP32 window
  static_assert(kCarryWindow % CW == 0, "windows tile the sweep's source chunks");
  constexpr bool kSmemCarry = kCarry && VPM_SMEM_CARRY;
  constexpr uint32_t kRecBytes = sizeof(RecT);
  static_assert(R % L == 0, "targets per thread must fill whole lanes");

  extern __shared__ __align__(128) unsigned char smem_raw[];
  RecT* tiles = reinterpret_cast<RecT*>(smem_raw);
  __shared__ __align__(8) uint64_t full_bar[STAGES];

  const int tid = threadIdx.x;
  const int64_t base = static_cast<int64_t>(blockIdx.x) * (THREADS * R);
  const int64_t j0 = static_cast<int64_t>(blockIdx.y) * a.chunk;
  const int64_t j1 = (j0 + a.chunk < a.n) ? j0 + a.chunk : a.n;
  const int64_t count = (j1 > j0) ? (j1 - j0) : 0;
  const int ntiles = static_cast<int>((count + TILE - 1) / TILE);

  typename Op::TgtT tg[P];
  int64_t ti[R];  // local target index
  int64_t gi[R];  // global index among the sources
  V acc[P][NV];
  double car[(kCarry && !kSmemCarry) ? R : 1][NV];
  double* scar = reinterpret_cast<double*>(smem_raw + size_t(STAGES) * TILE * sizeof(RecT));
  if constexpr (kSmemCarry) {
#pragma unroll
    for (int v = 0; v < NV; ++v)
#pragma unroll
      for (int r = 0; r < R; ++r) scar[(v * R + r) * THREADS + tid] = 0.0;
  }
#pragma unroll
  for (int p = 0; p < P; ++p) {
    const RecT* recs[L];
#pragma unroll
    for (int k = 0; k < L; ++k) {
      const int r = p * L + k;
      ti[r] = base + r * THREADS + tid;
      gi[r] = ti[r] + a.tgt_offset;
      recs[k] = a.tgt + (ti[r] < a.m ? ti[r] : a.m - 1);
    }
    tg[p] = Op::target(recs);
#pragma unroll
    for (int v = 0; v < NV; ++v) lane_zero(acc[p][v]);
  }
#pragma unroll
  for (int r = 0; r < ((kCarry && !kSmemCarry) ? R : 1); ++r)
#pragma unroll
    for (int v = 0; v < NV; ++v) car[r][v] = 0.0;

  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < STAGES; ++s) mbar_init(&full_bar[s], 1);
    fence_mbar_init();
  }
  __syncthreads();

  auto issue = [&](int t) {
    const int s = t % STAGES;
    const int64_t left = count - static_cast<int64_t>(t) * TILE;
    const uint32_t recs = static_cast<uint32_t>(left < TILE ? left : TILE);
    mbar_arrive_expect_tx(&full_bar[s], recs * kRecBytes);
    bulk_load_g2s(tiles + s * TILE, a.src + j0 + static_cast<int64_t>(t) * TILE,
                  recs * kRecBytes, &full_bar[s]);
  };

  if (tid == 0) {
    for (int t = 0; t < STAGES && t < ntiles; ++t) issue(t);
  }

  int failed_at = -1;
  for (int t = 0; t < ntiles; ++t) {
    const int s = t % STAGES;
    const bool ok = mbar_wait_bounded(&full_bar[s], static_cast<uint32_t>((t / STAGES) & 1));
    const RecT* tile = tiles + s * TILE;
    const int64_t jt = j0 + static_cast<int64_t>(t) * TILE;
    const int64_t left = count - static_cast<int64_t>(t) * TILE;
    const int cnt = static_cast<int>(left < TILE ? left : TILE);
    if (ok) {
      for (int w = 0; w < cnt; w += CW) {
        const int e = (w + CW < cnt) ? w + CW : cnt;
#pragma unroll kSrcUnroll
        for (int j = w; j < e; ++j) {
          const typename Op::SrcT src = Op::load(tile[j]);
#pragma unroll
          for (int p = 0; p < P; ++p) Op::pair(tg[p], acc[p], src, &gi[p * L], jt + j);
        }
        if constexpr (kSmemCarry) {
#pragma unroll
          for (int p = 0; p < P; ++p) {
#pragma unroll
            for (int v = 0; v < NV; ++v) {
#pragma unroll
              for (int k = 0; k < L; ++k)
                scar[(v * R + p * L + k) * THREADS + tid] += lane_get(acc[p][v], k);
              lane_zero(acc[p][v]);
            }
          }
        } else if constexpr (kCarry) {
#pragma unroll
          for (int p = 0; p < P; ++p) {
#pragma unroll
            for (int v = 0; v < NV; ++v) {
#pragma unroll
              for (int k = 0; k < L; ++k) car[p * L + k][v] += lane_get(acc[p][v], k);
              lane_zero(acc[p][v]);
            }
          }
        }
      }
    }
    // All warps are done reading stage s; a failed wait anywhere aborts the block.
    if (__syncthreads_or(!ok)) {
      failed_at = t;
      break;
    }
    if (tid == 0 && t + STAGES < ntiles) issue(t + STAGES);
  }

  if (failed_at >= 0) {
    // Let the copies this block still has in flight land before the block exits.
    if (tid == 0) {
      const int last = (failed_at + STAGES < ntiles) ? failed_at + STAGES : ntiles;
      for (int u = failed_at; u < last; ++u)
        mbar_wait_bounded(&full_bar[u % STAGES], static_cast<uint32_t>((u / STAGES) & 1));
    }
    return;
  }

  double* out = a.partial + static_cast<int64_t>(blockIdx.y) * NV * a.m;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    if (ti[r] < a.m) {
#pragma unroll
      for (int v = 0; v < NV; ++v) {
        double val;
        if constexpr (kSmemCarry)
          val = scar[(v * R + r) * THREADS + tid];
        else if constexpr (kCarry)
          val = car[r][v];
        else
          val = lane_get(acc[r / L][v], r % L);
        out[static_cast<int64_t>(v) * a.m + ti[r]] = val;
      }
    }
  }
}

}  // namespace vpm
