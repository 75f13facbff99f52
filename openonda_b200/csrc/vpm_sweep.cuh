// vpm_sweep.cuh -- the tiled all-pairs sweep (one kernel template for every operator).
//
// Grid: blockIdx.x = a block of THREADS*R targets, blockIdx.y = one contiguous chunk of
// sources (a "split").  Each thread owns R targets (i = base + r*THREADS + tid) in
// registers.  Source records stream through shared memory in tiles of TILE records:
// one elected thread issues a bulk-async (TMA) copy per tile into a STAGES-deep ring,
// completion is signalled on an mbarrier, and all warps read the tile by broadcast.
//
// Accumulation: in FP64 the partial sums accumulate directly in double.  In FP32 each
// target keeps an FP32 accumulator for a window of CW=32 consecutive sources and folds
// it into an FP64 carry at the end of every window (one DADD per value per 32 pairs), so
// rounding grows only over 32 terms and the long sum over N sources runs in FP64.
//
// Each (split, value, target) partial is written as FP64 to
// partial[(split * NV + v) * m + i]; a finalize pass sums the splits in split order, so
// the result does not depend on scheduling.
#pragma once

#include "vpm_pairs.cuh"

namespace vpm {

constexpr int kCarryWindow = 32;

template <class T>
struct SweepArgs {
  const Rec<T>* tgt;
  int64_t m;
  int64_t tgt_offset;  // global index of tgt[0] among the sources (self-pair exclusion)
  const Rec<T>* src;
  int64_t n;
  int64_t chunk;  // sources per split (multiple of kCarryWindow unless it is the last)
  double* partial;
};

template <class Op, class T, int R, int THREADS, int TILE, int STAGES>
__global__ void __launch_bounds__(THREADS)
sweep_kernel(const SweepArgs<T> a) {
  constexpr int NV = Op::NV;
  constexpr bool kFp32 = sizeof(T) == 4;
  constexpr uint32_t kRecBytes = sizeof(Rec<T>);

  extern __shared__ __align__(128) unsigned char smem_raw[];
  Rec<T>* tiles = reinterpret_cast<Rec<T>*>(smem_raw);
  __shared__ __align__(8) uint64_t full_bar[STAGES];

  const int tid = threadIdx.x;
  const int64_t base = static_cast<int64_t>(blockIdx.x) * (THREADS * R);
  const int64_t j0 = static_cast<int64_t>(blockIdx.y) * a.chunk;
  const int64_t j1 = (j0 + a.chunk < a.n) ? j0 + a.chunk : a.n;
  const int64_t count = (j1 > j0) ? (j1 - j0) : 0;
  const int ntiles = static_cast<int>((count + TILE - 1) / TILE);

  Tgt<T> tg[R];
  int64_t ti[R];
  T acc[R][NV];
  double car[R][NV];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    ti[r] = base + r * THREADS + tid;
    const int64_t il = ti[r] < a.m ? ti[r] : a.m - 1;
    tg[r] = make_tgt<T>(a.tgt[il]);
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      acc[r][v] = T(0);
      car[r][v] = 0.0;
    }
  }

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
    const Rec<T>* tile = tiles + s * TILE;
    const int64_t jt = j0 + static_cast<int64_t>(t) * TILE;
    const int cnt = static_cast<int>((count - static_cast<int64_t>(t) * TILE) < TILE
                                         ? (count - static_cast<int64_t>(t) * TILE)
                                         : TILE);
    if (ok) {
      for (int w = 0; w < cnt; w += kCarryWindow) {
        const int e = (w + kCarryWindow < cnt) ? w + kCarryWindow : cnt;
#pragma unroll 2
        for (int j = w; j < e; ++j) {
          const Src<T> src = load_src<T>(tile[j]);
#pragma unroll
          for (int r = 0; r < R; ++r) Op::pair(tg[r], acc[r], src, ti[r] + a.tgt_offset, jt + j);
        }
        if constexpr (kFp32) {
#pragma unroll
          for (int r = 0; r < R; ++r) {
#pragma unroll
            for (int v = 0; v < NV; ++v) {
              car[r][v] += static_cast<double>(acc[r][v]);
              acc[r][v] = T(0);
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
        const double val = kFp32 ? car[r][v] : static_cast<double>(acc[r][v]);
        out[static_cast<int64_t>(v) * a.m + ti[r]] = val;
      }
    }
  }
}

}  // namespace vpm
