// vpm_abi.cu -- C-ABI entry points, launch planning, pack and finalize kernels.  The
// library is one translation unit: the step and initial-condition kernels are included at
// the end.
//
// One pair-sum call = pack (reference AoS float64 -> packed records in the compute
// precision, inside the caller's workspace) -> tiled sweep (partials per source split,
// FP64) -> finalize (sum the splits in order, apply target-only factors, write the
// reference's output layout).  Scalars reduce the per-target values in a single block in a
// fixed order, so every result is deterministic.
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <unordered_map>
#include <utility>

#include <cuda.h>  // CUcontext / CUresult types only; no libcuda link

#include "vpm_b200.h"
#include "vpm_sweep.cuh"
#include "vpm_adjoint.cuh"
#include "vpm_rot.cuh"

namespace vpm {
namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

int cuda_fail(cudaError_t e, const char* where) {
  return fail(VPM_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

constexpr size_t kAlign = 256;
size_t align_up(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

// ---- kernel configurations -----------------------------------------------------------
template <class T>
struct Cfg;
#ifndef VPM_FP32_R
#define VPM_FP32_R 4
#endif
#ifndef VPM_FP32_THREADS
#define VPM_FP32_THREADS 128
#endif
#ifndef VPM_FP32_MINB
#define VPM_FP32_MINB 1
#endif
// MINB: resident blocks per SM requested from the register allocator (launch bounds).
template <>
struct Cfg<float2> {
  static constexpr int R = VPM_FP32_R, THREADS = VPM_FP32_THREADS, TILE = 256, STAGES = 2,
                       MINB = VPM_FP32_MINB;
};
#ifndef VPM_FP64_R
#define VPM_FP64_R 1
#endif
#ifndef VPM_FP64_THREADS
#define VPM_FP64_THREADS 128
#endif
template <>
struct Cfg<double> {
  static constexpr int R = VPM_FP64_R, THREADS = VPM_FP64_THREADS, TILE = 128, STAGES = 2,
                       MINB = 1;
};

#ifndef VPM_MAX_SPLITS
#define VPM_MAX_SPLITS 64
#endif
#ifndef VPM_MIN_CHUNK
#define VPM_MIN_CHUNK 256
#endif
constexpr int kMaxSplits = VPM_MAX_SPLITS;
constexpr int64_t kMinChunk = VPM_MIN_CHUNK;
constexpr size_t kMaxPartialBytes = size_t(4) << 30;

struct Plan {
  int64_t tblocks = 0;
  int splits = 1;  // source splits; the both-sides sweep: its accumulator sets (2 per pair)
  int64_t chunk = 0;
  size_t smem = 0;
  int threads = 0;
  int r = 0;
  int nv = 0;
  int pairs = 0;  // both-sides sweep (vpm_rot.cuh): diagonal pairs per launch; 0 = one-sided
  // both-sides fused sum: 0 = built for VPM_ROT_MINB CTAs/SM, 1 = _ALT, 2 = 512-particle tiles
  int variant = 0;
  // both-sides sweep: the diagonal tiles run beside the (single) diagonal-pair launch on a
  // second stream, into their own accumulator sets after the pairs' ones
  int diag_beside = 0;
};

// FP32 self sums with at least this many particles evaluate each unordered pair once for both
// particles (vpm_set_symmetric_min_n changes it).  Measured crossover of the fused sum:
// one-sided 641 / 720 / 738 against both-sides 624 / 718 / 737 Gpairs/s at 16384 / 24576 /
// 32768 particles (velocity 1155 / 1258 / 1277 against 1160 / 1350 / 1419, PSE 1231 / 1344 /
// 1374 against 1380 / 1625 / 1728).
std::atomic<int64_t> g_sym_min_n{24576};

struct DevInfo {
  int sms = 0;
  int major = 0, minor = 0;
};

std::mutex g_mu;
std::unordered_map<int, DevInfo> g_dev;
std::map<std::pair<const void*, int>, int> g_occ;  // (kernel, device) -> resident blocks/SM

int device_info(DevInfo* out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  std::lock_guard<std::mutex> lk(g_mu);
  auto it = g_dev.find(dev);
  if (it == g_dev.end()) {
    DevInfo d;
    e = cudaDeviceGetAttribute(&d.sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaDeviceGetAttribute(SM count)");
    cudaDeviceGetAttribute(&d.major, cudaDevAttrComputeCapabilityMajor, dev);
    cudaDeviceGetAttribute(&d.minor, cudaDevAttrComputeCapabilityMinor, dev);
    it = g_dev.emplace(dev, d).first;
  }
  *out = it->second;
  return VPM_OK;
}

int check_arch() {
  DevInfo d;
  int rc = device_info(&d);
  if (rc) return rc;
  if (d.major != 10 || d.minor != 0)
    return fail(VPM_ERR_ARCH, "libvpm_b200 is built for sm_100a (B200); current device is sm_" +
                                  std::to_string(d.major) + std::to_string(d.minor));
  return VPM_OK;
}

template <class Op, class T>
struct Sweep {
  using C = Cfg<T>;
  using RecT = typename Op::Record;
  static constexpr int NV = Op::NV;
  static constexpr int R = Op::kR ? Op::kR : C::R;
  // about the same tile bytes for every record width; FP32 tiles hold whole carry windows
  static constexpr int kTileRaw = int(C::TILE * sizeof(Rec<T>) / sizeof(RecT));
  static constexpr int TILE =
      LaneTraits<T>::kLanes == 2 ? kTileRaw / kCarryWindow * kCarryWindow : kTileRaw;
  static_assert(TILE >= kCarryWindow || LaneTraits<T>::kLanes == 1, "tile below a window");
  static constexpr size_t kSmem =
      sweep_smem_bytes<T, RecT, Op::NV, R, C::THREADS, TILE, C::STAGES>();
  static void* kernel() {
    return reinterpret_cast<void*>(&sweep_kernel<Op, T, R, C::THREADS, TILE, C::STAGES, C::MINB>);
  }

  static int plan(int64_t m, int64_t n, Plan* p, size_t max_partial_bytes = kMaxPartialBytes) {
    DevInfo d;
    int rc = device_info(&d);
    if (rc) return rc;
    int occ = 0;
    {
      int dev = 0;
      cudaGetDevice(&dev);
      const auto key = std::make_pair(static_cast<const void*>(kernel()), dev);
      std::lock_guard<std::mutex> lk(g_mu);
      auto it = g_occ.find(key);
      if (it != g_occ.end()) {
        occ = it->second;
      } else {
        if (kSmem > 48 * 1024) {
          cudaError_t e = cudaFuncSetAttribute(kernel(), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               int(kSmem));
          if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(max dynamic smem)");
        }
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel(),
                                                                      C::THREADS, kSmem);
        if (e != cudaSuccess) return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
        g_occ[key] = occ;
      }
    }
    if (occ < 1) occ = 1;
    const int64_t per_block = int64_t(C::THREADS) * R;
    p->tblocks = (m + per_block - 1) / per_block;
    p->smem = kSmem;
    p->threads = C::THREADS;
    p->r = R;
    p->nv = NV;
    p->splits = 1;
    p->chunk = n;
    if (n <= 0 || m <= 0) return VPM_OK;
    const double slots = double(d.sms) * occ;
    double best = -1.0;
    for (int s = 1; s <= kMaxSplits; ++s) {
      int64_t chunk = (n + s - 1) / s;
      chunk = (chunk + kCarryWindow - 1) / kCarryWindow * kCarryWindow;
      if (s > 1 && chunk < kMinChunk) break;
      const int64_t se = (n + chunk - 1) / chunk;
      if (se != s) continue;
      if (size_t(se) * NV * size_t(m) * sizeof(double) > max_partial_bytes) break;
      const double waves = double(p->tblocks) * se / slots;
      const double eff = waves / std::ceil(waves);
      const double score = eff * (1.0 - 0.003 * (se - 1));
      if (score > best + 1e-12) {
        best = score;
        p->splits = int(se);
        p->chunk = chunk;
      }
    }
    return VPM_OK;
  }

  static size_t partial_bytes(const Plan& p, int64_t m) {
    return size_t(p.splits) * NV * size_t(m) * sizeof(double);
  }

  static int launch(const Plan& p, const RecT* tgt, int64_t m, int64_t tgt_offset,
                    const RecT* src, int64_t n, double* partial, cudaStream_t st) {
    SweepArgs<RecT> a{tgt, m, tgt_offset, src, n, p.chunk, partial};
    dim3 grid(unsigned(p.tblocks), unsigned(p.splits));
    sweep_kernel<Op, T, R, C::THREADS, TILE, C::STAGES, C::MINB><<<grid, C::THREADS, p.smem, st>>>(a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "sweep launch");
    return VPM_OK;
  }
};

// ---- pack kernels ----------------------------------------------------------------------
__device__ __forceinline__ void set_elem(double& e, double v) { e = v; }
__device__ __forceinline__ void set_elem(float2& e, double v) {
  const float f = float(v);
  e = make_float2(f, f);
}

template <class E>
__global__ void pack_particles_kernel(const double* __restrict__ pos,
                                      const double* __restrict__ str,
                                      const double* __restrict__ rad,
                                      const double* __restrict__ nu, int64_t n,
                                      Rec<E>* __restrict__ out, int check_uniform) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  if (check_uniform && rad[i] != rad[0]) atomicOr(&g_device_errors, VPM_DEVERR_NONUNIFORM_CORE);
  Rec<E> r;
  set_elem(r.x, pos[3 * i]);
  set_elem(r.y, pos[3 * i + 1]);
  set_elem(r.z, pos[3 * i + 2]);
  set_elem(r.s, rad ? rad[i] : 0.0);
  set_elem(r.ax, str ? str[3 * i] : 0.0);
  set_elem(r.ay, str ? str[3 * i + 1] : 0.0);
  set_elem(r.az, str ? str[3 * i + 2] : 0.0);
  set_elem(r.nu, nu ? nu[i] : 0.0);
  out[i] = r;
}

template <class T>
int pack(const double* pos, const double* str, const double* rad, const double* nu, int64_t n,
         Rec<T>* out, cudaStream_t st, bool check_uniform = false) {
  if (n <= 0) return VPM_OK;
  const int threads = 256;
  const int64_t blocks = (n + threads - 1) / threads;
  pack_particles_kernel<T><<<unsigned(blocks), threads, 0, st>>>(pos, str, rad, nu, n, out,
                                                                 int(check_uniform && rad));
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "pack launch");
  return VPM_OK;
}

// ---- finalize kernels -----------------------------------------------------------------
enum FinKind { FIN_VEL = 0, FIN_VORT = 1, FIN_STRETCH = 2, FIN_PSE = 3, FIN_VELSTRETCH = 4,
               FIN_LES = 5 };

template <int NV>
__device__ __forceinline__ void sum_splits(const double* __restrict__ part, int splits, int64_t m,
                                           int64_t i, double (&v)[NV]) {
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = 0.0;
  for (int s = 0; s < splits; ++s) {
    const double* p = part + int64_t(s) * NV * m;
#pragma unroll
    for (int k = 0; k < NV; ++k) v[k] += p[int64_t(k) * m + i];
  }
}

// The outputs of target i from its summed values v (KIND: which sums, which scaling).
template <class T, int KIND, int NV>
__device__ __forceinline__ void finalize_values(const double (&v)[NV], const Rec<T>* tgt,
                                                int64_t i, double* __restrict__ out,
                                                double* __restrict__ out2,
                                                double* __restrict__ out3) {
  if constexpr (KIND == FIN_VEL) {
    out[3 * i] = -v[0] * kOneOver4Pi;
    out[3 * i + 1] = -v[1] * kOneOver4Pi;
    out[3 * i + 2] = -v[2] * kOneOver4Pi;
  } else if constexpr (KIND == FIN_VORT) {
    const double c = 7.5 * kOneOver4Pi;
    out[3 * i] = v[0] * c;
    out[3 * i + 1] = v[1] * c;
    out[3 * i + 2] = v[2] * c;
  } else if constexpr (KIND == FIN_PSE) {
    const double c = 105.0 * elem(tgt[i].nu) * kOneOver4Pi;
    out[3 * i] = v[0] * c;
    out[3 * i + 1] = v[1] * c;
    out[3 * i + 2] = v[2] * c;
  } else {
    constexpr bool kVel = (KIND == FIN_VELSTRETCH || KIND == FIN_LES);
    constexpr int o = kVel ? 3 : 0;
    double* so = kVel ? out2 : out;
    const double bx = elem(tgt[i].ax), by = elem(tgt[i].ay), bz = elem(tgt[i].az);
    if constexpr (KIND == FIN_LES) {
      const double c = 7.5 * kOneOver4Pi;
      out3[3 * i] = v[9] * c;
      out3[3 * i + 1] = v[10] * c;
      out3[3 * i + 2] = v[11] * c;
    }
    if constexpr (kVel) {
      out[3 * i] = -v[0] * kOneOver4Pi;
      out[3 * i + 1] = -v[1] * kOneOver4Pi;
      out[3 * i + 2] = -v[2] * kOneOver4Pi;
    }
    const double Ax = v[o], Ay = v[o + 1], Az = v[o + 2];
    so[3 * i] = (by * Az - bz * Ay + 3.0 * v[o + 3]) * kOneOver4Pi;
    so[3 * i + 1] = (bz * Ax - bx * Az + 3.0 * v[o + 4]) * kOneOver4Pi;
    so[3 * i + 2] = (bx * Ay - by * Ax + 3.0 * v[o + 5]) * kOneOver4Pi;
  }
}

template <class T, int KIND, int NV>
__global__ void finalize_vec_kernel(const double* __restrict__ part, int splits, int64_t m,
                                    const Rec<T>* __restrict__ tgt, double* __restrict__ out,
                                    double* __restrict__ out2, double* __restrict__ out3) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= m) return;
  double v[NV];
  sum_splits<NV>(part, splits, m, i, v);
  finalize_values<T, KIND, NV>(v, tgt, i, out, out2, out3);
}

// Pair shards across GPUs: rows[i][v] = the sum over the sets s, in order, of acc[s][v][i].
// One particle's NV sums in a row, so each rank's target rows are one contiguous block for
// the reduce-scatter between the GPUs.
template <int NV>
__global__ void sets_to_rows_kernel(const double* __restrict__ acc, int sets, int64_t n,
                                    double* __restrict__ rows) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double v[NV];
  sum_splits<NV>(acc, sets, n, i, v);
#pragma unroll
  for (int k = 0; k < NV; ++k) rows[i * NV + k] = v[k];
}

// The outputs of targets [0, m) (records tgt) from their summed rows (m, NV).
template <class T, int KIND, int NV>
__global__ void finalize_rows_kernel(const double* __restrict__ rows, int64_t m,
                                     const Rec<T>* __restrict__ tgt, double* __restrict__ out,
                                     double* __restrict__ out2) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= m) return;
  double v[NV];
#pragma unroll
  for (int k = 0; k < NV; ++k) v[k] = rows[i * NV + k];
  finalize_values<T, KIND, NV>(v, tgt, i, out, out2, nullptr);
}

constexpr int kReduceThreads = 1024;

// Single-block, fixed-order reduction of  scale * a_i . V_i  over all targets, V_i being
// values OFF..OFF+2 of NV partial sums per target.
template <class T, int NV = 3, int OFF = 0>
__global__ void __launch_bounds__(kReduceThreads)
finalize_dot_kernel(const double* __restrict__ part, int splits, int64_t m,
                    const Rec<T>* __restrict__ tgt, double scale, double* __restrict__ out) {
  __shared__ double red[kReduceThreads];
  double acc = 0.0;
  for (int64_t i = threadIdx.x; i < m; i += kReduceThreads) {
    double v[3] = {0.0, 0.0, 0.0};
    for (int s = 0; s < splits; ++s) {
      const double* p = part + int64_t(s) * NV * m + int64_t(OFF) * m;
#pragma unroll
      for (int k = 0; k < 3; ++k) v[k] += p[int64_t(k) * m + i];
    }
    acc += elem(tgt[i].ax) * v[0] + elem(tgt[i].ay) * v[1] + elem(tgt[i].az) * v[2];
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int w = kReduceThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = red[0] * scale;
}

// scale * the sum over all targets of value OFF of NV partial sums per target, in a fixed
// order (the same one as finalize_dot_kernel)
template <int NV, int OFF>
__global__ void __launch_bounds__(kReduceThreads)
finalize_sum_kernel(const double* __restrict__ part, int splits, int64_t m, double scale,
                    double* __restrict__ out) {
  __shared__ double red[kReduceThreads];
  double acc = 0.0;
  for (int64_t i = threadIdx.x; i < m; i += kReduceThreads) {
    double v = 0.0;
    for (int s = 0; s < splits; ++s) v += part[(int64_t(s) * NV + OFF) * m + i];
    acc += v;
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int w = kReduceThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) out[0] = red[0] * scale;
}

__global__ void write_scalar_kernel(double* out, double v) { out[0] = v; }

template <class T, int KIND, int NV>
int finalize_vec(const double* part, int splits, int64_t m, const Rec<T>* tgt, double* out,
                 double* out2, cudaStream_t st, double* out3 = nullptr) {
  if (m <= 0) return VPM_OK;
  const int threads = 256;
  finalize_vec_kernel<T, KIND, NV><<<unsigned((m + threads - 1) / threads), threads, 0, st>>>(
      part, splits, m, tgt, out, out2, out3);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "finalize launch");
  return VPM_OK;
}

__global__ void zero_kernel(double* p, int64_t count) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i < count) p[i] = 0.0;
}

int zero_out(double* p, int64_t count, cudaStream_t st) {
  if (count <= 0) return VPM_OK;
  zero_kernel<<<unsigned((count + 255) / 256), 256, 0, st>>>(p, count);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "zero launch");
  return VPM_OK;
}

// Both-sides sweep of an FP32 self sum (vpm_rot.cuh): launch 0 on the diagonal tiles, then
// ceil(floor(nt/2) / m) launches of m diagonal pairs each.
int current_context(void** ctx);

// A second stream per device and context for the both-sides sweep's diagonal tiles, with the
// two events that fork it from and join it to the caller's stream.  Created on first use
// with that context current (a stream belongs to one context, so another context, or the
// same device after a reset, gets its own); g_side_mu serialises the fork-launch-join
// sequence, so calls from several host threads never mix their events.
struct SideStream {
  cudaStream_t stream = nullptr;
  cudaEvent_t fork = nullptr, join = nullptr;
};
std::mutex g_side_mu;
std::map<std::pair<int, void*>, SideStream> g_side;

// The calling thread holds g_side_mu.
int side_stream(SideStream** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  void* ctx = nullptr;
  int rc = current_context(&ctx);
  if (rc) return rc;
  const auto key = std::make_pair(dev, ctx);
  auto it = g_side.find(key);
  if (it == g_side.end()) {
    SideStream ss;
    e = cudaStreamCreateWithFlags(&ss.stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamCreateWithFlags(side stream)");
    e = cudaEventCreateWithFlags(&ss.fork, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&ss.join, cudaEventDisableTiming);
    if (e != cudaSuccess) return cuda_fail(e, "cudaEventCreateWithFlags(side stream)");
    it = g_side.emplace(key, ss).first;
  }
  *out = &it->second;
  return VPM_OK;
}

template <class Op>
struct RotSweep {
  static constexpr int NV = Op::NV;
  static constexpr int kMaxPairs = 32;
  static constexpr int kTile = rot_tile<Op>();
  static constexpr size_t kSmem = rot_smem_bytes<Op>();
  static int64_t tiles(int64_t n) { return (n + kTile - 1) / kTile; }
  static size_t set_bytes(int64_t n) { return size_t(NV) * size_t(n) * sizeof(double); }

  // Whether the planner takes this sweep for a self sum of n particles: the size threshold
  // (vpm_set_symmetric_min_n), two tiles at least, and the smallest set count (that of the
  // diagonal tiles' launch) within the caller's partial-sum budget.
  static bool usable(int64_t m, int64_t n, size_t max_partial_bytes) {
    return m == n && n >= g_sym_min_n.load() && tiles(n) >= 2 &&
           sets(1) * set_bytes(n) <= max_partial_bytes;
  }
  // accumulator sets of a plan with m diagonal pairs per launch: 2 per pair, and at least the
  // kRotDiagSplit the diagonal tiles' launch writes (after the pairs' sets when it runs beside
  // the pair launches)
  static int64_t sets(int m, bool beside = false) {
    if (beside) return 2 * int64_t(m) + kRotDiagSplit;
    return 2 * m > kRotDiagSplit ? 2 * m : kRotDiagSplit;
  }

  // The kernel of the operator's precision: rot_sweep_kernel (FP32 lanes) or
  // rot64_sweep_kernel (FP64).
  template <bool DIAG>
  static const void* kernel_ptr() {
    if constexpr (Op::kFP64)
      return reinterpret_cast<const void*>(&rot64_sweep_kernel<Op, DIAG>);
    else
      return reinterpret_cast<const void*>(&rot_sweep_kernel<Op, DIAG>);
  }
  template <bool DIAG>
  static void launch_kernel(unsigned grid, const RotArgs& a, cudaStream_t st) {
    if constexpr (Op::kFP64)
      rot64_sweep_kernel<Op, DIAG><<<grid, kRotThreads, kSmem, st>>>(a);
    else
      rot_sweep_kernel<Op, DIAG><<<grid, kRotThreads, kSmem, st>>>(a);
  }

  // Shared-memory attributes and resident CTAs per SM, once per device (cached like the
  // one-sided sweeps' plans).
  static int prepare(int* occ) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    const void* ks = kernel_ptr<false>();
    const void* kd = kernel_ptr<true>();
    const auto key = std::make_pair(ks, dev);
    std::lock_guard<std::mutex> lk(g_mu);
    auto it = g_occ.find(key);
    if (it != g_occ.end()) {
      *occ = it->second;
      return VPM_OK;
    }
    for (const void* fn : {kd, ks}) {
      e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(kSmem));
      if (e != cudaSuccess) return cuda_fail(e, "cudaFuncSetAttribute(both-sides sweep)");
    }
    int o = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&o, ks, kRotThreads, kSmem);
    if (e != cudaSuccess) return cuda_fail(e, "cudaOccupancyMaxActiveBlocksPerMultiprocessor");
    *occ = o > 0 ? o : 1;
    g_occ[key] = *occ;
    return VPM_OK;
  }

  // Waves (rounds of resident CTAs, each about one tile pair long) that the diagonal-pair
  // launches of a plan with m pairs per launch take: npairs / m launches of m nt CTAs and a
  // last one of the remaining pairs.
  static int64_t pair_waves(int64_t npairs, int64_t nt, int64_t m, int64_t slots) {
    const int64_t full = npairs / m, rem = npairs - full * m;
    return full * ((m * nt + slots - 1) / slots) + (rem * nt + slots - 1) / slots;
  }

  // eff_out: the fraction of whole waves the chosen launches fill (ideal waves / waves)
  static int plan(int64_t n, Plan* p, size_t max_partial_bytes, double* eff_out = nullptr) {
    DevInfo d;
    int rc = device_info(&d);
    if (rc) return rc;
    int occ = 1;
    rc = prepare(&occ);
    if (rc) return rc;
    const int64_t nt = tiles(n);
    const int64_t npairs = nt / 2;
    const int64_t slots = int64_t(d.sms) * occ;
    // Pairs per launch, two candidates within the caller's workspace budget: m0, the first m
    // whose own launch fills 97 % of whole waves (else the best such fill), and m1, the m whose
    // launches take the fewest waves in all (the smaller m on a tie).  m0 is kept unless m1
    // saves more than 1 % of the waves: at equal wave counts the launches of m0 measured up to
    // 5 % faster (fused sum at 65536, LES sums at 262144), while m1 gains 1.5 % at 2^20 and 7 %
    // at 49152.  (Splitting each tile pair's sources over several CTAs, to fill the waves at
    // small n, measured slower: every part repeats the target side's carries and final FP64
    // atomics, and the sets to zero and sum multiply.)
    int m0 = 1;
    double be = -1.0;
    for (int m = 1; m <= kMaxPairs && m <= npairs; ++m) {
      if (m > 1 && sets(m) * set_bytes(n) > max_partial_bytes) break;
      const double waves = double(m) * nt / double(slots);
      const double eff = waves / std::ceil(waves);
      if (eff > be + 1e-9) {
        be = eff;
        m0 = m;
      }
      if (eff >= 0.97) break;
    }
    int m1 = 1;
    int64_t w1 = pair_waves(npairs, nt, 1, slots);
    for (int m = 2; m <= kMaxPairs && m <= npairs; ++m) {
      if (sets(m) * set_bytes(n) > max_partial_bytes) break;
      const int64_t w = pair_waves(npairs, nt, m, slots);
      if (w < w1) {
        w1 = w;
        m1 = m;
      }
    }
    const int64_t w0 = pair_waves(npairs, nt, m0, slots);
    const bool keep0 = double(w0) <= 1.01 * double(w1);
    const int best_m = keep0 ? m0 : m1;
    const int64_t best_w = keep0 ? w0 : w1;
    const double best = double(npairs) * nt / double(slots) / double(best_w);
    if (eff_out) *eff_out = best;
    // Small n (pair launches of at most 64 waves of whole tile pairs): the diagonal tiles' CTAs
    // (a quarter tile of sources each) run beside the pair launches on a second stream, into
    // four sets of their own, and take the slots their waves leave free, instead of a launch
    // of their own before them.  Measured (Gpairs/s, own launch -> beside): fused sum 574 ->
    // 622 at 16384, 739 -> 748 at 32768; velocity 1427 -> 1477 and PSE 1733 -> 1808 at 32768;
    // 1-2 % at 49152.  At large n that launch is a few tenths of a percent of the sweep.
    const bool beside = best_w <= 64 && sets(best_m, true) * set_bytes(n) <= max_partial_bytes;
    if (beside) {
      // create the side stream now, outside any stream capture of the launch that follows
      std::lock_guard<std::mutex> lk(g_side_mu);
      SideStream* ss = nullptr;
      rc = side_stream(&ss);
      if (rc) return rc;
    }
    p->diag_beside = beside ? 1 : 0;
    p->pairs = best_m;
    p->tblocks = nt;
    p->splits = int(sets(best_m, beside));
    p->chunk = n;
    p->smem = kSmem;
    p->threads = kRotThreads;
    p->r = 2 * Op::kP;
    p->nv = NV;
    return VPM_OK;
  }

  // acc: [p.splits][NV][n] FP64, zeroed here.
  static int launch(const Plan& p, const void* rec, int64_t n, double* acc,
                    cudaStream_t st) {
    const int nt = int(tiles(n));
    int occ = 1;
    int rc = prepare(&occ);
    if (!rc) rc = zero_out(acc, int64_t(p.splits) * NV * n, st);
    if (rc) return rc;
    cudaError_t e = cudaSuccess;
    const int npairs = nt / 2;
    SideStream* ss = nullptr;
    std::unique_lock<std::mutex> lk(g_side_mu, std::defer_lock);
    if (p.diag_beside) {
      // the pair launches on the caller's stream, the diagonal tiles on the side stream into
      // sets [sets of the pairs, + kRotDiagSplit); the caller's stream waits for both (fork
      // and join by events, so CUDA-graph capture records the same dependencies)
      lk.lock();
      rc = side_stream(&ss);
      if (rc) return rc;
      e = cudaEventRecord(ss->fork, st);
      if (e != cudaSuccess) return cuda_fail(e, "cudaEventRecord(fork)");
    } else {
      launch_kernel<true>(unsigned(nt * kRotDiagSplit), RotArgs{rec, n, nt, 0, acc}, st);
      e = cudaGetLastError();
      if (e != cudaSuccess) return cuda_fail(e, "both-sides sweep launch");
    }
    for (int k0 = 1; k0 <= npairs; k0 += p.pairs) {
      const int m = (npairs - k0 + 1 < p.pairs) ? npairs - k0 + 1 : p.pairs;
      launch_kernel<false>(unsigned(m * nt), RotArgs{rec, n, nt, k0, acc}, st);
      e = cudaGetLastError();
      if (e != cudaSuccess) return cuda_fail(e, "both-sides sweep launch");
    }
    if (p.diag_beside) {
      e = cudaStreamWaitEvent(ss->stream, ss->fork, 0);
      if (e != cudaSuccess) return cuda_fail(e, "cudaStreamWaitEvent(fork)");
      RotArgs d{rec, n, nt, 0, acc};
      d.set0 = 2 * p.pairs;
      launch_kernel<true>(unsigned(nt * kRotDiagSplit), d, ss->stream);
      e = cudaGetLastError();
      if (e != cudaSuccess) return cuda_fail(e, "both-sides sweep launch");
      e = cudaEventRecord(ss->join, ss->stream);
      if (e != cudaSuccess) return cuda_fail(e, "cudaEventRecord(join)");
      e = cudaStreamWaitEvent(st, ss->join, 0);
      if (e != cudaSuccess) return cuda_fail(e, "cudaStreamWaitEvent(join)");
    }
    return VPM_OK;
  }

  // Part of a sweep (pair shards across GPUs): the diagonal tiles [t_begin, t_end) and the
  // diagonal pairs k in [k_begin, k_end) (k = 1 .. nt / 2), in launches of p.pairs pairs, on
  // the caller's stream into the sets of a plan without the side stream.
  // acc: [sets(p.pairs)][NV][n] FP64, zeroed here.
  static int launch_part(const Plan& p, const void* rec, int64_t n, double* acc, int t_begin,
                         int t_end, int k_begin, int k_end, cudaStream_t st) {
    const int nt = int(tiles(n));
    int occ = 1;
    int rc = prepare(&occ);
    if (!rc) rc = zero_out(acc, sets(p.pairs) * NV * n, st);
    if (rc) return rc;
    cudaError_t e = cudaSuccess;
    if (t_end > t_begin) {
      RotArgs d{rec, n, nt, 0, acc};
      d.tile0 = t_begin;
      launch_kernel<true>(unsigned((t_end - t_begin) * kRotDiagSplit), d, st);
      e = cudaGetLastError();
      if (e != cudaSuccess) return cuda_fail(e, "both-sides sweep launch");
    }
    for (int k0 = k_begin; k0 < k_end; k0 += p.pairs) {
      const int m = (k_end - k0 < p.pairs) ? k_end - k0 : p.pairs;
      launch_kernel<false>(unsigned(m * nt), RotArgs{rec, n, nt, k0, acc}, st);
      e = cudaGetLastError();
      if (e != cudaSuccess) return cuda_fail(e, "both-sides sweep launch");
    }
    return VPM_OK;
  }
};

// ---- adjoint: pack, finalize --------------------------------------------------------------
template <class E>
__global__ void pack_grad_kernel(const double* __restrict__ pos, const double* __restrict__ str,
                                 const double* __restrict__ rad, const double* __restrict__ nu,
                                 const double* __restrict__ gu, const double* __restrict__ gs,
                                 int64_t n, RecG<E>* __restrict__ out) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  RecG<E> r;
  set_elem(r.x, pos[3 * i]);
  set_elem(r.y, pos[3 * i + 1]);
  set_elem(r.z, pos[3 * i + 2]);
  set_elem(r.s, rad[i]);
  set_elem(r.ax, str[3 * i]);
  set_elem(r.ay, str[3 * i + 1]);
  set_elem(r.az, str[3 * i + 2]);
  set_elem(r.nu, nu ? 105.0 * nu[i] : 0.0);
  set_elem(r.ux, -kOneOver4Pi * gu[3 * i]);
  set_elem(r.uy, -kOneOver4Pi * gu[3 * i + 1]);
  set_elem(r.uz, -kOneOver4Pi * gu[3 * i + 2]);
  const double ax = str[3 * i], ay = str[3 * i + 1], az = str[3 * i + 2];
  const double sx = kOneOver4Pi * gs[3 * i], sy = kOneOver4Pi * gs[3 * i + 1],
               sz = kOneOver4Pi * gs[3 * i + 2];
  set_elem(r.gx, sx);
  set_elem(r.gy, sy);
  set_elem(r.gz, sz);
  set_elem(r.mx, ay * sz - az * sy);  // m = a x s'
  set_elem(r.my, az * sx - ax * sz);
  set_elem(r.mz, ax * sy - ay * sx);
  set_elem(r.pad0, 0.0);
  set_elem(r.pad1, 0.0);
  set_elem(r.pad2, 0.0);
  out[i] = r;
}

template <class E, int NV, bool PSE>
__global__ void finalize_vjp_kernel(const double* __restrict__ part, int splits, int64_t m,
                                    const RecG<E>* __restrict__ tgt, double* __restrict__ gx,
                                    double* __restrict__ ga, double* __restrict__ gsig,
                                    double* __restrict__ gnu) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= m) return;
  double v[NV];
  sum_splits<NV>(part, splits, m, i, v);
  const RecG<E>& t = tgt[i];
  const double ax = elem(t.ax), ay = elem(t.ay), az = elem(t.az);
  const double ux = elem(t.ux), uy = elem(t.uy), uz = elem(t.uz);
  const double sx = elem(t.gx), sy = elem(t.gy), sz = elem(t.gz);
  const double Gx = v[VJ_GA], Gy = v[VJ_GA + 1], Gz = v[VJ_GA + 2];
  const double Hx = v[VJ_GU], Hy = v[VJ_GU + 1], Hz = v[VJ_GU + 2];
  // xbar += G_a x u'_k - a_k x G_u
  gx[3 * i] = v[VJ_X] + (Gy * uz - Gz * uy) - (ay * Hz - az * Hy);
  gx[3 * i + 1] = v[VJ_X + 1] + (Gz * ux - Gx * uz) - (az * Hx - ax * Hz);
  gx[3 * i + 2] = v[VJ_X + 2] + (Gx * uy - Gy * ux) - (ax * Hy - ay * Hx);
  // abar += G_a x s'_k  (+ PSE: sum k nu'_l s'_l - (sum k) nu'_k s'_k)
  double bx = v[VJ_A] + (Gy * sz - Gz * sy);
  double by = v[VJ_A + 1] + (Gz * sx - Gx * sz);
  double bz = v[VJ_A + 2] + (Gx * sy - Gy * sx);
  if constexpr (PSE) {
    const double kn = v[VJ_K] * elem(t.nu);
    bx += v[VJ_KS] - kn * sx;
    by += v[VJ_KS + 1] - kn * sy;
    bz += v[VJ_KS + 2] - kn * sz;
  }
  ga[3 * i] = bx;
  ga[3 * i + 1] = by;
  ga[3 * i + 2] = bz;
  gsig[i] = 0.5 * v[VJ_S];
  if (gnu) gnu[i] = PSE ? 105.0 * v[VJ_NU] : 0.0;
}

__global__ void finalize_kegrad_kernel(const double* __restrict__ part, int splits, int64_t m,
                                       double* __restrict__ gx, double* __restrict__ ga,
                                       double* __restrict__ gsig) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= m) return;
  double v[7];
  sum_splits<7>(part, splits, m, i, v);
  const double c = 2.0 / (16.0 * kPi);
  gx[3 * i] = c * v[0];
  gx[3 * i + 1] = c * v[1];
  gx[3 * i + 2] = c * v[2];
  ga[3 * i] = c * v[3];
  ga[3 * i + 1] = c * v[4];
  ga[3 * i + 2] = c * v[5];
  gsig[i] = 0.5 * c * v[6];
}

// ---- operator selection -----------------------------------------------------------------
// UC: all cores equal (VPM_UNIFORM_CORE); the probe sums and the kinetic energy keep the
// general form.
template <class T, bool REFINE, bool UC = false>
struct Ops {
  using Vel = OpVel<T, REFINE, UC>;
  using VelAt = OpVelAt<T, REFINE>;
  using VortAt = OpVortAt<T, REFINE>;
  using Stretch = OpStretch<T, REFINE, UC>;
  using Pse = OpPse<T, REFINE, UC>;
  using Ke = OpKe<T, REFINE>;
  using Ens = OpEns<T, REFINE, UC>;
  using VelStretch = OpVelStretch<T, REFINE, UC>;
  using LesStep = OpLesStep<T, REFINE, UC>;
  using VelStretchBoth = OpVelStretchBoth<REFINE, UC>;  // FP32 only
  using VelStretchBothAlt = OpVelStretchBoth<REFINE, UC, VPM_ROT_MINB_ALT>;
  using VelStretchBothSmall = OpVelStretchBoth<REFINE, UC, VPM_ROT_MINB_ALT, 2>;
  using VelStretchBoth64 = OpVelStretchBoth64<UC>;  // FP64 only
  using VelBoth64 = OpVelBoth64<UC>;                // FP64 only
  using PseBoth64 = OpPseBoth64<UC>;                // FP64 only
  using LesStepBoth64 = OpLesStepBoth64<UC>;        // FP64 only
  using VelBoth = OpVelBoth<REFINE, UC>;                // FP32 only
  using PseBoth = OpPseBoth<REFINE, UC>;                // FP32 only
  using LesStepBoth = OpLesStepBoth<REFINE, UC>;        // FP32 only
  using RhsVjpBoth = OpRhsVjpBoth<REFINE, false>;       // FP32 only
  using RhsVjpPseBoth = OpRhsVjpBoth<REFINE, true>;     // FP32 only
  using RhsVjp = OpRhsVjp<T, REFINE, false>;
  using RhsVjpPse = OpRhsVjp<T, REFINE, true>;
  using KeGrad = OpKeGrad<T, REFINE>;
};

bool is_probe(int op) { return op == VPM_OP_INDUCED_VELOCITY_AT || op == VPM_OP_VORTICITY_FIELD_AT; }

template <class T, bool REFINE, bool UC = false>
int plan_op(int op, int64_t m, int64_t n, Plan* p, size_t mpb = kMaxPartialBytes) {
  using O = Ops<T, REFINE, UC>;
  switch (op) {
    case VPM_OP_SELFINDUCED_VELOCITY:
      if constexpr (LaneTraits<T>::kLanes == 2) {
        if (RotSweep<typename O::VelBoth>::usable(m, n, mpb))
          return RotSweep<typename O::VelBoth>::plan(n, p, mpb);
      } else {
        if (RotSweep<typename O::VelBoth64>::usable(m, n, mpb))
          return RotSweep<typename O::VelBoth64>::plan(n, p, mpb);
      }
      return Sweep<typename O::Vel, T>::plan(m, n, p, mpb);
    case VPM_OP_TOTAL_HELICITY:
      return Sweep<typename O::Vel, T>::plan(m, n, p, mpb);
    case VPM_OP_INDUCED_VELOCITY_AT:
      return Sweep<typename O::VelAt, T>::plan(m, n, p, mpb);
    case VPM_OP_VORTICITY_FIELD_AT:
      return Sweep<typename O::VortAt, T>::plan(m, n, p, mpb);
    case VPM_OP_STRENGTH_GRADIENTS:
      return Sweep<typename O::Stretch, T>::plan(m, n, p, mpb);
    case VPM_OP_STRENGTH_GRADIENTS_PSE:
      if constexpr (LaneTraits<T>::kLanes == 2) {
        if (RotSweep<typename O::PseBoth>::usable(m, n, mpb))
          return RotSweep<typename O::PseBoth>::plan(n, p, mpb);
      } else {
        if (RotSweep<typename O::PseBoth64>::usable(m, n, mpb))
          return RotSweep<typename O::PseBoth64>::plan(n, p, mpb);
      }
      return Sweep<typename O::Pse, T>::plan(m, n, p, mpb);
    case VPM_OP_TOTAL_KINETIC_ENERGY:
      return Sweep<typename O::Ke, T>::plan(m, n, p, mpb);
    case VPM_OP_TOTAL_ENSTROPHY:
      return Sweep<typename O::Ens, T>::plan(m, n, p, mpb);
    case VPM_OP_VELOCITY_AND_STRENGTH_GRADIENTS:
      if constexpr (LaneTraits<T>::kLanes == 2) {
        if (RotSweep<typename O::VelStretchBoth>::usable(m, n, mpb)) {
          // two builds of the fused sum on 768-particle tiles (3 and 2 resident CTAs per SM):
          // take the one whose launches fill the waves better, the 2-CTA build on a tie (it
          // measured equal or faster whenever its waves were as full).  A third on
          // 512-particle tiles (4 targets per lane, 2 CTAs per SM) evaluates pairs at about
          // 0.92 of their rate but makes 2.25x the tile pairs, so it fills the waves where
          // few 768-particle tiles do not (24576: 728 -> 768, 32768: 748 -> 790 Gpairs/s;
          // 49152 and up 6-9 % slower): taken when 0.92 of its fill beats theirs by 1 %.
          constexpr double kSmallTileRate = 0.92;
          Plan pa, pb, pc;
          double ea = 0.0, eb = 0.0, ec = 0.0;
          int rc = RotSweep<typename O::VelStretchBoth>::plan(n, &pa, mpb, &ea);
          if (!rc) rc = RotSweep<typename O::VelStretchBothAlt>::plan(n, &pb, mpb, &eb);
          if (rc) return rc;
          double e = ea;
          if (eb >= ea - 0.01) {
            pb.variant = 1;
            *p = pb;
            e = eb;
          } else {
            *p = pa;
          }
          if (RotSweep<typename O::VelStretchBothSmall>::usable(m, n, mpb)) {
            rc = RotSweep<typename O::VelStretchBothSmall>::plan(n, &pc, mpb, &ec);
            if (rc) return rc;
            if (kSmallTileRate * ec > e + 0.01) {
              pc.variant = 2;
              *p = pc;
            }
          }
          return VPM_OK;
        }
      } else {
        if (RotSweep<typename O::VelStretchBoth64>::usable(m, n, mpb))
          return RotSweep<typename O::VelStretchBoth64>::plan(n, p, mpb);
      }
      return Sweep<typename O::VelStretch, T>::plan(m, n, p, mpb);
    case VPM_OP_LES_STEP_SUMS:
      if constexpr (LaneTraits<T>::kLanes == 2) {
        if (RotSweep<typename O::LesStepBoth>::usable(m, n, mpb))
          return RotSweep<typename O::LesStepBoth>::plan(n, p, mpb);
      } else {
        if (RotSweep<typename O::LesStepBoth64>::usable(m, n, mpb))
          return RotSweep<typename O::LesStepBoth64>::plan(n, p, mpb);
      }
      return Sweep<typename O::LesStep, T>::plan(m, n, p, mpb);
    case VPM_OP_RHS_VJP:
      if constexpr (LaneTraits<T>::kLanes == 2) {
        if (RotSweep<typename O::RhsVjpBoth>::usable(m, n, mpb))
          return RotSweep<typename O::RhsVjpBoth>::plan(n, p, mpb);
      }
      return Sweep<typename O::RhsVjp, T>::plan(m, n, p, mpb);
    case VPM_OP_RHS_VJP_PSE:
      if constexpr (LaneTraits<T>::kLanes == 2) {
        if (RotSweep<typename O::RhsVjpPseBoth>::usable(m, n, mpb))
          return RotSweep<typename O::RhsVjpPseBoth>::plan(n, p, mpb);
      }
      return Sweep<typename O::RhsVjpPse, T>::plan(m, n, p, mpb);
    case VPM_OP_KINETIC_ENERGY_GRAD:
      return Sweep<typename O::KeGrad, T>::plan(m, n, p, mpb);
    case VPM_OP_LES_TEST_FILTER:
      return Sweep<OpTestFilter<T, REFINE>, T>::plan(m, n, p, mpb);
    default:
      return fail(VPM_ERR_ARG, "unknown op " + std::to_string(op));
  }
}

struct Layout {
  size_t src_off = 0, tgt_off = 0, part_off = 0, total = 0;
};

template <class T>
size_t op_record_bytes(int op) {
  if (op == VPM_OP_RHS_VJP || op == VPM_OP_RHS_VJP_PSE) return sizeof(RecG<T>);
  if (op == VPM_OP_LES_TEST_FILTER) return sizeof(RecF<T>);
  return sizeof(Rec<T>);
}

template <class T>
Layout layout_for(int op, const Plan& p, int64_t m, int64_t n) {
  Layout L;
  L.src_off = 0;
  size_t off = align_up(size_t(n > 0 ? n : 0) * op_record_bytes<T>(op));
  L.tgt_off = off;
  if (is_probe(op)) off = align_up(off + size_t(m > 0 ? m : 0) * sizeof(Rec<T>));
  L.part_off = off;
  off = align_up(off + size_t(p.splits) * p.nv * size_t(m > 0 ? m : 0) * sizeof(double));
  L.total = off;
  return L;
}

template <class T, bool REFINE, bool UC = false>
int workspace_for(int op, int64_t m, int64_t n, Layout* L, Plan* p,
                  size_t max_partial_bytes = kMaxPartialBytes) {
  int rc = plan_op<T, REFINE, UC>(op, m, n, p, max_partial_bytes);
  if (rc) return rc;
  *L = layout_for<T>(op, *p, m, n);
  return VPM_OK;
}

struct Call {
  int op;
  const double* tgt;  // probe targets (m,3) or null for self sums
  int64_t m;
  const double* pos;
  const double* str;
  const double* rad;
  const double* nu;
  int64_t n;
  double* out;
  double* out2;
  int ref_extra_4pi;
  void* ws;
  size_t ws_bytes;
  cudaStream_t st;
  const void* records = nullptr;  // pre-packed sources (self sums); null = pack from AoS
  int64_t tgt_begin = 0;          // self sums: targets are records[tgt_begin, tgt_begin + m)
  size_t max_partial_bytes = kMaxPartialBytes;  // caps the source splits of the plan
  double* out3 = nullptr;  // VPM_OP_LES_STEP_SUMS: vorticity (m,3)
  double* out4 = nullptr;  // VPM_OP_LES_STEP_SUMS: enstrophy (device scalar)
  const double* aux = nullptr;  // VPM_OP_LES_TEST_FILTER: the filtered fields (n,3)
};

template <class T, bool REFINE, bool UC>
int run(const Call& c) {
  using O = Ops<T, REFINE, UC>;
  int rc = check_arch();
  if (rc) return rc;
  const bool scalar = c.op == VPM_OP_TOTAL_KINETIC_ENERGY || c.op == VPM_OP_TOTAL_HELICITY ||
                      c.op == VPM_OP_TOTAL_ENSTROPHY;
  // Empty inputs: zero outputs, no sweep, no workspace needed.
  if (c.m <= 0 || c.n <= 0) {
    if (scalar) {
      write_scalar_kernel<<<1, 1, 0, c.st>>>(c.out, 0.0);
      cudaError_t e = cudaGetLastError();
      return e == cudaSuccess ? VPM_OK : cuda_fail(e, "write launch");
    }
    rc = zero_out(c.out, 3 * (c.m > 0 ? c.m : 0), c.st);
    if (!rc && c.out2) rc = zero_out(c.out2, 3 * (c.m > 0 ? c.m : 0), c.st);
    if (!rc && c.out3) rc = zero_out(c.out3, 3 * (c.m > 0 ? c.m : 0), c.st);
    if (!rc && c.out4) rc = zero_out(c.out4, 1, c.st);
    return rc;
  }

  Plan p;
  Layout L;
  rc = workspace_for<T, REFINE, UC>(c.op, c.m, c.n, &L, &p, c.max_partial_bytes);
  if (rc) return rc;
  if (c.ws == nullptr) return fail(VPM_ERR_WORKSPACE, "workspace is null");
  if (reinterpret_cast<uintptr_t>(c.ws) % kAlign != 0)
    return fail(VPM_ERR_ALIGN, "workspace must be 256-byte aligned");
  if (c.ws_bytes < L.total)
    return fail(VPM_ERR_WORKSPACE, "workspace has " + std::to_string(c.ws_bytes) +
                                       " bytes, needs " + std::to_string(L.total));
  char* ws = static_cast<char*>(c.ws);
  Rec<T>* src = c.records ? const_cast<Rec<T>*>(static_cast<const Rec<T>*>(c.records))
                          : reinterpret_cast<Rec<T>*>(ws + L.src_off);
  Rec<T>* tgt = is_probe(c.op) ? reinterpret_cast<Rec<T>*>(ws + L.tgt_off) : src + c.tgt_begin;
  double* part = reinterpret_cast<double*>(ws + L.part_off);

  if (!c.records) {
    rc = pack<T>(c.pos, c.str, c.rad, c.nu, c.n, src, c.st, UC);
    if (rc) return rc;
  }
  if (is_probe(c.op)) {
    rc = pack<T>(c.tgt, nullptr, nullptr, nullptr, c.m, tgt, c.st);
    if (rc) return rc;
  }

  switch (c.op) {
    case VPM_OP_SELFINDUCED_VELOCITY:
      rc = VPM_OK;
      if (p.pairs) {  // m == n: the targets are all the records (tgt_begin == 0)
        if constexpr (LaneTraits<T>::kLanes == 2)
          rc = RotSweep<typename O::VelBoth>::launch(p, src, c.n, part, c.st);
        else
          rc = RotSweep<typename O::VelBoth64>::launch(p, src, c.n, part, c.st);
      }
      if (!p.pairs)
        rc = Sweep<typename O::Vel, T>::launch(p, tgt, c.m, c.tgt_begin, src, c.n, part, c.st);
      if (!rc) rc = finalize_vec<T, FIN_VEL, 3>(part, p.splits, c.m, tgt, c.out, nullptr, c.st);
      return rc;
    case VPM_OP_INDUCED_VELOCITY_AT:
      rc = Sweep<typename O::VelAt, T>::launch(p, tgt, c.m, c.tgt_begin, src, c.n, part, c.st);
      if (!rc) rc = finalize_vec<T, FIN_VEL, 3>(part, p.splits, c.m, tgt, c.out, nullptr, c.st);
      return rc;
    case VPM_OP_VORTICITY_FIELD_AT:
      rc = Sweep<typename O::VortAt, T>::launch(p, tgt, c.m, c.tgt_begin, src, c.n, part, c.st);
      if (!rc) rc = finalize_vec<T, FIN_VORT, 3>(part, p.splits, c.m, tgt, c.out, nullptr, c.st);
      return rc;
    case VPM_OP_STRENGTH_GRADIENTS:
      rc = Sweep<typename O::Stretch, T>::launch(p, tgt, c.m, c.tgt_begin, src, c.n, part, c.st);
      if (!rc)
        rc = finalize_vec<T, FIN_STRETCH, 6>(part, p.splits, c.m, tgt, c.out, nullptr, c.st);
      return rc;
    case VPM_OP_STRENGTH_GRADIENTS_PSE:
      rc = VPM_OK;
      if (p.pairs) {
        if constexpr (LaneTraits<T>::kLanes == 2)
          rc = RotSweep<typename O::PseBoth>::launch(p, src, c.n, part, c.st);
        else
          rc = RotSweep<typename O::PseBoth64>::launch(p, src, c.n, part, c.st);
      }
      if (!p.pairs)
        rc = Sweep<typename O::Pse, T>::launch(p, tgt, c.m, c.tgt_begin, src, c.n, part, c.st);
      if (!rc) rc = finalize_vec<T, FIN_PSE, 3>(part, p.splits, c.m, tgt, c.out, nullptr, c.st);
      return rc;
    case VPM_OP_VELOCITY_AND_STRENGTH_GRADIENTS:
      if constexpr (LaneTraits<T>::kLanes == 2) {
        if (p.pairs && p.variant == 2)  // m == n: the targets are all the records
          rc = RotSweep<typename O::VelStretchBothSmall>::launch(p, src, c.n, part, c.st);
        else if (p.pairs && p.variant == 1)
          rc = RotSweep<typename O::VelStretchBothAlt>::launch(p, src, c.n, part, c.st);
        else if (p.pairs)
          rc = RotSweep<typename O::VelStretchBoth>::launch(p, src, c.n, part, c.st);
        else
          rc = Sweep<typename O::VelStretch, T>::launch(p, tgt, c.m, c.tgt_begin, src, c.n,
                                                        part, c.st);
      } else if (p.pairs) {
        rc = RotSweep<typename O::VelStretchBoth64>::launch(p, src, c.n, part, c.st);
      } else {
        rc = Sweep<typename O::VelStretch, T>::launch(p, tgt, c.m, c.tgt_begin, src, c.n, part,
                                                      c.st);
      }
      if (!rc)
        rc = finalize_vec<T, FIN_VELSTRETCH, O::VelStretch::NV>(part, p.splits, c.m, tgt, c.out,
                                                               c.out2, c.st);
      return rc;
    case VPM_OP_LES_STEP_SUMS: {
      using Op = typename O::LesStep;
      rc = VPM_OK;
      if (p.pairs) {
        if constexpr (LaneTraits<T>::kLanes == 2)
          rc = RotSweep<typename O::LesStepBoth>::launch(p, src, c.n, part, c.st);
        else
          rc = RotSweep<typename O::LesStepBoth64>::launch(p, src, c.n, part, c.st);
      }
      if (!p.pairs) rc = Sweep<Op, T>::launch(p, tgt, c.m, c.tgt_begin, src, c.n, part, c.st);
      if (rc) return rc;
      double scale = 1.0 / (8.0 * kPi);
      if (c.ref_extra_4pi) scale /= 4.0 * kPi;
      if (p.pairs) {
        // both sides: the per-target scalar sum_j ke (a_i . a_j) (value 12), taken once per
        // unordered pair, so the sum is doubled
        constexpr int NVB = O::LesStepBoth::NV;
        static_assert(O::LesStepBoth64::NV == NVB, "one row layout for both precisions");
        rc = finalize_vec<T, FIN_LES, NVB>(part, p.splits, c.m, tgt, c.out, c.out2, c.st,
                                           c.out3);
        if (rc) return rc;
        finalize_sum_kernel<NVB, 12><<<1, kReduceThreads, 0, c.st>>>(part, p.splits, c.m,
                                                                     2.0 * scale, c.out4);
      } else {
        rc = finalize_vec<T, FIN_LES, Op::NV>(part, p.splits, c.m, tgt, c.out, c.out2, c.st,
                                               c.out3);
        if (rc) return rc;
        finalize_dot_kernel<T, Op::NV, 12><<<1, kReduceThreads, 0, c.st>>>(part, p.splits, c.m,
                                                                            tgt, scale, c.out4);
      }
      cudaError_t e = cudaGetLastError();
      return e == cudaSuccess ? VPM_OK : cuda_fail(e, "reduce launch");
    }
    case VPM_OP_TOTAL_KINETIC_ENERGY:
    case VPM_OP_TOTAL_HELICITY:
    case VPM_OP_TOTAL_ENSTROPHY: {
      double scale = 0.0;
      if (c.op == VPM_OP_TOTAL_KINETIC_ENERGY) {
        rc = Sweep<typename O::Ke, T>::launch(p, tgt, c.m, c.tgt_begin, src, c.n, part, c.st);
        scale = 1.0 / (16.0 * kPi);
      } else if (c.op == VPM_OP_TOTAL_HELICITY) {
        rc = Sweep<typename O::Vel, T>::launch(p, tgt, c.m, c.tgt_begin, src, c.n, part, c.st);
        scale = -1.0 / (4.0 * kPi);
        if (c.ref_extra_4pi) scale /= 4.0 * kPi;
      } else {
        rc = Sweep<typename O::Ens, T>::launch(p, tgt, c.m, c.tgt_begin, src, c.n, part, c.st);
        scale = 1.0 / (8.0 * kPi);
        if (c.ref_extra_4pi) scale /= 4.0 * kPi;
      }
      if (rc) return rc;
      finalize_dot_kernel<T><<<1, kReduceThreads, 0, c.st>>>(part, p.splits, c.m, tgt, scale,
                                                             c.out);
      cudaError_t e = cudaGetLastError();
      return e == cudaSuccess ? VPM_OK : cuda_fail(e, "reduce launch");
    }
    default:
      return fail(VPM_ERR_ARG, "unknown op " + std::to_string(c.op));
  }
}

// ---- LES test filter (least-squares dynamic coefficient) ----------------------------------
template <class E>
__global__ void pack_filter_kernel(const double* __restrict__ pos, const double* __restrict__ str,
                                   const double* __restrict__ rad, const double* __restrict__ f,
                                   int64_t n, RecF<E>* __restrict__ out) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  RecF<E> r;
  set_elem(r.x, pos[3 * i]);
  set_elem(r.y, pos[3 * i + 1]);
  set_elem(r.z, pos[3 * i + 2]);
  set_elem(r.s, rad[i]);
  set_elem(r.ax, str[3 * i]);
  set_elem(r.ay, str[3 * i + 1]);
  set_elem(r.az, str[3 * i + 2]);
  set_elem(r.f1, f[3 * i]);
  set_elem(r.f2, f[3 * i + 1]);
  set_elem(r.pad, 0.0);
  out[i] = r;
}

// w_hat (m,3) and the two filtered fields (m,3; third column 0), both with the zeta kernel's
// 7.5/(4 pi) as in vpm_vorticity_field_at.
template <class T>
__global__ void finalize_filter_kernel(const double* __restrict__ part, int splits, int64_t m,
                                       double* __restrict__ w_hat, double* __restrict__ f_hat) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= m) return;
  double v[5];
  sum_splits<5>(part, splits, m, i, v);
  const double c = 7.5 * kOneOver4Pi;
  w_hat[3 * i] = v[0] * c;
  w_hat[3 * i + 1] = v[1] * c;
  w_hat[3 * i + 2] = v[2] * c;
  f_hat[3 * i] = v[3] * c;
  f_hat[3 * i + 1] = v[4] * c;
  f_hat[3 * i + 2] = 0.0;
}

template <class T, bool REFINE>
int run_filter(const Call& c) {
  using Op = OpTestFilter<T, REFINE>;
  int rc = check_arch();
  if (rc) return rc;
  if (c.n == 0) return VPM_OK;
  Plan p;
  Layout L;
  rc = workspace_for<T, REFINE>(c.op, c.n, c.n, &L, &p, c.max_partial_bytes);
  if (rc) return rc;
  if (c.ws == nullptr) return fail(VPM_ERR_WORKSPACE, "workspace is null");
  if (reinterpret_cast<uintptr_t>(c.ws) % kAlign != 0)
    return fail(VPM_ERR_ALIGN, "workspace must be 256-byte aligned");
  if (c.ws_bytes < L.total)
    return fail(VPM_ERR_WORKSPACE, "workspace has " + std::to_string(c.ws_bytes) +
                                       " bytes, needs " + std::to_string(L.total));
  char* ws = static_cast<char*>(c.ws);
  RecF<T>* rec = reinterpret_cast<RecF<T>*>(ws + L.src_off);
  double* part = reinterpret_cast<double*>(ws + L.part_off);
  const unsigned blocks = unsigned((c.n + 255) / 256);
  pack_filter_kernel<T><<<blocks, 256, 0, c.st>>>(c.pos, c.str, c.rad, c.aux, c.n, rec);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "pack launch");
  rc = Sweep<Op, T>::launch(p, rec, c.n, 0, rec, c.n, part, c.st);
  if (rc) return rc;
  finalize_filter_kernel<T><<<blocks, 256, 0, c.st>>>(part, p.splits, c.n, c.out, c.out2);
  e = cudaGetLastError();
  return e == cudaSuccess ? VPM_OK : cuda_fail(e, "finalize launch");
}

// Decoded precision code: compute type, Newton-refined rsqrt, uniform cores.
template <class T, bool REFINE, bool UC>
struct Prec {
  using type = T;
  static constexpr bool refine = REFINE, uc = UC;
};

template <class F>
int with_precision(int precision, F&& f) {
  const bool uc = (precision & VPM_UNIFORM_CORE) != 0;
  switch (precision & ~VPM_UNIFORM_CORE) {
    case VPM_FP64:
      return uc ? f(Prec<double, false, true>{}) : f(Prec<double, false, false>{});
    case VPM_FP32C:
      return uc ? f(Prec<float2, false, true>{}) : f(Prec<float2, false, false>{});
    case VPM_FP32C_REFINED:
      return uc ? f(Prec<float2, true, true>{}) : f(Prec<float2, true, false>{});
    default:
      return fail(VPM_ERR_ARG, "unknown precision " + std::to_string(precision));
  }
}

int dispatch(const Call& c, int precision) {
  if (c.n < 0 || c.m < 0) return fail(VPM_ERR_ARG, "negative size");
  if (c.records) {
    if (is_probe(c.op)) return fail(VPM_ERR_ARG, "record entry points are for self sums");
    if (c.tgt_begin < 0 || c.tgt_begin + c.m > c.n)
      return fail(VPM_ERR_ARG, "target range outside the records");
    if (reinterpret_cast<uintptr_t>(c.records) % 16 != 0)
      return fail(VPM_ERR_ALIGN, "records must be 16-byte aligned");
  } else {
    if (c.n > 0 && (!c.pos || !c.rad)) return fail(VPM_ERR_ARG, "null input pointer");
    if (c.n > 0 && !c.str) return fail(VPM_ERR_ARG, "null strengths pointer");
  }
  if (c.m > 0 && !c.out) return fail(VPM_ERR_ARG, "null output pointer");
  if (is_probe(c.op) && c.m > 0 && !c.tgt) return fail(VPM_ERR_ARG, "null targets pointer");
  if (c.op == VPM_OP_STRENGTH_GRADIENTS_PSE && c.n > 0 && !c.nu && !c.records)
    return fail(VPM_ERR_ARG, "null viscosities pointer");
  if ((c.op == VPM_OP_VELOCITY_AND_STRENGTH_GRADIENTS || c.op == VPM_OP_LES_STEP_SUMS) &&
      c.m > 0 && !c.out2)
    return fail(VPM_ERR_ARG, "null second output pointer");
  if (c.op == VPM_OP_LES_STEP_SUMS && ((c.m > 0 && !c.out3) || !c.out4))
    return fail(VPM_ERR_ARG, "null vorticity or enstrophy pointer");
  return with_precision(precision, [&](auto P) {
    using Pp = decltype(P);
    return run<typename Pp::type, Pp::refine, Pp::uc>(c);
  });
}

struct GradCall {
  int op;
  const double *pos, *str, *rad, *nu, *gu, *gs;
  int64_t n;
  double *ox, *oa, *os, *onu;
  void* ws;
  size_t ws_bytes;
  cudaStream_t st;
};

template <class T, bool REFINE>
int run_grad(const GradCall& c) {
  using O = Ops<T, REFINE>;
  int rc = check_arch();
  if (rc) return rc;
  if (c.n == 0) return VPM_OK;
  Plan p;
  Layout L;
  rc = workspace_for<T, REFINE>(c.op, c.n, c.n, &L, &p);
  if (rc) return rc;
  if (c.ws == nullptr) return fail(VPM_ERR_WORKSPACE, "workspace is null");
  if (reinterpret_cast<uintptr_t>(c.ws) % kAlign != 0)
    return fail(VPM_ERR_ALIGN, "workspace must be 256-byte aligned");
  if (c.ws_bytes < L.total)
    return fail(VPM_ERR_WORKSPACE, "workspace has " + std::to_string(c.ws_bytes) +
                                       " bytes, needs " + std::to_string(L.total));
  char* ws = static_cast<char*>(c.ws);
  double* part = reinterpret_cast<double*>(ws + L.part_off);
  const unsigned blocks = unsigned((c.n + 255) / 256);
  cudaError_t e;
  if (c.op == VPM_OP_KINETIC_ENERGY_GRAD) {
    Rec<T>* rec = reinterpret_cast<Rec<T>*>(ws + L.src_off);
    rc = pack<T>(c.pos, c.str, c.rad, nullptr, c.n, rec, c.st);
    if (!rc) rc = Sweep<typename O::KeGrad, T>::launch(p, rec, c.n, 0, rec, c.n, part, c.st);
    if (rc) return rc;
    finalize_kegrad_kernel<<<blocks, 256, 0, c.st>>>(part, p.splits, c.n, c.ox, c.oa, c.os);
    e = cudaGetLastError();
    return e == cudaSuccess ? VPM_OK : cuda_fail(e, "finalize launch");
  }
  RecG<T>* rec = reinterpret_cast<RecG<T>*>(ws + L.src_off);
  pack_grad_kernel<T><<<blocks, 256, 0, c.st>>>(c.pos, c.str, c.rad, c.nu, c.gu, c.gs, c.n, rec);
  e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "pack launch");
  if (c.op == VPM_OP_RHS_VJP_PSE) {
    rc = VPM_OK;
    if constexpr (LaneTraits<T>::kLanes == 2) {
      if (p.pairs) rc = RotSweep<typename O::RhsVjpPseBoth>::launch(p, rec, c.n, part, c.st);
    }
    if (!p.pairs)
      rc = Sweep<typename O::RhsVjpPse, T>::launch(p, rec, c.n, 0, rec, c.n, part, c.st);
    if (rc) return rc;
    finalize_vjp_kernel<T, O::RhsVjpPse::NV, true>
        <<<blocks, 256, 0, c.st>>>(part, p.splits, c.n, rec, c.ox, c.oa, c.os, c.onu);
  } else {
    rc = VPM_OK;
    if constexpr (LaneTraits<T>::kLanes == 2) {
      if (p.pairs) rc = RotSweep<typename O::RhsVjpBoth>::launch(p, rec, c.n, part, c.st);
    }
    if (!p.pairs) rc = Sweep<typename O::RhsVjp, T>::launch(p, rec, c.n, 0, rec, c.n, part, c.st);
    if (rc) return rc;
    finalize_vjp_kernel<T, O::RhsVjp::NV, false>
        <<<blocks, 256, 0, c.st>>>(part, p.splits, c.n, rec, c.ox, c.oa, c.os, c.onu);
  }
  e = cudaGetLastError();
  return e == cudaSuccess ? VPM_OK : cuda_fail(e, "finalize launch");
}

int dispatch_grad(const GradCall& c, int precision) {
  precision &= ~VPM_UNIFORM_CORE;  // the adjoint keeps the general pair core
  if (c.n < 0) return fail(VPM_ERR_ARG, "negative size");
  if (c.n > 0 && (!c.pos || !c.str || !c.rad || !c.ox || !c.oa || !c.os))
    return fail(VPM_ERR_ARG, "null pointer");
  if (c.op != VPM_OP_KINETIC_ENERGY_GRAD && c.n > 0 && (!c.gu || !c.gs))
    return fail(VPM_ERR_ARG, "null cotangent pointer");
  switch (precision) {
    case VPM_FP64:
      return run_grad<double, false>(c);
    case VPM_FP32C:
      return run_grad<float2, false>(c);
    case VPM_FP32C_REFINED:
      return run_grad<float2, true>(c);
    default:
      return fail(VPM_ERR_ARG, "unknown precision " + std::to_string(precision));
  }
}


// ---- scratch for the no-allocation entry point --------------------------------------------
// Some callers may not allocate device memory at all: a solver plugin that runs inside a
// host application which owns the whole GPU memory budget through its own pool, or a
// fixed-latency loop where a cudaMalloc (which may synchronise the device, and fails once
// memory is exhausted) is not permitted.  For them one entry point takes its scratch from
// this array, which the library image reserves on every GPU that loads it, until exit.
// Host code must not use the array's name as a device address: the address is fetched per
// device with cudaGetSymbolAddress.
constexpr int64_t kNoAllocMaxN = VPM_NOALLOC_MAX_N;
constexpr size_t kNoAllocScratchBytes = VPM_NOALLOC_SCRATCH_BYTES;
constexpr size_t kNoAllocRecordBytes = size_t(kNoAllocMaxN) * 64;  // packed records
static_assert(kNoAllocRecordBytes % kAlign == 0, "record region stays 256-byte aligned");
static_assert(kNoAllocScratchBytes > kNoAllocRecordBytes, "room for partials");

// (device, driver context) -> device address of the scratch in that context.  A __device__
// array has one address per context, so a host application that makes another context
// current on the same device gets its own lookup.
std::map<std::pair<int, void*>, void*> g_noalloc_addr;

int noalloc_scratch(void** out);

// ---- bounded-wait self-test -----------------------------------------------------------------
// One block waits on an mbarrier phase that nothing completes (16 transaction bytes are
// expected and never sent).  mbar_wait_bounded gives up after its time limit, records
// VPM_DEVERR_WAIT_TIMEOUT and the kernel returns: the same path a sweep takes when a tile copy
// never lands.  No copy is issued, so nothing is in flight when the block exits.
__global__ void bounded_wait_selftest_kernel(int* __restrict__ result) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    fence_mbar_init();
  }
  __syncthreads();
  if (threadIdx.x == 0) mbar_arrive_expect_tx(&bar, 16);
  __syncthreads();
  const bool ok = mbar_wait_bounded(&bar, 0);
  if (__syncthreads_or(!ok) && threadIdx.x == 0) result[0] = 1;
}

// ---- FMA throughput kernels ------------------------------------------------------------
template <class T>
__global__ void fma_peak_kernel(int iters, T* sink) {
  T a[16];
  const T m = T(1.0) - T(1e-7) * T(threadIdx.x & 7);
  const T b = T(1e-9) * T(blockIdx.x & 3);
#pragma unroll
  for (int k = 0; k < 16; ++k) a[k] = T(threadIdx.x + k);
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int k = 0; k < 16; ++k) a[k] = fma(a[k], m, b);
  }
  T s = 0;
#pragma unroll
  for (int k = 0; k < 16; ++k) s += a[k];
  sink[int64_t(blockIdx.x) * blockDim.x + threadIdx.x] = s;
}

// Packed FP32 FMA throughput: 16 independent chains of FFMA2 (two FP32 lanes each).
__global__ void ffma2_peak_kernel(int iters, float* sink) {
  float2 a[16];
  const float2 m = make_float2(1.0f - 1e-7f * float(threadIdx.x & 7), 1.0f - 2e-7f);
  const float2 b = make_float2(1e-9f * float(blockIdx.x & 3), 1e-9f);
#pragma unroll
  for (int k = 0; k < 16; ++k) a[k] = make_float2(float(threadIdx.x + k), float(k));
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int k = 0; k < 16; ++k) a[k] = fma(a[k], m, b);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 16; ++k) s += a[k].x + a[k].y;
  sink[int64_t(blockIdx.x) * blockDim.x + threadIdx.x] = s;
}

// Mixed FP32 FMA throughput: 8 packed FFMA2 chains and 16 scalar FFMA chains per thread (32
// lane FMAs per iteration in 24 instructions).
__global__ void ffma_mixed_peak_kernel(int iters, float* sink) {
  float2 a[8];
  float c[16];
  const float2 m = make_float2(1.0f - 1e-7f * float(threadIdx.x & 7), 1.0f - 2e-7f);
  const float2 b = make_float2(1e-9f * float(blockIdx.x & 3), 1e-9f);
#pragma unroll
  for (int k = 0; k < 8; ++k) a[k] = make_float2(float(threadIdx.x + k), float(k));
#pragma unroll
  for (int k = 0; k < 16; ++k) c[k] = float(threadIdx.x + 2 * k);
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      a[k] = fma(a[k], m, b);
      c[2 * k] = fmaf(c[2 * k], m.x, b.x);
      c[2 * k + 1] = fmaf(c[2 * k + 1], m.y, b.y);
    }
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += a[k].x + a[k].y + c[2 * k] + c[2 * k + 1];
  sink[int64_t(blockIdx.x) * blockDim.x + threadIdx.x] = s;
}

// MUFU (SFU) throughput: 16 independent chains of rsqrt.approx per thread; the one FADD per
// step runs on the FMA pipe, which has 8x the lanes of the SFU, so the SFU bounds the loop.
__global__ void rsqrt_peak_kernel(int iters, float* sink) {
  float a[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) a[k] = 1.0f + 1e-3f * float(threadIdx.x) + float(k);
  for (int it = 0; it < iters; ++it) {
#pragma unroll
    for (int k = 0; k < 16; ++k) a[k] = rsqrt_approx(a[k] + 0.5f);
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 16; ++k) s += a[k];
  sink[int64_t(blockIdx.x) * blockDim.x + threadIdx.x] = s;
}

}  // namespace

// File-scope scratch of vpm_selfinduced_velocity_noalloc (see noalloc_scratch).
static __device__ __align__(256) unsigned char g_noalloc_scratch[VPM_NOALLOC_SCRATCH_BYTES];

namespace {
// The driver context current on the calling thread (cuCtxGetCurrent, reached through the
// runtime's driver entry-point table so the library needs no link against libcuda).
int current_context(void** ctx) {
  using CtxGetCurrent = CUresult (*)(CUcontext*);
  static CtxGetCurrent fn = nullptr;
  static std::once_flag once;
  static cudaError_t lookup = cudaSuccess;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
    lookup = cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q);
    if (lookup == cudaSuccess && q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<CtxGetCurrent>(p);
  });
  if (lookup != cudaSuccess) return cuda_fail(lookup, "cudaGetDriverEntryPoint(cuCtxGetCurrent)");
  if (!fn) return fail(VPM_ERR_CUDA, "cuCtxGetCurrent not found in the driver");
  CUcontext c = nullptr;
  if (fn(&c) != CUDA_SUCCESS || !c) return fail(VPM_ERR_CUDA, "no current CUDA context");
  *ctx = c;
  return VPM_OK;
}

// Device address of g_noalloc_scratch in the current context, looked up once per (device,
// context) with that context current, and cached.
int noalloc_scratch(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
  void* ctx = nullptr;
  int rc = current_context(&ctx);
  if (rc) return rc;
  std::lock_guard<std::mutex> lk(g_mu);
  const auto key = std::make_pair(dev, ctx);
  auto it = g_noalloc_addr.find(key);
  if (it == g_noalloc_addr.end()) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-allocation scratch)");
    it = g_noalloc_addr.emplace(key, p).first;
  }
  *out = it->second;
  return VPM_OK;
}
}  // namespace
}  // namespace vpm

using namespace vpm;

// ---- pair shards across GPUs: the fused sum's both-sides schedule split by tile ranges ----
// Calls f(RotSweep<X>{}, plan) for the both-sides build the planner takes for a self sum of n
// particles (every rank plans the same n, so all ranks use the same tiles and launch sizes).
template <class T, bool REFINE, bool UC, class F>
int with_fused_both(int64_t n, F&& f) {
  using O = Ops<T, REFINE, UC>;
  Plan p;
  int rc = plan_op<T, REFINE, UC>(VPM_OP_VELOCITY_AND_STRENGTH_GRADIENTS, n, n, &p);
  if (rc) return rc;
  if (!p.pairs)
    return fail(VPM_ERR_ARG, "n = " + std::to_string(n) +
                                 " does not take the both-sides schedule "
                                 "(vpm_set_symmetric_min_n); shard the targets instead");
  if constexpr (LaneTraits<T>::kLanes != 2) {
    return f(RotSweep<typename O::VelStretchBoth64>{}, p);
  } else {
    if (p.variant == 2) return f(RotSweep<typename O::VelStretchBothSmall>{}, p);
    if (p.variant == 1) return f(RotSweep<typename O::VelStretchBothAlt>{}, p);
    return f(RotSweep<typename O::VelStretchBoth>{}, p);
  }
}

extern "C" {

int vpm_abi_version(void) { return VPM_ABI_VERSION; }

const char* vpm_last_error(void) { return g_last_error.c_str(); }

int vpm_check_device(void) { return check_arch(); }

int vpm_binary_info(int* binary_version, int* ptx_version) {
  if (!binary_version || !ptx_version) return fail(VPM_ERR_ARG, "null result pointer");
  cudaFuncAttributes fa;
  cudaError_t e = cudaFuncGetAttributes(&fa, reinterpret_cast<const void*>(&zero_kernel));
  if (e != cudaSuccess) return cuda_fail(e, "cudaFuncGetAttributes");
  *binary_version = fa.binaryVersion;
  *ptx_version = fa.ptxVersion;
  return VPM_OK;
}

int vpm_device_errors(int* out, int clear) {
  int v = 0;
  cudaError_t e = cudaMemcpyFromSymbol(&v, g_device_errors, sizeof(int));
  if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyFromSymbol");
  if (out) *out = v;
  if (clear) {
    const int z = 0;
    e = cudaMemcpyToSymbol(g_device_errors, &z, sizeof(int));
    if (e != cudaSuccess) return cuda_fail(e, "cudaMemcpyToSymbol");
  }
  return VPM_OK;
}

size_t vpm_workspace_bytes(int op, int precision, int64_t m, int64_t n) {
  if (op == VPM_OP_RHS_VJP || op == VPM_OP_RHS_VJP_PSE || op == VPM_OP_KINETIC_ENERGY_GRAD)
    precision &= ~VPM_UNIFORM_CORE;
  size_t total = 0;
  const int rc = with_precision(precision, [&](auto P) {
    using Pp = decltype(P);
    Plan p;
    Layout L;
    const int r = workspace_for<typename Pp::type, Pp::refine, Pp::uc>(op, m, n, &L, &p);
    if (!r) total = L.total;
    return r;
  });
  return rc ? 0 : total;
}

int vpm_pairs_layout(int op, int precision, int64_t n, int64_t* tiles, int64_t* pairs,
                     int* pairs_per_launch, int* values, size_t* workspace_bytes) {
  if (op != VPM_OP_VELOCITY_AND_STRENGTH_GRADIENTS)
    return fail(VPM_ERR_ARG, "pair shards are built for the fused velocity + stretching sum");
  if (n < 0) return fail(VPM_ERR_ARG, "negative size");
  return with_precision(precision, [&](auto P) {
    using Pp = decltype(P);
    return with_fused_both<typename Pp::type, Pp::refine, Pp::uc>(n, [&](auto rs,
                                                                        const Plan& p) {
      using RS = decltype(rs);
      const int64_t nt = RS::tiles(n);
      if (tiles) *tiles = nt;
      if (pairs) *pairs = nt / 2;
      if (pairs_per_launch) *pairs_per_launch = p.pairs;
      if (values) *values = RS::NV;
      if (workspace_bytes) *workspace_bytes = size_t(RS::sets(p.pairs)) * RS::set_bytes(n);
      return VPM_OK;
    });
  });
}

int vpm_sweep_pairs_partial(int op, const void* records, int64_t n, int64_t tile_begin,
                            int64_t tile_end, int64_t pair_begin, int64_t pair_end,
                            double* rows, int precision, void* workspace,
                            size_t workspace_bytes, void* stream) {
  if (op != VPM_OP_VELOCITY_AND_STRENGTH_GRADIENTS)
    return fail(VPM_ERR_ARG, "pair shards are built for the fused velocity + stretching sum");
  if (n <= 0) return fail(VPM_ERR_ARG, "n must be positive");
  if (!records || !rows || !workspace) return fail(VPM_ERR_ARG, "null pointer");
  if (reinterpret_cast<uintptr_t>(records) % 16 != 0)
    return fail(VPM_ERR_ALIGN, "records must be 16-byte aligned");
  if (reinterpret_cast<uintptr_t>(workspace) % kAlign != 0)
    return fail(VPM_ERR_ALIGN, "workspace must be 256-byte aligned");
  int rc = check_arch();
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  return with_precision(precision, [&](auto P) {
    using Pp = decltype(P);
    return with_fused_both<typename Pp::type, Pp::refine, Pp::uc>(n, [&](auto rs,
                                                                        const Plan& p) {
      using RS = decltype(rs);
      const int64_t nt = RS::tiles(n);
      if (tile_begin < 0 || tile_end < tile_begin || tile_end > nt)
        return fail(VPM_ERR_ARG, "tile range outside [0, " + std::to_string(nt) + ")");
      if (pair_begin < 0 || pair_end < pair_begin || pair_end > nt / 2)
        return fail(VPM_ERR_ARG, "pair range outside [0, " + std::to_string(nt / 2) + ")");
      const size_t need = size_t(RS::sets(p.pairs)) * RS::set_bytes(n);
      if (workspace_bytes < need)
        return fail(VPM_ERR_WORKSPACE, "workspace has " + std::to_string(workspace_bytes) +
                                           " bytes, needs " + std::to_string(need));
      double* acc = static_cast<double*>(workspace);
      int r = RS::launch_part(p, records, n, acc, int(tile_begin), int(tile_end),
                              int(pair_begin) + 1, int(pair_end) + 1, st);
      if (r) return r;
      sets_to_rows_kernel<RS::NV><<<unsigned((n + 255) / 256), 256, 0, st>>>(
          acc, int(RS::sets(p.pairs)), n, rows);
      cudaError_t e = cudaGetLastError();
      return e == cudaSuccess ? VPM_OK : cuda_fail(e, "rows launch");
    });
  });
}

int vpm_finalize_pairs_partial(int op, const double* rows, const void* records,
                               int64_t target_begin, int64_t m, double* out, double* out2,
                               int precision, void* stream) {
  if (op != VPM_OP_VELOCITY_AND_STRENGTH_GRADIENTS)
    return fail(VPM_ERR_ARG, "pair shards are built for the fused velocity + stretching sum");
  if (m < 0 || target_begin < 0) return fail(VPM_ERR_ARG, "negative size or offset");
  if (m == 0) return VPM_OK;
  if (!rows || !records || !out || !out2) return fail(VPM_ERR_ARG, "null pointer");
  if (reinterpret_cast<uintptr_t>(records) % 16 != 0)
    return fail(VPM_ERR_ALIGN, "records must be 16-byte aligned");
  int rc = check_arch();
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  static_assert(OpVelStretchBoth<false, false>::NV == 9 && OpVelStretchBoth64<false>::NV == 9,
                "the fused sum's 9 values per row");
  const unsigned blocks = unsigned((m + 255) / 256);
  switch (precision & ~VPM_UNIFORM_CORE) {
    case VPM_FP64:
      finalize_rows_kernel<double, FIN_VELSTRETCH, 9><<<blocks, 256, 0, st>>>(
          rows, m, static_cast<const Rec<double>*>(records) + target_begin, out, out2);
      break;
    case VPM_FP32C:
    case VPM_FP32C_REFINED:
      finalize_rows_kernel<float2, FIN_VELSTRETCH, 9><<<blocks, 256, 0, st>>>(
          rows, m, static_cast<const Rec<float2>*>(records) + target_begin, out, out2);
      break;
    default:
      return fail(VPM_ERR_ARG, "unknown precision " + std::to_string(precision));
  }
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? VPM_OK : cuda_fail(e, "finalize launch");
}

int vpm_plan_info(int op, int precision, int64_t m, int64_t n, int64_t* target_blocks,
                  int* splits, int* threads, int* targets_per_thread) {
  if (op == VPM_OP_RHS_VJP || op == VPM_OP_RHS_VJP_PSE || op == VPM_OP_KINETIC_ENERGY_GRAD)
    precision &= ~VPM_UNIFORM_CORE;
  Plan p;
  const int rc = with_precision(precision, [&](auto P) {
    using Pp = decltype(P);
    return plan_op<typename Pp::type, Pp::refine, Pp::uc>(op, m, n, &p);
  });
  if (rc) return rc;
  if (target_blocks) *target_blocks = p.tblocks;
  if (splits) *splits = p.splits;
  if (threads) *threads = p.threads;
  if (targets_per_thread) *targets_per_thread = p.r;
  return VPM_OK;
}

int vpm_induced_velocity_at(const double* targets, int64_t m, const double* positions,
                            const double* strengths, const double* radii, int64_t n,
                            double* velocities, int precision, void* workspace,
                            size_t workspace_bytes, void* stream) {
  Call c{VPM_OP_INDUCED_VELOCITY_AT, targets, m, positions, strengths, radii, nullptr, n,
         velocities, nullptr, 0, workspace, workspace_bytes, static_cast<cudaStream_t>(stream)};
  return dispatch(c, precision);
}

int vpm_selfinduced_velocity(const double* positions, const double* strengths,
                             const double* radii, int64_t n, double* velocities, int precision,
                             void* workspace, size_t workspace_bytes, void* stream) {
  Call c{VPM_OP_SELFINDUCED_VELOCITY, nullptr, n, positions, strengths, radii, nullptr, n,
         velocities, nullptr, 0, workspace, workspace_bytes, static_cast<cudaStream_t>(stream)};
  return dispatch(c, precision);
}

int vpm_vorticity_field_at(const double* targets, int64_t m, const double* positions,
                           const double* strengths, const double* radii, int64_t n,
                           double* vorticities, int precision, void* workspace,
                           size_t workspace_bytes, void* stream) {
  Call c{VPM_OP_VORTICITY_FIELD_AT, targets, m, positions, strengths, radii, nullptr, n,
         vorticities, nullptr, 0, workspace, workspace_bytes, static_cast<cudaStream_t>(stream)};
  return dispatch(c, precision);
}

int vpm_strength_gradients(const double* positions, const double* strengths,
                           const double* radii, int64_t n, double* dalpha_dt, int precision,
                           void* workspace, size_t workspace_bytes, void* stream) {
  Call c{VPM_OP_STRENGTH_GRADIENTS, nullptr, n, positions, strengths, radii, nullptr, n,
         dalpha_dt, nullptr, 0, workspace, workspace_bytes, static_cast<cudaStream_t>(stream)};
  return dispatch(c, precision);
}

int vpm_strength_gradients_pse(const double* positions, const double* strengths,
                               const double* radii, const double* viscosities, int64_t n,
                               double* dalpha_dt, int precision, void* workspace,
                               size_t workspace_bytes, void* stream) {
  Call c{VPM_OP_STRENGTH_GRADIENTS_PSE, nullptr, n, positions, strengths, radii, viscosities, n,
         dalpha_dt, nullptr, 0, workspace, workspace_bytes, static_cast<cudaStream_t>(stream)};
  return dispatch(c, precision);
}

int vpm_total_kinetic_energy(const double* positions, const double* strengths,
                             const double* radii, int64_t n, double* energy, int precision,
                             void* workspace, size_t workspace_bytes, void* stream) {
  if (!energy) return fail(VPM_ERR_ARG, "null output pointer");
  Call c{VPM_OP_TOTAL_KINETIC_ENERGY, nullptr, n, positions, strengths, radii, nullptr, n,
         energy, nullptr, 0, workspace, workspace_bytes, static_cast<cudaStream_t>(stream)};
  return dispatch(c, precision);
}

int vpm_total_helicity(const double* positions, const double* strengths, const double* radii,
                       int64_t n, int ref_extra_4pi, double* helicity, int precision,
                       void* workspace, size_t workspace_bytes, void* stream) {
  if (!helicity) return fail(VPM_ERR_ARG, "null output pointer");
  Call c{VPM_OP_TOTAL_HELICITY, nullptr, n, positions, strengths, radii, nullptr, n,
         helicity, nullptr, ref_extra_4pi, workspace, workspace_bytes,
         static_cast<cudaStream_t>(stream)};
  return dispatch(c, precision);
}

int vpm_total_enstrophy(const double* positions, const double* strengths, const double* radii,
                        int64_t n, int ref_extra_4pi, double* enstrophy, int precision,
                        void* workspace, size_t workspace_bytes, void* stream) {
  if (!enstrophy) return fail(VPM_ERR_ARG, "null output pointer");
  Call c{VPM_OP_TOTAL_ENSTROPHY, nullptr, n, positions, strengths, radii, nullptr, n,
         enstrophy, nullptr, ref_extra_4pi, workspace, workspace_bytes,
         static_cast<cudaStream_t>(stream)};
  return dispatch(c, precision);
}

int vpm_velocity_and_strength_gradients(const double* positions, const double* strengths,
                                        const double* radii, int64_t n, double* velocities,
                                        double* dalpha_dt, int precision, void* workspace,
                                        size_t workspace_bytes, void* stream) {
  Call c{VPM_OP_VELOCITY_AND_STRENGTH_GRADIENTS, nullptr, n, positions, strengths, radii,
         nullptr, n, velocities, dalpha_dt, 0, workspace, workspace_bytes,
         static_cast<cudaStream_t>(stream)};
  return dispatch(c, precision);
}

int64_t vpm_set_symmetric_min_n(int64_t n) { return g_sym_min_n.exchange(n); }

int64_t vpm_sweep_launches(int op, int precision, int64_t m, int64_t n) {
  if (m <= 0 || n <= 0) return 0;
  if (op == VPM_OP_RHS_VJP || op == VPM_OP_RHS_VJP_PSE || op == VPM_OP_KINETIC_ENERGY_GRAD)
    precision &= ~VPM_UNIFORM_CORE;
  Plan p;
  const int rc = with_precision(precision, [&](auto P) {
    using Pp = decltype(P);
    return plan_op<typename Pp::type, Pp::refine, Pp::uc>(op, m, n, &p);
  });
  if (rc) return -1;
  if (p.pairs) {  // zero the accumulators, the diagonal tiles, the diagonal-pair launches, finalize
    const int64_t npairs = p.tblocks / 2;
    return 3 + (npairs + p.pairs - 1) / p.pairs;
  }
  return 2;  // sweep, finalize (or the single-block reduction of a scalar)
}

int vpm_les_step_sums(const double* positions, const double* strengths, const double* radii,
                      int64_t n, double* velocities, double* dalpha_dt, double* vorticity,
                      double* enstrophy, int ref_extra_4pi, int precision, void* workspace,
                      size_t workspace_bytes, void* stream) {
  Call c{VPM_OP_LES_STEP_SUMS, nullptr, n, positions, strengths, radii,
         nullptr, n, velocities, dalpha_dt, ref_extra_4pi, workspace, workspace_bytes,
         static_cast<cudaStream_t>(stream)};
  c.out3 = vorticity;
  c.out4 = enstrophy;
  return dispatch(c, precision);
}

int vpm_les_test_filter(const double* positions, const double* strengths,
                        const double* test_radii, const double* fields, int64_t n,
                        double* test_vorticity, double* test_filtered, int precision,
                        void* workspace, size_t workspace_bytes, void* stream) {
  if (n < 0) return fail(VPM_ERR_ARG, "negative size");
  if (n > 0 && (!positions || !strengths || !test_radii || !fields || !test_vorticity ||
                !test_filtered))
    return fail(VPM_ERR_ARG, "null pointer");
  Call c{VPM_OP_LES_TEST_FILTER, nullptr, n, positions, strengths, test_radii, nullptr, n,
         test_vorticity, test_filtered, 0, workspace, workspace_bytes,
         static_cast<cudaStream_t>(stream)};
  c.aux = fields;
  switch (precision & ~VPM_UNIFORM_CORE) {
    case VPM_FP64:
      return run_filter<double, false>(c);
    case VPM_FP32C:
      return run_filter<float2, false>(c);
    case VPM_FP32C_REFINED:
      return run_filter<float2, true>(c);
    default:
      return fail(VPM_ERR_ARG, "unknown precision " + std::to_string(precision));
  }
}

size_t vpm_record_bytes(int precision) {
  switch (precision & ~VPM_UNIFORM_CORE) {
    case VPM_FP64:
      return sizeof(Rec<double>);
    case VPM_FP32C:
    case VPM_FP32C_REFINED:
      return sizeof(Rec<float2>);
    default:
      fail(VPM_ERR_ARG, "unknown precision");
      return 0;
  }
}

int vpm_pack_records(const double* positions, const double* strengths, const double* radii,
                     const double* viscosities, int64_t n, int precision, void* records,
                     void* stream) {
  if (n < 0) return fail(VPM_ERR_ARG, "negative size");
  if (n > 0 && (!positions || !strengths || !radii || !records))
    return fail(VPM_ERR_ARG, "null pointer");
  if (reinterpret_cast<uintptr_t>(records) % 16 != 0)
    return fail(VPM_ERR_ALIGN, "records must be 16-byte aligned");
  int rc = check_arch();
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const bool uc = (precision & VPM_UNIFORM_CORE) != 0;
  precision &= ~VPM_UNIFORM_CORE;
  if (precision == VPM_FP64)
    return pack<double>(positions, strengths, radii, viscosities, n,
                        static_cast<Rec<double>*>(records), st, uc);
  if (precision == VPM_FP32C || precision == VPM_FP32C_REFINED)
    return pack<float2>(positions, strengths, radii, viscosities, n,
                        static_cast<Rec<float2>*>(records), st, uc);
  return fail(VPM_ERR_ARG, "unknown precision");
}

int vpm_sweep_records(int op, const void* records, int64_t n, int64_t target_begin, int64_t m,
                      int ref_extra_4pi, double* out, double* out2, int precision,
                      void* workspace, size_t workspace_bytes, void* stream) {
  Call c{op, nullptr, m, nullptr, nullptr, nullptr, nullptr, n, out, out2, ref_extra_4pi,
         workspace, workspace_bytes, static_cast<cudaStream_t>(stream)};
  c.records = records;
  c.tgt_begin = target_begin;
  if (n > 0 && !records) return fail(VPM_ERR_ARG, "null records pointer");
  return dispatch(c, precision);
}

int vpm_rhs_vjp(const double* positions, const double* strengths, const double* radii,
                const double* viscosities, int64_t n, const double* grad_velocities,
                const double* grad_rates, double* grad_positions, double* grad_strengths,
                double* grad_radii, double* grad_viscosities, int precision, void* workspace,
                size_t workspace_bytes, void* stream) {
  GradCall c{viscosities ? VPM_OP_RHS_VJP_PSE : VPM_OP_RHS_VJP, positions, strengths, radii,
             viscosities, grad_velocities, grad_rates, n, grad_positions, grad_strengths,
             grad_radii, grad_viscosities, workspace, workspace_bytes,
             static_cast<cudaStream_t>(stream)};
  return dispatch_grad(c, precision);
}

int vpm_kinetic_energy_grad(const double* positions, const double* strengths,
                            const double* radii, int64_t n, double* grad_positions,
                            double* grad_strengths, double* grad_radii, int precision,
                            void* workspace, size_t workspace_bytes, void* stream) {
  GradCall c{VPM_OP_KINETIC_ENERGY_GRAD, positions, strengths, radii, nullptr, nullptr, nullptr,
             n, grad_positions, grad_strengths, grad_radii, nullptr, workspace,
             workspace_bytes, static_cast<cudaStream_t>(stream)};
  return dispatch_grad(c, precision);
}

// Self-induced velocity without any allocation: the scratch (packed records and per-split
// partial sums) lives in the library's static device array.  Every call shares that array
// and leaves its contents behind; nothing in it needs clearing, because each call that
// completes rewrites every record and partial it reads.  A sweep whose bounded wait gives up
// returns without writing its partials: the call's output is then built from what the
// previous call left, and only the device error word (vpm_device_errors) shows it.  Calls
// that overlap on the GPU (two streams, two host threads) race on the array.  The first call
// in a context looks up the array's address there (cudaGetSymbolAddress) and the kernels'
// occupancy; make that first call before any stream capture.
int vpm_selfinduced_velocity_noalloc(const double* positions, const double* strengths,
                                     const double* radii, int64_t n, double* velocities,
                                     int precision, void* stream) {
  if (n < 0) return fail(VPM_ERR_ARG, "negative size");
  if (n > kNoAllocMaxN)
    return fail(VPM_ERR_ARG, "n = " + std::to_string(n) +
                                 " exceeds the no-allocation limit of " +
                                 std::to_string(kNoAllocMaxN) +
                                 " particles; call vpm_selfinduced_velocity with a workspace");
  int rc = check_arch();
  if (rc) return rc;
  void* scratch = nullptr;
  rc = noalloc_scratch(&scratch);
  if (rc) return rc;
  Call c{VPM_OP_SELFINDUCED_VELOCITY, nullptr, n, positions, strengths, radii, nullptr, n,
         velocities, nullptr, 0, scratch, kNoAllocScratchBytes,
         static_cast<cudaStream_t>(stream)};
  c.max_partial_bytes = kNoAllocScratchBytes - kNoAllocRecordBytes;
  return dispatch(c, precision);
}

int vpm_selftest_bounded_wait(int* timed_out, void* stream) {
  if (!timed_out) return fail(VPM_ERR_ARG, "null result pointer");
  int rc = check_arch();
  if (rc) return rc;
  bounded_wait_selftest_kernel<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(timed_out);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? VPM_OK : cuda_fail(e, "selftest launch");
}

int vpm_launch_fma_peak(int fp64, int blocks, int threads, int iters, void* sink, void* stream) {
  if (blocks <= 0 || threads <= 0 || threads > 1024 || iters <= 0 || !sink || fp64 < 0 ||
      fp64 > 4)
    return fail(VPM_ERR_ARG, "bad fma peak launch arguments");
  int rc = check_arch();
  if (rc) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (fp64 == 4)
    ffma_mixed_peak_kernel<<<blocks, threads, 0, st>>>(iters, static_cast<float*>(sink));
  else if (fp64 == 3)
    ffma2_peak_kernel<<<blocks, threads, 0, st>>>(iters, static_cast<float*>(sink));
  else if (fp64 == 2)
    rsqrt_peak_kernel<<<blocks, threads, 0, st>>>(iters, static_cast<float*>(sink));
  else if (fp64)
    fma_peak_kernel<double><<<blocks, threads, 0, st>>>(iters, static_cast<double*>(sink));
  else
    fma_peak_kernel<float><<<blocks, threads, 0, st>>>(iters, static_cast<float*>(sink));
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? VPM_OK : cuda_fail(e, "fma peak launch");
}

}  // extern "C"

// Element-wise time-step kernels and O(N) diagnostics (same translation unit).
#include "vpm_step.cuh"

// Initial conditions and particle lattices on the device.
#include "vpm_ic.cuh"
