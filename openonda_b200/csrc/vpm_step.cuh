// vpm_step.cuh -- element-wise (HBM-bound) kernels of the device-resident time step and the
// O(N) FP64 diagnostics.  Included by vpm_abi.cu (the library is one translation unit).
//
// Each kernel restates one piece of vpmModule.ParticleSystem (OpenONDA/solvers/VPM/
// vpmModule.py) with the reference's operation order; products and sums use the _rn
// intrinsics so the compiler does not contract them into FMAs, and the results round like
// the reference's numpy expressions.
#pragma once

namespace vpm {
namespace {

constexpr int kEwThreads = 256;
constexpr double kModuleEps = 1e-9;  // vpmModule.py:22

unsigned ew_blocks(int64_t count) {
  const int64_t b = (count + kEwThreads - 1) / kEwThreads;
  return unsigned(b > 0 ? b : 1);
}

// The RK kernels are HBM-bound: each thread handles kEwVec consecutive doubles
// through 16-byte loads and stores when every array is 16-byte aligned (the host checks), one
// double per thread otherwise.  The per-element arithmetic is the same function either way.
constexpr int kEwVec = 4;

bool aligned16(const void* p) { return reinterpret_cast<uintptr_t>(p) % 16 == 0; }

unsigned ew_vec_blocks(int64_t count) {
  const int64_t per = int64_t(kEwThreads) * kEwVec;
  const int64_t b = (count + per - 1) / per;
  return unsigned(b > 0 ? b : 1);
}

__device__ __forceinline__ int64_t ew_base(bool vec) {
  const int64_t t = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  return vec ? t * kEwVec : t;
}

// out = x + c * k   (RK stages: vpmModule.py:580, 604, 637, 641, 676, 680, 684)
__device__ __forceinline__ double axpy_elem(double x, double k, double c) {
  return __dadd_rn(x, __dmul_rn(c, k));
}
template <bool VEC>
__global__ void axpy_kernel(const double* __restrict__ x, const double* __restrict__ k, double c,
                            int64_t count, double* __restrict__ out) {
  const int64_t i = ew_base(VEC);
  if (VEC && i + kEwVec <= count) {
    const double2* x2 = reinterpret_cast<const double2*>(x + i);
    const double2* k2 = reinterpret_cast<const double2*>(k + i);
    double2* o2 = reinterpret_cast<double2*>(out + i);
    const double2 a0 = x2[0], a1 = x2[1], b0 = k2[0], b1 = k2[1];
    o2[0] = make_double2(axpy_elem(a0.x, b0.x, c), axpy_elem(a0.y, b0.y, c));
    o2[1] = make_double2(axpy_elem(a1.x, b1.x, c), axpy_elem(a1.y, b1.y, c));
    return;
  }
  const int64_t e = VEC ? (i + kEwVec < count ? i + kEwVec : count) : (i < count ? i + 1 : i);
  for (int64_t j = i; j < e; ++j) out[j] = axpy_elem(x[j], k[j], c);
}

// out = x + (dt/6) * (k1 + 2 k2 + 2 k3 + k4)   (vpmModule.py:688)
__device__ __forceinline__ double rk4_elem(double x, double k1, double k2, double k3, double k4,
                                           double dt6) {
  double s = __dadd_rn(k1, __dmul_rn(2.0, k2));
  s = __dadd_rn(s, __dmul_rn(2.0, k3));
  s = __dadd_rn(s, k4);
  return __dadd_rn(x, __dmul_rn(dt6, s));
}
template <bool VEC>
__global__ void rk4_combine_kernel(const double* __restrict__ x, const double* __restrict__ k1,
                                   const double* __restrict__ k2, const double* __restrict__ k3,
                                   const double* __restrict__ k4, double dt6, int64_t count,
                                   double* __restrict__ out) {
  const int64_t i = ew_base(VEC);
  if (VEC && i + kEwVec <= count) {
#pragma unroll
    for (int h = 0; h < kEwVec; h += 2) {
      const double2 a = *reinterpret_cast<const double2*>(x + i + h);
      const double2 b1 = *reinterpret_cast<const double2*>(k1 + i + h);
      const double2 b2 = *reinterpret_cast<const double2*>(k2 + i + h);
      const double2 b3 = *reinterpret_cast<const double2*>(k3 + i + h);
      const double2 b4 = *reinterpret_cast<const double2*>(k4 + i + h);
      *reinterpret_cast<double2*>(out + i + h) =
          make_double2(rk4_elem(a.x, b1.x, b2.x, b3.x, b4.x, dt6),
                       rk4_elem(a.y, b1.y, b2.y, b3.y, b4.y, dt6));
    }
    return;
  }
  const int64_t e = VEC ? (i + kEwVec < count ? i + kEwVec : count) : (i < count ? i + 1 : i);
  for (int64_t j = i; j < e; ++j) out[j] = rk4_elem(x[j], k1[j], k2[j], k3[j], k4[j], dt6);
}

// Strength update with the reference's BDF ladder and history rotation
// (vpmModule.py:751-787 for stretching, :801-841 for PSE; identical code):
//   step 0: s + dt r;  1: (4s - p1)/3 + (2/3 dt) r;  2: (18s - 9p1 + 2p2)/11 + (6/11 dt) r;
//   >= 3:   (48s - 36p1 + 16p2 - 3p3)/25 + (12/25 dt) r;
//   then p3 <- p2 (step >= 3), p2 <- p1 (step >= 2), p1 <- new.
// `coef` is the step's rate coefficient (dt, (2/3) dt, (6/11) dt or (12/25) dt).
__device__ __forceinline__ double bdf_elem(double si, double a, double b, double c, double r,
                                           int step, double coef) {
  const double cr = __dmul_rn(coef, r);
  if (step == 0) return __dadd_rn(si, cr);
  if (step == 1) return __dadd_rn(__ddiv_rn(__dsub_rn(__dmul_rn(4.0, si), a), 3.0), cr);
  if (step == 2) {
    const double t = __dadd_rn(__dsub_rn(__dmul_rn(18.0, si), __dmul_rn(9.0, a)),
                               __dmul_rn(2.0, b));
    return __dadd_rn(__ddiv_rn(t, 11.0), cr);
  }
  double t = __dsub_rn(__dmul_rn(48.0, si), __dmul_rn(36.0, a));
  t = __dadd_rn(t, __dmul_rn(16.0, b));
  t = __dsub_rn(t, __dmul_rn(3.0, c));
  return __dadd_rn(__ddiv_rn(t, 25.0), cr);
}
// One element per thread: the 16-byte-load form of this kernel (5 streams in, 4 out) measured
// slower (147.5 against 140.4 us at 2^22 particles).
__global__ void bdf_kernel(double* __restrict__ s, double* __restrict__ p1,
                           double* __restrict__ p2, double* __restrict__ p3,
                           const double* __restrict__ rate, int64_t count, int step,
                           double coef) {
  const int64_t j = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (j >= count) return;
  const double a = p1[j], b = p2[j], c = p3[j];
  const double nw = bdf_elem(s[j], a, b, c, rate[j], step, coef);
  if (step >= 3) p3[j] = b;
  if (step >= 2) p2[j] = a;
  p1[j] = nw;
  s[j] = nw;
}

// Core spreading: sigma <- sqrt(sigma^2 + C nu_eff dt), nu_eff = nu + nu_t (vpmModule.py:853-860)
__global__ void core_spreading_kernel(double* __restrict__ sigma, const double* __restrict__ nu,
                                      const double* __restrict__ nut, double C, double dt,
                                      int64_t n) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double ne = __dadd_rn(nu[i], nut[i]);
  const double r = sigma[i];
  sigma[i] = __dsqrt_rn(__dadd_rn(__dmul_rn(r, r), __dmul_rn(__dmul_rn(C, ne), dt)));
}

// Dynamic LES constant (vpmModule.py:887-909); state = {Cnu, enstrophy_ref, initialised}.
__global__ void les_constant_kernel(const double* __restrict__ enstrophy, double* __restrict__ st) {
  const double rms = __dsqrt_rn(enstrophy[0]);
  if (st[2] == 0.0) {
    st[1] = rms;
    st[2] = 1.0;
  }
  st[1] = __dadd_rn(__dmul_rn(0.1, rms), __dmul_rn(0.9, st[1]));
  double c = __dmul_rn(st[0], __ddiv_rn(rms, __dadd_rn(st[1], kModuleEps)));
  c = fmin(c, 0.0761);
  st[0] = fmax(kModuleEps, c);
}

// Single-block fixed-order sums of `cols` interleaved columns (mean vorticity etc.).
template <int COLS>
__global__ void __launch_bounds__(1024)
column_sums_kernel(const double* __restrict__ v, int64_t n, double* __restrict__ out) {
  __shared__ double red[COLS][1024];
  double acc[COLS];
#pragma unroll
  for (int c = 0; c < COLS; ++c) acc[c] = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += 1024)
#pragma unroll
    for (int c = 0; c < COLS; ++c) acc[c] += v[i * COLS + c];
#pragma unroll
  for (int c = 0; c < COLS; ++c) red[c][threadIdx.x] = acc[c];
  __syncthreads();
  for (int w = 512; w > 0; w >>= 1) {
    if (threadIdx.x < w)
#pragma unroll
      for (int c = 0; c < COLS; ++c) red[c][threadIdx.x] += red[c][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0)
#pragma unroll
    for (int c = 0; c < COLS; ++c) out[c] = red[c][0];
}

// nu_t candidate per particle (vpmModule.py:932-951):
//   psi = 1 where the angle between w_i and the mean vorticity is in [pi/4, 3pi/4],
//   nu_t = psi (Cnu sigma)^2 |w|; also the block maxima of nu_t.
__global__ void les_viscosity_kernel(const double* __restrict__ w, const double* __restrict__ sigma,
                                     const double* __restrict__ wsum, const double* __restrict__ st,
                                     int64_t n, double* __restrict__ nut_new,
                                     double* __restrict__ block_max) {
  __shared__ double red[kEwThreads];
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  double v = 0.0;
  if (i < n) {
    const double inv_n = 1.0 / double(n);
    const double mx = wsum[0] * inv_n, my = wsum[1] * inv_n, mz = wsum[2] * inv_n;
    const double mm = sqrt(mx * mx + my * my + mz * mz);
    const double ux = mx / mm, uy = my / mm, uz = mz / mm;
    const double wx = w[3 * i], wy = w[3 * i + 1], wz = w[3 * i + 2];
    const double wm = sqrt(wx * wx + wy * wy + wz * wz);
    double cb = (wx / wm) * ux + (wy / wm) * uy + (wz / wm) * uz;
    cb = fmin(1.0, fmax(-1.0, cb));
    const double beta = acos(cb);
    const double b0 = kPi / 4.0;
    const double psi = (b0 <= beta && beta <= kPi - b0) ? 1.0 : 0.0;
    const double cs = st[0] * sigma[i];
    v = psi * (cs * cs) * wm;
    nut_new[i] = v;
  }
  red[threadIdx.x] = v;
  __syncthreads();
  for (int s = kEwThreads / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  if (threadIdx.x == 0) block_max[blockIdx.x] = red[0];
}

// Commit nu_t only if max(nu_t) > eps (vpmModule.py:954-960).
__global__ void les_commit_kernel(const double* __restrict__ nut_new,
                                  const double* __restrict__ block_max, int nblocks, int64_t n,
                                  double* __restrict__ nut, double* __restrict__ nut_max) {
  __shared__ double s_max;
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int b = 0; b < nblocks; ++b) m = fmax(m, block_max[b]);
    s_max = m;
    if (blockIdx.x == 0 && nut_max) nut_max[0] = m;
  }
  __syncthreads();
  if (!(s_max > kModuleEps)) return;
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    nut[i] = nut_new[i];
}

// Strength relaxation towards the local vorticity direction (vpmModule.py:867-883, with the
// row-wise normalisation the reference intends; the reference itself raises there).
__global__ void relax_kernel(double* __restrict__ s, const double* __restrict__ w, double alpha,
                             int64_t n) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double wx = w[3 * i], wy = w[3 * i + 1], wz = w[3 * i + 2];
  const double sx = s[3 * i], sy = s[3 * i + 1], sz = s[3 * i + 2];
  const double wn = sqrt(wx * wx + wy * wy + wz * wz);
  const double sn = sqrt(sx * sx + sy * sy + sz * sz);
  const double b = 1.0 - alpha;
  s[3 * i] = sx * alpha + b * (wx / wn) * sn;
  s[3 * i + 1] = sy * alpha + b * (wy / wn) * sn;
  s[3 * i + 2] = sz * alpha + b * (wz / wn) * sn;
}

// FP64 O(N) diagnostics in one pass, one block of 256 threads, fixed order
// (vpmModule.py:264-284):
// out = [sum|a|, sum a (3), 1/2 sum x x a (3), 1/3 sum x x (x x a) (3)].
constexpr int kDiagThreads = 256;
__global__ void __launch_bounds__(kDiagThreads)
diagnostics_kernel(const double* __restrict__ x, const double* __restrict__ a, int64_t n,
                   double* __restrict__ out) {
  constexpr int K = 10;
  __shared__ double red[K][kDiagThreads];
  double acc[K];
#pragma unroll
  for (int k = 0; k < K; ++k) acc[k] = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += kDiagThreads) {
    const double px = x[3 * i], py = x[3 * i + 1], pz = x[3 * i + 2];
    const double ax = a[3 * i], ay = a[3 * i + 1], az = a[3 * i + 2];
    acc[0] += sqrt(ax * ax + ay * ay + az * az);
    acc[1] += ax;
    acc[2] += ay;
    acc[3] += az;
    const double cx = py * az - pz * ay, cy = pz * ax - px * az, cz = px * ay - py * ax;
    acc[4] += cx;
    acc[5] += cy;
    acc[6] += cz;
    acc[7] += py * cz - pz * cy;
    acc[8] += pz * cx - px * cz;
    acc[9] += px * cy - py * cx;
  }
#pragma unroll
  for (int k = 0; k < K; ++k) red[k][threadIdx.x] = acc[k];
  __syncthreads();
  for (int w = kDiagThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w)
#pragma unroll
      for (int k = 0; k < K; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    out[0] = red[0][0];
    out[1] = red[1][0];
    out[2] = red[2][0];
    out[3] = red[3][0];
    out[4] = 0.5 * red[4][0];
    out[5] = 0.5 * red[5][0];
    out[6] = 0.5 * red[6][0];
    out[7] = (1.0 / 3.0) * red[7][0];
    out[8] = (1.0 / 3.0) * red[8][0];
    out[9] = (1.0 / 3.0) * red[9][0];
  }
}

// ---- least-squares dynamic coefficient (no counterpart in the reference) ------------------
// Germano identity for the sub-filter kinetic energy between the particle filter (core sigma)
// and a test filter of twice the core, with the model k(D) = C^2 D^2 |w_D|^2 (w_D: vorticity
// filtered at width D):
//   L_i = 1/2 (hat(|u|^2)_i - |hat u_i|^2)        resolved energy between the two filters
//   M_i = (2 sigma_i)^2 |hat w_i|^2 - hat(sigma^2 |w|^2)_i
//   C^2 = sum_i L_i M_i / sum_i M_i^2             (least squares over all particles, FP64)
// hat f_i = sum_j zeta_{2 sigma_j}(x_i - x_j) f_j v_j is the test filter of a particle field,
// with the particle volume v_j = |alpha_j| / |w_j| (0 where w_j = 0).  Cnu = sqrt(C^2) clipped to
// the reference's range [1e-9, 0.0761]; where C^2 <= 0 or sum M^2 = 0 Cnu stays unchanged.

// w_j = (|u_j|^2 v_j, sigma_j^2 |w_j|^2 v_j, 0): the fields the test filter acts on.
__global__ void les_lsq_weights_kernel(const double* __restrict__ u, const double* __restrict__ w,
                                       const double* __restrict__ a,
                                       const double* __restrict__ sigma, int64_t n,
                                       double* __restrict__ out) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double ux = u[3 * i], uy = u[3 * i + 1], uz = u[3 * i + 2];
  const double wx = w[3 * i], wy = w[3 * i + 1], wz = w[3 * i + 2];
  const double ax = a[3 * i], ay = a[3 * i + 1], az = a[3 * i + 2];
  const double w2 = wx * wx + wy * wy + wz * wz;
  const double vol = w2 > 0.0 ? sqrt(ax * ax + ay * ay + az * az) / sqrt(w2) : 0.0;
  const double s = sigma[i];
  out[3 * i] = (ux * ux + uy * uy + uz * uz) * vol;
  out[3 * i + 1] = s * s * w2 * vol;
  out[3 * i + 2] = 0.0;
}

// Single block, fixed order: sum L M and sum M M, then the coefficient update.
__global__ void __launch_bounds__(1024)
les_lsq_kernel(const double* __restrict__ uh, const double* __restrict__ wh,
               const double* __restrict__ fh, const double* __restrict__ sigma, int64_t n,
               double* __restrict__ st, double* __restrict__ sums) {
  __shared__ double red[2][1024];
  double lm = 0.0, mm = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += 1024) {
    const double hx = uh[3 * i], hy = uh[3 * i + 1], hz = uh[3 * i + 2];
    const double gx = wh[3 * i], gy = wh[3 * i + 1], gz = wh[3 * i + 2];
    const double L = 0.5 * (fh[3 * i] - (hx * hx + hy * hy + hz * hz));
    const double d = 2.0 * sigma[i];
    const double M = d * d * (gx * gx + gy * gy + gz * gz) - fh[3 * i + 1];
    lm += L * M;
    mm += M * M;
  }
  red[0][threadIdx.x] = lm;
  red[1][threadIdx.x] = mm;
  __syncthreads();
  for (int k = 512; k > 0; k >>= 1) {
    if (threadIdx.x < k) {
      red[0][threadIdx.x] += red[0][threadIdx.x + k];
      red[1][threadIdx.x] += red[1][threadIdx.x + k];
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double slm = red[0][0], smm = red[1][0];
    if (sums) {
      sums[0] = slm;
      sums[1] = smm;
    }
    if (smm > 0.0 && slm > 0.0) {
      const double c = sqrt(slm / smm);
      st[0] = fmax(kModuleEps, fmin(c, 0.0761));
    }
  }
}

int launch_status(const char* what) {
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? VPM_OK : cuda_fail(e, what);
}

}  // namespace
}  // namespace vpm

extern "C" {

int vpm_axpy(const double* x, const double* k, double c, int64_t count, double* out,
             void* stream) {
  using namespace vpm;
  if (count < 0 || (count > 0 && (!x || !k || !out))) return fail(VPM_ERR_ARG, "bad axpy args");
  if (count == 0) return VPM_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (aligned16(x) && aligned16(k) && aligned16(out))
    axpy_kernel<true><<<ew_vec_blocks(count), kEwThreads, 0, st>>>(x, k, c, count, out);
  else
    axpy_kernel<false><<<ew_blocks(count), kEwThreads, 0, st>>>(x, k, c, count, out);
  return launch_status("axpy launch");
}

int vpm_rk4_combine(const double* x, const double* k1, const double* k2, const double* k3,
                    const double* k4, double dt, int64_t count, double* out, void* stream) {
  using namespace vpm;
  if (count < 0 || (count > 0 && (!x || !k1 || !k2 || !k3 || !k4 || !out)))
    return fail(VPM_ERR_ARG, "bad rk4 combine args");
  if (count == 0) return VPM_OK;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (aligned16(x) && aligned16(k1) && aligned16(k2) && aligned16(k3) && aligned16(k4) &&
      aligned16(out))
    rk4_combine_kernel<true><<<ew_vec_blocks(count), kEwThreads, 0, st>>>(x, k1, k2, k3, k4,
                                                                          dt / 6.0, count, out);
  else
    rk4_combine_kernel<false><<<ew_blocks(count), kEwThreads, 0, st>>>(x, k1, k2, k3, k4,
                                                                       dt / 6.0, count, out);
  return launch_status("rk4 combine launch");
}

int vpm_bdf_update(double* strengths, double* hist1, double* hist2, double* hist3,
                   const double* rate, int64_t count, int time_step, double coef, void* stream) {
  using namespace vpm;
  if (count < 0 || time_step < 0 ||
      (count > 0 && (!strengths || !hist1 || !hist2 || !hist3 || !rate)))
    return fail(VPM_ERR_ARG, "bad bdf args");
  if (count == 0) return VPM_OK;
  bdf_kernel<<<ew_blocks(count), kEwThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      strengths, hist1, hist2, hist3, rate, count, time_step, coef);
  return launch_status("bdf launch");
}

int vpm_core_spreading(double* radii, const double* viscosities, const double* viscosities_t,
                       int64_t n, double C, double dt, void* stream) {
  using namespace vpm;
  if (n < 0 || (n > 0 && (!radii || !viscosities || !viscosities_t)))
    return fail(VPM_ERR_ARG, "bad core spreading args");
  if (n == 0) return VPM_OK;
  core_spreading_kernel<<<ew_blocks(n), kEwThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      radii, viscosities, viscosities_t, C, dt, n);
  return launch_status("core spreading launch");
}

size_t vpm_les_workspace_bytes(int64_t n) {
  using namespace vpm;
  return align_up(size_t(n > 0 ? n : 0) * 8) + align_up(size_t(ew_blocks(n)) * 8) + 256;
}

int vpm_les_update(const double* vorticity, const double* radii, const double* enstrophy,
                   int64_t n, int advance_constant, double* les_state, double* viscosities_t,
                   double* nut_max, void* workspace, size_t workspace_bytes, void* stream) {
  using namespace vpm;
  if (n < 0 || !les_state || (advance_constant && !enstrophy))
    return fail(VPM_ERR_ARG, "bad les args");
  if (n > 0 && (!vorticity || !radii || !viscosities_t))
    return fail(VPM_ERR_ARG, "bad les args");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int rc = VPM_OK;
  if (advance_constant) {
    les_constant_kernel<<<1, 1, 0, st>>>(enstrophy, les_state);
    rc = launch_status("les constant launch");
  }
  if (rc || n == 0) return rc;
  if (!workspace || reinterpret_cast<uintptr_t>(workspace) % kAlign != 0)
    return fail(VPM_ERR_ALIGN, "les workspace must be 256-byte aligned");
  if (workspace_bytes < vpm_les_workspace_bytes(n))
    return fail(VPM_ERR_WORKSPACE, "les workspace too small");
  char* ws = static_cast<char*>(workspace);
  double* nut_new = reinterpret_cast<double*>(ws);
  double* bmax = reinterpret_cast<double*>(ws + align_up(size_t(n) * 8));
  double* wsum = reinterpret_cast<double*>(ws + align_up(size_t(n) * 8) +
                                           align_up(size_t(ew_blocks(n)) * 8));
  column_sums_kernel<3><<<1, 1024, 0, st>>>(vorticity, n, wsum);
  rc = launch_status("column sums launch");
  if (rc) return rc;
  const unsigned nb = ew_blocks(n);
  les_viscosity_kernel<<<nb, kEwThreads, 0, st>>>(vorticity, radii, wsum, les_state, n, nut_new,
                                                  bmax);
  rc = launch_status("les viscosity launch");
  if (rc) return rc;
  les_commit_kernel<<<nb < 1184 ? nb : 1184, kEwThreads, 0, st>>>(nut_new, bmax, int(nb), n,
                                                                   viscosities_t, nut_max);
  return launch_status("les commit launch");
}

int vpm_les_lsq_weights(const double* velocities, const double* vorticity,
                        const double* strengths, const double* radii, int64_t n,
                        double* weights, void* stream) {
  using namespace vpm;
  if (n < 0 || (n > 0 && (!velocities || !vorticity || !strengths || !radii || !weights)))
    return fail(VPM_ERR_ARG, "bad les lsq weights args");
  if (n == 0) return VPM_OK;
  les_lsq_weights_kernel<<<ew_blocks(n), kEwThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      velocities, vorticity, strengths, radii, n, weights);
  return launch_status("les lsq weights launch");
}

int vpm_les_lsq_update(const double* test_velocities, const double* test_vorticity,
                       const double* test_filtered, const double* radii, int64_t n,
                       double* les_state, double* sums, void* stream) {
  using namespace vpm;
  if (n < 0 || !les_state ||
      (n > 0 && (!test_velocities || !test_vorticity || !test_filtered || !radii)))
    return fail(VPM_ERR_ARG, "bad les lsq args");
  les_lsq_kernel<<<1, 1024, 0, static_cast<cudaStream_t>(stream)>>>(
      test_velocities, test_vorticity, test_filtered, radii, n, les_state, sums);
  return launch_status("les lsq launch");
}

int vpm_relax_strengths(double* strengths, const double* vorticity, int64_t n, double alpha,
                        void* stream) {
  using namespace vpm;
  if (n < 0 || (n > 0 && (!strengths || !vorticity))) return fail(VPM_ERR_ARG, "bad relax args");
  if (n == 0) return VPM_OK;
  relax_kernel<<<ew_blocks(n), kEwThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      strengths, vorticity, alpha, n);
  return launch_status("relax launch");
}

int vpm_particle_diagnostics(const double* positions, const double* strengths, int64_t n,
                             double* out10, void* stream) {
  using namespace vpm;
  if (n < 0 || !out10 || (n > 0 && (!positions || !strengths)))
    return fail(VPM_ERR_ARG, "bad diagnostics args");
  diagnostics_kernel<<<1, kDiagThreads, 0, static_cast<cudaStream_t>(stream)>>>(positions, strengths, n,
                                                                         out10);
  return launch_status("diagnostics launch");
}

}  // extern "C"
