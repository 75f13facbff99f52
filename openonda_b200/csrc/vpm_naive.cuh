// vpm_naive.cuh -- the reference's GPU algorithm restated in CUDA C++, for measurement only.
//
// OpenONDA's Numba-CUDA kernels (ParticlesPhysicsCuda.py:133-191 self-induced velocity,
// :375-445 stretching) run one thread per target particle, 512 threads per block
// (:5), read every source straight from global memory, and evaluate the regularised kernel
// with FP64 powers.  These two kernels keep exactly that structure so bench.py can report
// what the reference's algorithm achieves on the same B200.  They are not used by any
// library entry point that computes results for callers.
#pragma once

namespace vpm {
namespace {

constexpr int kNaiveThreads = 512;  // ParticlesPhysicsCuda.py:5

__global__ void naive_selfinduced_velocity_kernel(const double* __restrict__ pos,
                                                  const double* __restrict__ str,
                                                  const double* __restrict__ rad, int64_t n,
                                                  double* __restrict__ out) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double tx = pos[3 * i], ty = pos[3 * i + 1], tz = pos[3 * i + 2], ri = rad[i];
  double ux = 0.0, uy = 0.0, uz = 0.0;
  for (int64_t j = 0; j < n; ++j) {
    if (j == i) continue;
    const double s = (ri + rad[j]) / 2.0;
    const double rx = tx - pos[3 * j], ry = ty - pos[3 * j + 1], rz = tz - pos[3 * j + 2];
    const double r2 = rx * rx + ry * ry + rz * rz;
    const double s2 = s * s;
    const double rho2 = r2 / s2;
    const double q = (rho2 + 2.5) / (pow(rho2 + 1.0, 2.5) * s * s2);
    const double ax = str[3 * j], ay = str[3 * j + 1], az = str[3 * j + 2];
    ux -= q * (ry * az - rz * ay);
    uy -= q * (rz * ax - rx * az);
    uz -= q * (rx * ay - ry * ax);
  }
  out[3 * i] = kOneOver4Pi * ux;
  out[3 * i + 1] = kOneOver4Pi * uy;
  out[3 * i + 2] = kOneOver4Pi * uz;
}

__global__ void naive_strength_gradients_kernel(const double* __restrict__ pos,
                                                const double* __restrict__ str,
                                                const double* __restrict__ rad, int64_t n,
                                                double* __restrict__ out) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double ri = rad[i];
  const double px = pos[3 * i], py = pos[3 * i + 1], pz = pos[3 * i + 2];
  const double bx = str[3 * i], by = str[3 * i + 1], bz = str[3 * i + 2];
  double gx = 0.0, gy = 0.0, gz = 0.0;
  for (int64_t j = 0; j < n; ++j) {
    if (i == j) continue;
    const double rx = px - pos[3 * j], ry = py - pos[3 * j + 1], rz = pz - pos[3 * j + 2];
    const double d2 = rx * rx + ry * ry + rz * rz;
    const double s = (ri + rad[j]) * 0.5;
    const double s2 = s * s;
    const double s3 = s2 * s;
    const double p1 = d2 / s2 + 1.0;
    const double f1 = (p1 + 1.5) / (s3 * pow(p1, 2.5));
    const double f2 = 3.0 * (p1 + 2.5) / (s3 * s2 * pow(p1, 3.5));
    const double ax = str[3 * j], ay = str[3 * j + 1], az = str[3 * j + 2];
    const double c2x = ry * az - rz * ay, c2y = rz * ax - rx * az, c2z = rx * ay - ry * ax;
    const double d3 = bx * c2x + by * c2y + bz * c2z;
    gx += (f1 * (by * az - bz * ay) + f2 * d3 * rx) * kOneOver4Pi;
    gy += (f1 * (bz * ax - bx * az) + f2 * d3 * ry) * kOneOver4Pi;
    gz += (f1 * (bx * ay - by * ax) + f2 * d3 * rz) * kOneOver4Pi;
  }
  out[3 * i] = gx;
  out[3 * i + 1] = gy;
  out[3 * i + 2] = gz;
}

}  // namespace
}  // namespace vpm

extern "C" {

// which = 0: self-induced velocity, 1: stretching.  Reference-layout device arrays.
int vpm_naive_reference_kernel(int which, const double* positions, const double* strengths,
                               const double* radii, int64_t n, double* out, void* stream) {
  using namespace vpm;
  if (n < 0 || (n > 0 && (!positions || !strengths || !radii || !out)) || which < 0 ||
      which > 1)
    return fail(VPM_ERR_ARG, "bad naive kernel args");
  if (n == 0) return VPM_OK;
  int rc = check_arch();
  if (rc) return rc;
  const unsigned blocks = unsigned((n + kNaiveThreads - 1) / kNaiveThreads);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (which == 0)
    naive_selfinduced_velocity_kernel<<<blocks, kNaiveThreads, 0, st>>>(positions, strengths,
                                                                      radii, n, out);
  else
    naive_strength_gradients_kernel<<<blocks, kNaiveThreads, 0, st>>>(positions, strengths,
                                                                    radii, n, out);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? VPM_OK : cuda_fail(e, "naive kernel launch");
}

}  // extern "C"
