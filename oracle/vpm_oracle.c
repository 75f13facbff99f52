/*
 * vpm_oracle.c -- CPU restatement of OpenONDA's VPM pair sums (TEST INFRASTRUCTURE).
 *
 * This file is the parity oracle and the timed CPU baseline.  It is never part of the
 * product path: only tests/, __graft_entry__.smoke() and bench.py (CPU-baseline leg and
 * the reference arm) load it, and only to check or to time against the CUDA library.
 *
 * Two families of functions restate the two reference modules in plain FP64 C:
 *
 *   oracle_gpu_*  follow OpenONDA/solvers/VPM/ParticlesPhysicsCuda.py (the Numba-CUDA
 *                 module, i.e. the semantics the B200 drop-in reproduces), with two
 *                 documented fixes: scalar accumulators start at zero (the reference
 *                 allocates them with cuda.device_array and never clears them,
 *                 ParticlesPhysicsCuda.py:545,655,764) and the vorticity probe produces
 *                 one row per target (the reference sizes its grid and output by the
 *                 number of sources, ParticlesPhysicsCuda.py:200,207).
 *   oracle_cpu_*  follow OpenONDA/solvers/VPM/ParticlesPhysics.py (the Numba-CPU module,
 *                 i.e. the reference's CPU path that the baseline times).
 *
 * Arrays use the reference layout: positions/strengths (n,3) row-major float64,
 * radii/viscosities (n,) float64.  Loops over targets run under OpenMP; scalar results
 * are summed per target and then over targets in index order, so they are deterministic.
 * The arithmetic keeps the reference's formulas (pow with the same exponents) so that
 * agreement with the reference is at the level of libm rounding.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define ORACLE_EPS 1e-8 /* ParticlesPhysicsCuda.py:6, ParticlesPhysics.py:4 */
static const double ONE_OVER_FOUR_PI = 1.0 / (4.0 * M_PI);

int oracle_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void oracle_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

/* ------------------------------------------------------------------------------------ */
/* GPU semantics (ParticlesPhysicsCuda.py)                                               */
/* ------------------------------------------------------------------------------------ */

/* get_induced_velocity_at_kernel, ParticlesPhysicsCuda.py:39-97: source core sigma_j,
 * pairs with r^2 <= 1e-8 skipped. */
void oracle_gpu_induced_velocity_at(const double* tgt, int64_t m, const double* pos,
                                    const double* str, const double* rad, int64_t n,
                                    double* out) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m; ++i) {
    double ux = 0.0, uy = 0.0, uz = 0.0;
    const double tx = tgt[3 * i], ty = tgt[3 * i + 1], tz = tgt[3 * i + 2];
    for (int64_t j = 0; j < n; ++j) {
      const double rx = tx - pos[3 * j], ry = ty - pos[3 * j + 1], rz = tz - pos[3 * j + 2];
      const double r2 = rx * rx + ry * ry + rz * rz;
      if (r2 > ORACLE_EPS) {
        const double s = rad[j];
        const double s2 = s * s;
        const double rho2 = r2 / s2;
        const double q = (rho2 + 2.5) / (pow(rho2 + 1.0, 2.5) * s2 * s);
        const double ax = str[3 * j], ay = str[3 * j + 1], az = str[3 * j + 2];
        ux -= q * (ry * az - rz * ay);
        uy -= q * (rz * ax - rx * az);
        uz -= q * (rx * ay - ry * ax);
      }
    }
    out[3 * i] = ux * ONE_OVER_FOUR_PI;
    out[3 * i + 1] = uy * ONE_OVER_FOUR_PI;
    out[3 * i + 2] = uz * ONE_OVER_FOUR_PI;
  }
}

/* get_selfinduced_velocity_kernel, ParticlesPhysicsCuda.py:133-191: j != i, pair core
 * (sigma_i + sigma_j)/2, no r^2 threshold. */
void oracle_gpu_selfinduced_velocity_range(const double* pos, const double* str,
                                           const double* rad, int64_t n, int64_t t0, int64_t t1,
                                           double* out) {
#pragma omp parallel for schedule(static)
  for (int64_t i = t0; i < t1; ++i) {
    double ux = 0.0, uy = 0.0, uz = 0.0;
    const double tx = pos[3 * i], ty = pos[3 * i + 1], tz = pos[3 * i + 2];
    const double ti = rad[i];
    for (int64_t j = 0; j < n; ++j) {
      if (j == i) continue;
      const double s = (ti + rad[j]) / 2.0;
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
    out[3 * (i - t0)] = ONE_OVER_FOUR_PI * ux;
    out[3 * (i - t0) + 1] = ONE_OVER_FOUR_PI * uy;
    out[3 * (i - t0) + 2] = ONE_OVER_FOUR_PI * uz;
  }
}

void oracle_gpu_selfinduced_velocity(const double* pos, const double* str, const double* rad,
                                     int64_t n, double* out) {
  oracle_gpu_selfinduced_velocity_range(pos, str, rad, n, 0, n, out);
}

/* get_vorticity_field_at_kernel_simplified, ParticlesPhysicsCuda.py:291-346 (the kernel
 * the wrapper at :198-219 launches): zeta-only regularised vorticity, source core sigma_j,
 * pairs with r^2 <= 1e-8 skipped.  One output row per target. */
void oracle_gpu_vorticity_field_at(const double* tgt, int64_t m, const double* pos,
                                   const double* str, const double* rad, int64_t n,
                                   double* out) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m; ++i) {
    double wx = 0.0, wy = 0.0, wz = 0.0;
    const double tx = tgt[3 * i], ty = tgt[3 * i + 1], tz = tgt[3 * i + 2];
    for (int64_t j = 0; j < n; ++j) {
      const double rx = tx - pos[3 * j], ry = ty - pos[3 * j + 1], rz = tz - pos[3 * j + 2];
      const double r2 = rx * rx + ry * ry + rz * rz;
      if (r2 > ORACLE_EPS) {
        const double s = rad[j];
        const double rho2 = r2 / (s * s);
        const double s3 = s * s * s;
        const double xi = 7.5 / (pow(rho2 + 1.0, 3.5) * s3);
        wx += xi * str[3 * j];
        wy += xi * str[3 * j + 1];
        wz += xi * str[3 * j + 2];
      }
    }
    out[3 * i] = wx * ONE_OVER_FOUR_PI;
    out[3 * i + 1] = wy * ONE_OVER_FOUR_PI;
    out[3 * i + 2] = wz * ONE_OVER_FOUR_PI;
  }
}

/* get_strength_gradients_kernel, ParticlesPhysicsCuda.py:375-445: vortex stretching in the
 * transpose scheme, j != i, pair core (sigma_i + sigma_j)/2. */
void oracle_gpu_strength_gradients_range(const double* pos, const double* str,
                                         const double* rad, int64_t n, int64_t t0, int64_t t1,
                                         double* out) {
#pragma omp parallel for schedule(static)
  for (int64_t i = t0; i < t1; ++i) {
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
      const double c1x = by * az - bz * ay, c1y = bz * ax - bx * az, c1z = bx * ay - by * ax;
      const double c2x = ry * az - rz * ay, c2y = rz * ax - rx * az, c2z = rx * ay - ry * ax;
      const double d3 = bx * c2x + by * c2y + bz * c2z;
      gx += (f1 * c1x + f2 * d3 * rx) * ONE_OVER_FOUR_PI;
      gy += (f1 * c1y + f2 * d3 * ry) * ONE_OVER_FOUR_PI;
      gz += (f1 * c1z + f2 * d3 * rz) * ONE_OVER_FOUR_PI;
    }
    out[3 * (i - t0)] = gx;
    out[3 * (i - t0) + 1] = gy;
    out[3 * (i - t0) + 2] = gz;
  }
}

void oracle_gpu_strength_gradients(const double* pos, const double* str, const double* rad,
                                   int64_t n, double* out) {
  oracle_gpu_strength_gradients_range(pos, str, rad, n, 0, n, out);
}

/* get_strength_gradients_PSE_kernel, ParticlesPhysicsCuda.py:478-530: PSE diffusion with
 * the target's viscosity nu_i only, pair core (sigma_i + sigma_j)/2, j != i, no epsilon. */
void oracle_gpu_strength_gradients_pse(const double* pos, const double* str, const double* rad,
                                       const double* nu, int64_t n, double* out) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    const double ri = rad[i], vi = nu[i];
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
      const double s5 = s2 * s3;
      const double p1 = d2 / s2 + 1.0;
      const double f3 = 105.0 * vi / (s5 * pow(p1, 4.5));
      gx += f3 * s3 * (str[3 * j] - bx) * ONE_OVER_FOUR_PI;
      gy += f3 * s3 * (str[3 * j + 1] - by) * ONE_OVER_FOUR_PI;
      gz += f3 * s3 * (str[3 * j + 2] - bz) * ONE_OVER_FOUR_PI;
    }
    out[3 * i] = gx;
    out[3 * i + 1] = gy;
    out[3 * i + 2] = gz;
  }
}

/* Sum per-target partials in index order (deterministic). */
static double ordered_sum(const double* v, int64_t n) {
  double s = 0.0;
  for (int64_t i = 0; i < n; ++i) s += v[i];
  return s;
}

/* get_total_kinetic_energy_kernel, ParticlesPhysicsCuda.py:563-642, with the wrapper
 * :537-558 (accumulator zeroed here).  j != i, no epsilon inside sqrt(rho^2 + 1). */
double oracle_gpu_total_kinetic_energy(const double* pos, const double* str, const double* rad,
                                       int64_t n) {
  double* part = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    const double px = pos[3 * i], py = pos[3 * i + 1], pz = pos[3 * i + 2];
    const double bx = str[3 * i], by = str[3 * i + 1], bz = str[3 * i + 2];
    const double ri = rad[i];
    double e = 0.0;
    for (int64_t j = 0; j < n; ++j) {
      if (j == i) continue;
      const double rx = px - pos[3 * j], ry = py - pos[3 * j + 1], rz = pz - pos[3 * j + 2];
      const double rn = pow(rx * rx + ry * ry + rz * rz, 0.5);
      const double ux = rx / rn, uy = ry / rn, uz = rz / rn;
      const double s = (ri + rad[j]) * 0.5;
      const double rho = rn / s;
      const double p1 = pow(rho, 2) + 1.0;
      const double t1 = 2.0 * rho / pow(p1, 0.5);
      const double t2 = pow(rho, 3) / pow(p1, 1.5);
      const double ax = str[3 * j], ay = str[3 * j + 1], az = str[3 * j + 2];
      const double q1 = bx * ax + by * ay + bz * az;
      const double q2 = ux * bx + uy * by + uz * bz;
      const double q3 = ux * ax + uy * ay + uz * az;
      e += (t1 * q1 + t2 * (q2 * q3 - q1)) / rn;
    }
    part[i] = e;
  }
  const double total = ordered_sum(part, n) / (16.0 * M_PI);
  free(part);
  return total;
}

/* get_total_helicity_kernel, ParticlesPhysicsCuda.py:673-750, with the wrapper :647-668
 * (accumulator zeroed here; the wrapper's second division by 4*pi at :668 is applied when
 * ref_extra_4pi is nonzero). */
double oracle_gpu_total_helicity(const double* pos, const double* str, const double* rad,
                                 int64_t n, int ref_extra_4pi) {
  double* part = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    const double px = pos[3 * i], py = pos[3 * i + 1], pz = pos[3 * i + 2];
    const double bx = str[3 * i], by = str[3 * i + 1], bz = str[3 * i + 2];
    const double ri = rad[i];
    double h = 0.0;
    for (int64_t j = 0; j < n; ++j) {
      if (i == j) continue;
      const double rx = px - pos[3 * j], ry = py - pos[3 * j + 1], rz = pz - pos[3 * j + 2];
      const double s = 0.5 * (ri + rad[j]);
      const double qx = rx / s, qy = ry / s, qz = rz / s;
      const double rho2 = qx * qx + qy * qy + qz * qz;
      const double term = (rho2 + 2.5) / (s * s * s * pow(rho2 + 1.0, 2.5));
      const double ax = str[3 * j], ay = str[3 * j + 1], az = str[3 * j + 2];
      const double cx = by * az - bz * ay, cy = bz * ax - bx * az, cz = bx * ay - by * ax;
      h += (rx * cx + ry * cy + rz * cz) * term;
    }
    part[i] = h;
  }
  double total = ordered_sum(part, n) / (4.0 * M_PI);
  if (ref_extra_4pi) total /= (4.0 * M_PI);
  free(part);
  return total;
}

/* get_total_enstrophy_kernel_simple, ParticlesPhysicsCuda.py:867-920, with the wrapper
 * :756-777 (accumulator zeroed; the wrapper's extra 1/(4*pi) at :777 when ref_extra_4pi).
 * All pairs including i == j. */
double oracle_gpu_total_enstrophy(const double* pos, const double* str, const double* rad,
                                  int64_t n, int ref_extra_4pi) {
  double* part = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    const double px = pos[3 * i], py = pos[3 * i + 1], pz = pos[3 * i + 2];
    const double bx = str[3 * i], by = str[3 * i + 1], bz = str[3 * i + 2];
    const double ri = rad[i];
    double e = 0.0;
    for (int64_t j = 0; j < n; ++j) {
      const double rx = px - pos[3 * j], ry = py - pos[3 * j + 1], rz = pz - pos[3 * j + 2];
      const double r2 = rx * rx + ry * ry + rz * rz;
      const double s = (ri + rad[j]) * 0.5;
      const double s2 = s * s;
      const double t1 = (r2 + 3.2 * s2) / pow(r2 + s2, 1.5);
      e += t1 * (bx * str[3 * j] + by * str[3 * j + 1] + bz * str[3 * j + 2]);
    }
    part[i] = e;
  }
  double total = ordered_sum(part, n) / (8.0 * M_PI);
  if (ref_extra_4pi) total /= (4.0 * M_PI);
  free(part);
  return total;
}

/* ------------------------------------------------------------------------------------ */
/* CPU semantics (ParticlesPhysics.py)                                                   */
/* ------------------------------------------------------------------------------------ */

/* get_induced_velocity_at, ParticlesPhysics.py:10-74 (same math as the GPU probe). */
void oracle_cpu_induced_velocity_at(const double* tgt, int64_t m, const double* pos,
                                    const double* str, const double* rad, int64_t n,
                                    double* out) {
  oracle_gpu_induced_velocity_at(tgt, m, pos, str, rad, n, out);
}

/* get_selfinduced_velocity, ParticlesPhysics.py:82-143: core sigma_i of the TARGET. */
void oracle_cpu_selfinduced_velocity_range(const double* pos, const double* str,
                                           const double* rad, int64_t n, int64_t t0, int64_t t1,
                                           double* out) {
#pragma omp parallel for schedule(static)
  for (int64_t i = t0; i < t1; ++i) {
    double ux = 0.0, uy = 0.0, uz = 0.0;
    const double tx = pos[3 * i], ty = pos[3 * i + 1], tz = pos[3 * i + 2];
    const double s = rad[i];
    const double s2 = s * s;
    for (int64_t j = 0; j < n; ++j) {
      if (i == j) continue;
      const double rx = tx - pos[3 * j], ry = ty - pos[3 * j + 1], rz = tz - pos[3 * j + 2];
      const double r2 = rx * rx + ry * ry + rz * rz;
      const double rho2 = r2 / s2;
      const double q = (rho2 + 2.5) / (pow(rho2 + 1.0, 2.5) * s * s2);
      const double ax = str[3 * j], ay = str[3 * j + 1], az = str[3 * j + 2];
      ux -= q * (ry * az - rz * ay);
      uy -= q * (rz * ax - rx * az);
      uz -= q * (rx * ay - ry * ax);
    }
    out[3 * (i - t0)] = ux * ONE_OVER_FOUR_PI;
    out[3 * (i - t0) + 1] = uy * ONE_OVER_FOUR_PI;
    out[3 * (i - t0) + 2] = uz * ONE_OVER_FOUR_PI;
  }
}

void oracle_cpu_selfinduced_velocity(const double* pos, const double* str, const double* rad,
                                     int64_t n, double* out) {
  oracle_cpu_selfinduced_velocity_range(pos, str, rad, n, 0, n, out);
}

/* get_vorticity_field_at, ParticlesPhysics.py:212-262: full zeta/q regularised kernel. */
void oracle_cpu_vorticity_field_at(const double* tgt, int64_t m, const double* pos,
                                   const double* str, const double* rad, int64_t n,
                                   double* out) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < m; ++i) {
    double wx = 0.0, wy = 0.0, wz = 0.0;
    const double tx = tgt[3 * i], ty = tgt[3 * i + 1], tz = tgt[3 * i + 2];
    for (int64_t j = 0; j < n; ++j) {
      const double rx = tx - pos[3 * j], ry = ty - pos[3 * j + 1], rz = tz - pos[3 * j + 2];
      const double r2 = rx * rx + ry * ry + rz * rz;
      if (r2 > ORACLE_EPS) {
        const double s = rad[j];
        const double rho2 = r2 / pow(s, 2);
        const double s3 = pow(s, 3);
        const double xi = 7.5 / (pow(rho2 + 1.0, 3.5) * s3);
        const double q = (rho2 + 2.5) / (pow(rho2 + 1.0, 2.5) * s3);
        const double ax = str[3 * j], ay = str[3 * j + 1], az = str[3 * j + 2];
        const double t1 = xi - q;
        const double t2 = (3.0 * q - xi) * (rx * ax + ry * ay + rz * az) / r2;
        wx += t1 * ax + t2 * rx;
        wy += t1 * ay + t2 * ry;
        wz += t1 * az + t2 * rz;
      }
    }
    out[3 * i] = wx * ONE_OVER_FOUR_PI;
    out[3 * i + 1] = wy * ONE_OVER_FOUR_PI;
    out[3 * i + 2] = wz * ONE_OVER_FOUR_PI;
  }
}

/* get_strength_gradients, ParticlesPhysics.py:269-312 (same math as the GPU kernel). */
void oracle_cpu_strength_gradients(const double* pos, const double* str, const double* rad,
                                   int64_t n, double* out) {
  oracle_gpu_strength_gradients(pos, str, rad, n, out);
}

void oracle_cpu_strength_gradients_range(const double* pos, const double* str,
                                         const double* rad, int64_t n, int64_t t0, int64_t t1,
                                         double* out) {
  oracle_gpu_strength_gradients_range(pos, str, rad, n, t0, t1, out);
}

/* get_strength_gradients_PSE, ParticlesPhysics.py:319-382: viscosity (nu_i + nu_j)/2 and
 * epsilon added to rho^2 + 1. */
void oracle_cpu_strength_gradients_pse(const double* pos, const double* str, const double* rad,
                                       const double* nu, int64_t n, double* out) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    const double ri = rad[i], vi = nu[i];
    const double px = pos[3 * i], py = pos[3 * i + 1], pz = pos[3 * i + 2];
    const double bx = str[3 * i], by = str[3 * i + 1], bz = str[3 * i + 2];
    double gx = 0.0, gy = 0.0, gz = 0.0;
    for (int64_t j = 0; j < n; ++j) {
      if (j == i) continue;
      const double v = (vi + nu[j]) * 0.5;
      const double s = (ri + rad[j]) * 0.5;
      const double rx = px - pos[3 * j], ry = py - pos[3 * j + 1], rz = pz - pos[3 * j + 2];
      const double d2 = rx * rx + ry * ry + rz * rz;
      const double s2 = s * s;
      const double s3 = s2 * s;
      const double p1 = (d2 / s2) + 1.0 + ORACLE_EPS;
      const double f3 = 105.0 * v / (s2 * s3 * pow(p1, 4.5));
      gx += f3 * s3 * (str[3 * j] - bx);
      gy += f3 * s3 * (str[3 * j + 1] - by);
      gz += f3 * s3 * (str[3 * j + 2] - bz);
    }
    out[3 * i] = gx * ONE_OVER_FOUR_PI;
    out[3 * i + 1] = gy * ONE_OVER_FOUR_PI;
    out[3 * i + 2] = gz * ONE_OVER_FOUR_PI;
  }
}

/* get_total_kinetic_energy, ParticlesPhysics.py:389-429: epsilon inside rho^2 + 1. */
double oracle_cpu_total_kinetic_energy(const double* pos, const double* str, const double* rad,
                                       int64_t n) {
  double* part = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    const double px = pos[3 * i], py = pos[3 * i + 1], pz = pos[3 * i + 2];
    const double bx = str[3 * i], by = str[3 * i + 1], bz = str[3 * i + 2];
    const double ri = rad[i];
    double e = 0.0;
    for (int64_t j = 0; j < n; ++j) {
      if (i == j) continue;
      const double rx = px - pos[3 * j], ry = py - pos[3 * j + 1], rz = pz - pos[3 * j + 2];
      const double rn = pow(rx * rx + ry * ry + rz * rz, 0.5);
      const double ux = rx / rn, uy = ry / rn, uz = rz / rn;
      const double s = (ri + rad[j]) * 0.5;
      const double rho = rn / s;
      const double p1 = rho * rho + 1.0 + ORACLE_EPS;
      const double t1 = 2.0 * rho / pow(p1, 0.5);
      const double t2 = rho * rho * rho / pow(p1, 1.5);
      const double ax = str[3 * j], ay = str[3 * j + 1], az = str[3 * j + 2];
      const double q1 = bx * ax + by * ay + bz * az;
      const double q2 = ux * bx + uy * by + uz * bz;
      const double q3 = ux * ax + uy * ay + uz * az;
      e += (t1 * q1 + t2 * (q2 * q3 - q1)) / rn;
    }
    part[i] = e;
  }
  const double total = ordered_sum(part, n) / (16.0 * M_PI);
  free(part);
  return total;
}

/* get_total_helicity, ParticlesPhysics.py:433-468 (no second 1/(4*pi)). */
double oracle_cpu_total_helicity(const double* pos, const double* str, const double* rad,
                                 int64_t n) {
  double* part = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    const double px = pos[3 * i], py = pos[3 * i + 1], pz = pos[3 * i + 2];
    const double bx = str[3 * i], by = str[3 * i + 1], bz = str[3 * i + 2];
    const double ri = rad[i];
    double h = 0.0;
    for (int64_t j = 0; j < n; ++j) {
      if (i == j) continue;
      const double rx = px - pos[3 * j], ry = py - pos[3 * j + 1], rz = pz - pos[3 * j + 2];
      const double rm = pow(rx * rx + ry * ry + rz * rz, 0.5);
      const double s = (ri + rad[j]) * 0.5;
      const double rho = rm / s;
      const double rho2 = rho * rho;
      const double term = (rho2 + 2.5) / (s * s * s * pow(rho2 + 1.0, 2.5));
      const double ax = str[3 * j], ay = str[3 * j + 1], az = str[3 * j + 2];
      const double cx = by * az - bz * ay, cy = bz * ax - bx * az, cz = bx * ay - by * ax;
      h += (rx * cx + ry * cy + rz * cz) * term;
    }
    part[i] = h;
  }
  const double total = ordered_sum(part, n) / (4.0 * M_PI);
  free(part);
  return total;
}

/* get_total_enstrophy, ParticlesPhysics.py:518-550 (no second 1/(4*pi)). */
double oracle_cpu_total_enstrophy(const double* pos, const double* str, const double* rad,
                                  int64_t n) {
  return oracle_gpu_total_enstrophy(pos, str, rad, n, 0);
}
