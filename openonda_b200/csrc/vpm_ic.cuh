// vpm_ic.cuh -- initial conditions and particle lattices built on the device, so that a
// million-particle field is set up where it is used instead of in host loops and copied.
// Included by vpm_abi.cu (the library is one translation unit).
//
// Each kernel restates one function of OpenONDA/utilities/vpm_flow_models.py or
// vpm_solver_helper.py with the reference's operation order.  Products and sums use the _rn
// intrinsics (no FMA contraction) so that lattice coordinates round like numpy's
// `start + i * step`; the transcendental functions are CUDA's double-precision ones.
#pragma once

namespace vpm {
namespace {

constexpr int kIcThreads = 256;
constexpr int kIcMaxBlocks = 1184;  // 148 SMs x 8 blocks: grid-stride cap for the reduction

// np.linspace(start, stop, num)[i] as numpy and numba compute it: start + i * step with
// step = (stop - start) / (num - 1), and the last element set to stop.
__device__ __forceinline__ double linspace_at(double start, double stop, int64_t num,
                                              int64_t i) {
  if (num > 1 && i == num - 1) return stop;
  if (num <= 1) return start;
  const double step = __ddiv_rn(__dsub_rn(stop, start), double(num - 1));
  return __dadd_rn(start, __dmul_rn(double(i), step));
}

// np.arange(start, stop, step)[i] as numba computes it: start + i * step.
__device__ __forceinline__ double arange_at(double start, double step, int64_t i) {
  return __dadd_rn(start, __dmul_rn(double(i), step));
}

struct RingIc {
  double cx, cy, cz, radius, peak, thickness2, eps, phase, nw, gamma_theo;
  double particle_radius, particle_viscosity;
};

// vortex_ring_vpm (vpm_flow_models.py:87-163), first pass: unnormalised strengths, cores,
// viscosities, and each block's share of the total circulation sum |alpha| (fixed order).
__global__ void __launch_bounds__(kIcThreads)
ring_ic_kernel(const double* __restrict__ pos, const double* __restrict__ vol, int64_t n,
               RingIc p, double* __restrict__ strengths, double* __restrict__ radii,
               double* __restrict__ visc, double* __restrict__ block_sum) {
  __shared__ double red[kIcThreads];
  double acc = 0.0;
  for (int64_t i = int64_t(blockIdx.x) * kIcThreads + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * kIcThreads) {
    const double X = __dsub_rn(pos[3 * i], p.cx);
    double Y = __dsub_rn(pos[3 * i + 1], p.cy);
    double Z = __dsub_rn(pos[3 * i + 2], p.cz);
    const double theta = atan2(Z, Y);
    const double arg = __dadd_rn(p.phase, __dmul_rn(p.nw, theta));
    Y = __dsub_rn(Y, __dmul_rn(p.eps, cos(arg)));
    Z = __dsub_rn(Z, __dmul_rn(p.eps, sin(arg)));
    const double ryz = sqrt(__dadd_rn(__dmul_rn(Y, Y), __dmul_rn(Z, Z)));
    const double d = fabs(__dsub_rn(ryz, p.radius));
    const double mag = __dmul_rn(p.peak, exp(__ddiv_rn(-__dmul_rn(d, d), p.thickness2)));
    const double decay = exp(__ddiv_rn(-__dmul_rn(X, X), p.thickness2));
    const double wy = __dmul_rn(__dmul_rn(-mag, sin(theta)), decay);
    const double wz = __dmul_rn(__dmul_rn(mag, cos(theta)), decay);
    const double v = vol[i];
    const double ax = __dmul_rn(0.0, v), ay = __dmul_rn(wy, v), az = __dmul_rn(wz, v);
    strengths[3 * i] = ax;
    strengths[3 * i + 1] = ay;
    strengths[3 * i + 2] = az;
    radii[i] = p.particle_radius;
    visc[i] = p.particle_viscosity;
    acc += sqrt(__dadd_rn(__dadd_rn(__dmul_rn(ax, ax), __dmul_rn(ay, ay)), __dmul_rn(az, az)));
  }
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int w = kIcThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  if (threadIdx.x == 0) block_sum[blockIdx.x] = red[0];
}

// Second pass: every block sums the block shares in the same fixed order (so all blocks
// hold the same total), then scales its particles by |Gamma_theo / Gamma_total|.  A zero
// total gives an infinite factor (the reference raises ZeroDivisionError there).
__global__ void __launch_bounds__(kIcThreads)
ring_scale_kernel(const double* __restrict__ block_sum, int nblocks, double gamma_theo,
                  int64_t n, double* __restrict__ strengths) {
  __shared__ double red[kIcThreads];
  double acc = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += kIcThreads) acc += block_sum[b];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int w = kIcThreads / 2; w > 0; w >>= 1) {
    if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
    __syncthreads();
  }
  const double f = fabs(__ddiv_rn(gamma_theo, red[0]));
  for (int64_t i = int64_t(blockIdx.x) * kIcThreads + threadIdx.x; i < 3 * n;
       i += int64_t(gridDim.x) * kIcThreads)
    strengths[i] = __dmul_rn(strengths[i], f);
}

struct LambOseenIc {
  double cx, cy, cz, peak, core2, eps, phase, nw;
  double particle_radius, particle_viscosity;
};

// lamb_oseen_vpm (vpm_flow_models.py:14-83): axial vorticity of a Gaussian core whose axis
// is displaced sinusoidally along z.
__global__ void lamb_oseen_ic_kernel(const double* __restrict__ pos,
                                     const double* __restrict__ vol, int64_t n, LambOseenIc p,
                                     double* __restrict__ strengths, double* __restrict__ radii,
                                     double* __restrict__ visc) {
  const int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double z = pos[3 * i + 2];
  const double arg = __dadd_rn(p.phase, __dmul_rn(p.nw, z));
  const double px = __dadd_rn(p.cx, __dmul_rn(p.eps, sin(arg)));
  const double py = __dadd_rn(p.cy, __dmul_rn(p.eps, cos(arg)));
  const double x = __dsub_rn(pos[3 * i], px);
  const double y = __dsub_rn(pos[3 * i + 1], py);
  const double r = sqrt(__dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y)));
  const double wz = __dmul_rn(p.peak, exp(__ddiv_rn(-__dmul_rn(r, r), p.core2)));
  strengths[3 * i] = 0.0;
  strengths[3 * i + 1] = 0.0;
  strengths[3 * i + 2] = __dmul_rn(wz, vol[i]);
  radii[i] = p.particle_radius;
  visc[i] = p.particle_viscosity;
}

// get_rectangular_point_distribuition / get_2D_... (vpm_solver_helper.py:21-117): meshgrid
// (indexing 'ij') of three linspaces, raveled in C order; z = 0 in 2D (nz = 1).
__global__ void rect_lattice_kernel(double x0, double x1, double y0, double y1, double z0,
                                    double z1, int64_t nx, int64_t ny, int64_t nz, int dims,
                                    double vol, double* __restrict__ pts,
                                    double* __restrict__ vols) {
  const int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t total = nx * ny * nz;
  if (p >= total) return;
  const int64_t ix = p / (ny * nz), iy = (p / nz) % ny, iz = p % nz;
  pts[3 * p] = linspace_at(x0, x1, nx, ix);
  pts[3 * p + 1] = linspace_at(y0, y1, ny, iy);
  pts[3 * p + 2] = dims == 3 ? linspace_at(z0, z1, nz, iz) : 0.0;
  vols[p] = vol;
}

// get_hexagonal_point_distribution (vpm_solver_helper.py:120-161): loops z, y (row i), x;
// odd rows shifted by spacing / 2.
__global__ void hex_lattice_kernel(double x0, double y0, double z0, double sx, double sy,
                                   double sz, int64_t nx, int64_t ny, int64_t nz, double half,
                                   double vol, double* __restrict__ pts,
                                   double* __restrict__ vols) {
  const int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if (p >= nx * ny * nz) return;
  const int64_t iz = p / (ny * nx), iy = (p / nx) % ny, ix = p % nx;
  const double off = (iy % 2 == 1) ? half : 0.0;
  pts[3 * p] = __dadd_rn(arange_at(x0, sx, ix), off);
  pts[3 * p + 1] = arange_at(y0, sy, iy);
  pts[3 * p + 2] = arange_at(z0, sz, iz);
  vols[p] = vol;
}

struct CylLattice {
  double radius, height, dr, dz, dtheta, axis_vol, c[3];
  int64_t nr, nzp, nth;  // radii, z levels (num_points_height + 1), angles kept (num - 1)
  int axis;              // 0 = x, 1 = y, 2 = z
};

// get_cylindrical_point_distribuition (vpm_solver_helper.py:164-253): rings of points
// for r in linspace(dr, R, nr), z in linspace(-H/2, H/2, nz + 1) and theta in
// linspace(0, 2 pi, nth)[:-1], then one point per z level on the axis.
__global__ void cyl_lattice_kernel(CylLattice g, double* __restrict__ pts,
                                   double* __restrict__ vols) {
  const int64_t p = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  const int64_t body = g.nr * g.nzp * g.nth;
  if (p >= body + g.nzp) return;
  double a, b, zi, v;  // in-plane coordinates, axial coordinate, volume
  if (p < body) {
    const int64_t ir = p / (g.nzp * g.nth), iz = (p / g.nth) % g.nzp, it = p % g.nth;
    const double ri = linspace_at(g.dr, g.radius, g.nr, ir);
    zi = linspace_at(-0.5 * g.height, 0.5 * g.height, g.nzp, iz);
    const double th = linspace_at(0.0, 2.0 * M_PI, g.nth + 1, it);
    a = __dmul_rn(ri, cos(th));
    b = __dmul_rn(ri, sin(th));
    v = __dmul_rn(__dmul_rn(__dmul_rn(ri, g.dtheta), g.dr), g.dz);
  } else {
    zi = linspace_at(-0.5 * g.height, 0.5 * g.height, g.nzp, p - body);
    a = 0.0;
    b = 0.0;
    v = g.axis_vol;
  }
  double q[3];
  if (g.axis == 0) {
    q[0] = zi; q[1] = a; q[2] = b;
  } else if (g.axis == 1) {
    q[0] = a; q[1] = zi; q[2] = b;
  } else {
    q[0] = a; q[1] = b; q[2] = zi;
  }
  pts[3 * p] = __dadd_rn(q[0], g.c[0]);
  pts[3 * p + 1] = __dadd_rn(q[1], g.c[1]);
  pts[3 * p + 2] = __dadd_rn(q[2], g.c[2]);
  vols[p] = v;
}

// ---- host-side lattice sizes (same arithmetic as the reference) -----------------------
void rect_counts(const double* b, double spacing, int dims, int64_t* nx, int64_t* ny,
                 int64_t* nz) {
  auto num = [&](double lo, double hi) {
    int64_t k = int64_t(std::ceil((hi - lo) / spacing)) + 1;
    return (k % 2 == 0) ? k + 1 : k;
  };
  *nx = num(b[0], b[1]);
  *ny = num(b[2], b[3]);
  *nz = dims == 3 ? num(b[4], b[5]) : 1;
}

int64_t arange_count(double start, double stop, double step) {
  const double c = std::ceil((stop - start) / step);
  return c > 0 ? int64_t(c) : 0;
}

}  // namespace
}  // namespace vpm

extern "C" {

size_t vpm_ic_workspace_bytes(int64_t n) {
  using namespace vpm;
  const int64_t b = (n + kIcThreads - 1) / kIcThreads;
  return align_up(size_t(b < 1 ? 1 : (b > kIcMaxBlocks ? kIcMaxBlocks : b)) * 8);
}

int vpm_ic_vortex_ring(const double* positions, const double* volumes, int64_t n,
                       double particle_radius, double particle_viscosity, double center_x,
                       double center_y, double center_z, double ring_radius,
                       double ring_strength, double ring_thickness, double epsilon_w,
                       double phase_w, double n_w, double* strengths, double* radii,
                       double* viscosities, void* workspace, size_t workspace_bytes,
                       void* stream) {
  using namespace vpm;
  if (n < 0) return fail(VPM_ERR_ARG, "vortex ring: n must be >= 0");
  if (n == 0) return VPM_OK;
  if (!positions || !volumes || !strengths || !radii || !viscosities)
    return fail(VPM_ERR_ARG, "vortex ring: null pointer");
  if (!(ring_thickness != 0.0)) return fail(VPM_ERR_ARG, "vortex ring: ring_thickness is 0");
  if (!workspace || reinterpret_cast<uintptr_t>(workspace) % kAlign != 0)
    return fail(VPM_ERR_ALIGN, "vortex ring workspace must be 256-byte aligned");
  if (workspace_bytes < vpm_ic_workspace_bytes(n))
    return fail(VPM_ERR_WORKSPACE, "vortex ring workspace too small");
  RingIc p;
  p.cx = center_x;
  p.cy = center_y;
  p.cz = center_z;
  p.radius = ring_radius;
  p.thickness2 = ring_thickness * ring_thickness;
  p.peak = ring_strength / (M_PI * p.thickness2);
  p.eps = epsilon_w;
  p.phase = phase_w;
  p.nw = n_w;
  p.gamma_theo = 2.0 * M_PI * ring_radius * ring_strength;
  p.particle_radius = particle_radius;
  p.particle_viscosity = particle_viscosity;
  const int64_t b = (n + kIcThreads - 1) / kIcThreads;
  const int nb = int(b > kIcMaxBlocks ? kIcMaxBlocks : b);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double* block_sum = static_cast<double*>(workspace);
  ring_ic_kernel<<<nb, kIcThreads, 0, st>>>(positions, volumes, n, p, strengths, radii,
                                             viscosities, block_sum);
  int rc = launch_status("vortex ring launch");
  if (rc) return rc;
  ring_scale_kernel<<<nb, kIcThreads, 0, st>>>(block_sum, nb, p.gamma_theo, n, strengths);
  return launch_status("vortex ring scale launch");
}

int vpm_ic_lamb_oseen(const double* positions, const double* volumes, int64_t n,
                      double particle_radius, double particle_viscosity, double center_x,
                      double center_y, double center_z, double vortex_strength,
                      double core_radius, double epsilon_w, double phase_w, double n_w,
                      double* strengths, double* radii, double* viscosities, void* stream) {
  using namespace vpm;
  if (n < 0) return fail(VPM_ERR_ARG, "lamb-oseen: n must be >= 0");
  if (n == 0) return VPM_OK;
  if (!positions || !volumes || !strengths || !radii || !viscosities)
    return fail(VPM_ERR_ARG, "lamb-oseen: null pointer");
  if (!(core_radius != 0.0)) return fail(VPM_ERR_ARG, "lamb-oseen: core_radius is 0");
  LambOseenIc p;
  p.cx = center_x;
  p.cy = center_y;
  p.cz = center_z;
  p.core2 = core_radius * core_radius;
  p.peak = vortex_strength / (M_PI * p.core2);
  p.eps = epsilon_w;
  p.phase = phase_w;
  p.nw = n_w;
  p.particle_radius = particle_radius;
  p.particle_viscosity = particle_viscosity;
  lamb_oseen_ic_kernel<<<ew_blocks(n), kEwThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      positions, volumes, n, p, strengths, radii, viscosities);
  return launch_status("lamb-oseen launch");
}

int vpm_lattice_rectangular(const double* box_limits, double spacing, int dims,
                            double* points, double* volumes, int64_t capacity, int64_t* count,
                            void* stream) {
  using namespace vpm;
  if (!box_limits || !count) return fail(VPM_ERR_ARG, "rectangular lattice: null pointer");
  if (dims != 2 && dims != 3) return fail(VPM_ERR_ARG, "rectangular lattice: dims is 2 or 3");
  if (!(spacing > 0.0)) return fail(VPM_ERR_ARG, "rectangular lattice: spacing must be > 0");
  const double* b = box_limits;
  for (int k = 0; k < 2 * dims; k += 2)
    if (!(b[k + 1] >= b[k])) return fail(VPM_ERR_ARG, "rectangular lattice: empty box");
  int64_t nx, ny, nz;
  rect_counts(b, spacing, dims, &nx, &ny, &nz);
  const int64_t total = nx * ny * nz;
  *count = total;
  if (!points && !volumes) return VPM_OK;
  if (!points || !volumes) return fail(VPM_ERR_ARG, "rectangular lattice: null output");
  if (capacity < total) return fail(VPM_ERR_ARG, "rectangular lattice: capacity too small");
  double box = (b[1] - b[0]) * (b[3] - b[2]);
  if (dims == 3) box *= (b[5] - b[4]);
  const double vol = box / double(total);
  rect_lattice_kernel<<<ew_blocks(total), kEwThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      b[0], b[1], b[2], b[3], dims == 3 ? b[4] : 0.0, dims == 3 ? b[5] : 0.0, nx, ny, nz, dims,
      vol, points, volumes);
  return launch_status("rectangular lattice launch");
}

int vpm_lattice_hexagonal(const double* box_limits, double spacing, double* points,
                          double* volumes, int64_t capacity, int64_t* count, void* stream) {
  using namespace vpm;
  if (!box_limits || !count) return fail(VPM_ERR_ARG, "hexagonal lattice: null pointer");
  if (!(spacing > 0.0)) return fail(VPM_ERR_ARG, "hexagonal lattice: spacing must be > 0");
  const double* b = box_limits;
  const double sq3 = std::sqrt(3.0);
  const double sy = spacing * sq3 / 2.0;
  const int64_t nx = arange_count(b[0], b[1] + spacing, spacing);
  const int64_t ny = arange_count(b[2], b[3] + sy, sy);
  const int64_t nz = arange_count(b[4], b[5] + spacing, spacing);
  const int64_t total = nx * ny * nz;
  *count = total;
  if (!points && !volumes) return VPM_OK;
  if (!points || !volumes) return fail(VPM_ERR_ARG, "hexagonal lattice: null output");
  if (capacity < total) return fail(VPM_ERR_ARG, "hexagonal lattice: capacity too small");
  if (total == 0) return VPM_OK;
  const double vol = spacing * spacing * spacing * sq3 / 2.0;
  hex_lattice_kernel<<<ew_blocks(total), kEwThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      b[0], b[2], b[4], spacing, sy, spacing, nx, ny, nz, spacing / 2.0, vol, points, volumes);
  return launch_status("hexagonal lattice launch");
}

int vpm_lattice_cylindrical(double particle_distance, double radius, double height,
                            const double* center, int axis, double* points, double* volumes,
                            int64_t capacity, int64_t* count, void* stream) {
  using namespace vpm;
  if (!center || !count) return fail(VPM_ERR_ARG, "cylindrical lattice: null pointer");
  if (axis < 0 || axis > 2)
    return fail(VPM_ERR_ARG, "Invalid axis. Choose from 'x', 'y', or 'z'.");
  if (!(particle_distance > 0.0) || !(radius > 0.0) || !(height > 0.0))
    return fail(VPM_ERR_ARG, "cylindrical lattice: sizes must be > 0");
  CylLattice g;
  g.nr = int64_t(radius / particle_distance);
  const int64_t nh = int64_t(height / particle_distance);
  const int64_t nth = int64_t(M_PI * radius / particle_distance);
  if (g.nr < 1 || nh < 1 || nth < 1)
    return fail(VPM_ERR_ARG, "cylindrical lattice: particle_distance larger than the cylinder");
  g.nzp = nh + 1;
  g.nth = nth - 1;
  g.radius = radius;
  g.height = height;
  g.dtheta = 2.0 * M_PI / double(nth);
  g.dz = height / double(nh);
  g.dr = radius / double(g.nr);
  g.axis_vol = M_PI * (radius * radius) * g.dz / double(g.nzp);
  g.c[0] = center[0];
  g.c[1] = center[1];
  g.c[2] = center[2];
  g.axis = axis;
  const int64_t total = g.nr * g.nzp * g.nth + g.nzp;
  *count = total;
  if (!points && !volumes) return VPM_OK;
  if (!points || !volumes) return fail(VPM_ERR_ARG, "cylindrical lattice: null output");
  if (capacity < total) return fail(VPM_ERR_ARG, "cylindrical lattice: capacity too small");
  cyl_lattice_kernel<<<ew_blocks(total), kEwThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      g, points, volumes);
  return launch_status("cylindrical lattice launch");
}

}  // extern "C"
