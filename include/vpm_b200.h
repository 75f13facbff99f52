/*
 * vpm_b200.h -- C ABI of the B200 (sm_100a) VPM pair-sum library (libvpm_b200.so).
 *
 * The pair-sum entry points replace the module-level functions of OpenONDA's Numba-CUDA
 * physics module, OpenONDA/solvers/VPM/ParticlesPhysicsCuda.py, which
 * vpmModule.ParticleSystem selects in _load_physics_module (vpmModule.py:141-154).  The
 * element-wise step kernels restate vpmModule.ParticleSystem's updates, and the
 * initial-condition entry points OpenONDA/utilities/vpm_flow_models.py and
 * vpm_solver_helper.py.  The fused sums, the adjoint, the uniform-core flag and the
 * no-allocation variant have no counterpart in the reference (each says so).
 *
 * Conventions
 *   - Arrays are DEVICE pointers in the reference's layout: positions, strengths and
 *     outputs (n,3) row-major float64; radii and viscosities (n,) float64.
 *   - `precision`: VPM_FP64 computes in FP64 and is the exact drop-in (matches the
 *     reference's routine to 1e-12 relative); VPM_FP32C computes the pair terms in FP32
 *     with FP64 carries (inputs are rounded to FP32 once, outputs are FP64);
 *     VPM_FP32C_REFINED adds one Newton step to the hardware rsqrt.
 *   - `workspace`/`workspace_bytes`: caller-owned device scratch of at least
 *     vpm_workspace_bytes(op, precision, m, n) bytes, 256-byte aligned.  The library never
 *     allocates.
 *   - `stream`: a cudaStream_t (NULL = legacy default stream).  Calls are asynchronous
 *     with respect to the host; scalar results are written to a device double.
 *   - Return value: VPM_OK (0) or an error code; vpm_last_error() gives the message for
 *     the calling thread.  Inputs are never modified; nothing throws across the ABI.
 *   - Radii must be positive.  Results are deterministic for a given device and sizes.
 */
#ifndef VPM_B200_H
#define VPM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VPM_ABI_VERSION 1

enum vpm_status {
  VPM_OK = 0,
  VPM_ERR_ARG = 1,        /* bad size, null pointer, unknown op or precision */
  VPM_ERR_ALIGN = 2,      /* workspace not 256-byte aligned */
  VPM_ERR_WORKSPACE = 3,  /* workspace smaller than vpm_workspace_bytes() */
  VPM_ERR_CUDA = 4,       /* CUDA runtime error (launch, attribute query) */
  VPM_ERR_ARCH = 5        /* current device is not compute capability 10.0 */
};

enum vpm_precision { VPM_FP64 = 0, VPM_FP32C = 1, VPM_FP32C_REFINED = 2 };
/* Flag OR-ed into `precision` (self sums, records and workspace queries): the caller
 * guarantees that every particle has the same core radius, so the pair core
 * (sigma_i + sigma_j)/2 is sigma_i and the kernels skip forming it (2 FP32 operations fewer
 * per pair, same values).  The pack step checks the claim and sets bit 1 of the device error
 * word when a radius differs from radii[0] (results are then wrong).  Probe sums, the kinetic
 * energy and the adjoint ignore the flag.  No counterpart in the reference. */
#define VPM_UNIFORM_CORE 0x100

enum vpm_op {
  VPM_OP_SELFINDUCED_VELOCITY = 0,
  VPM_OP_INDUCED_VELOCITY_AT = 1,
  VPM_OP_VORTICITY_FIELD_AT = 2,
  VPM_OP_STRENGTH_GRADIENTS = 3,
  VPM_OP_STRENGTH_GRADIENTS_PSE = 4,
  VPM_OP_TOTAL_KINETIC_ENERGY = 5,
  VPM_OP_TOTAL_HELICITY = 6,
  VPM_OP_TOTAL_ENSTROPHY = 7,
  VPM_OP_VELOCITY_AND_STRENGTH_GRADIENTS = 8,
  VPM_OP_RHS_VJP = 9,             /* adjoint of (velocity, stretching) */
  VPM_OP_RHS_VJP_PSE = 10,        /* adjoint of (velocity, stretching + PSE) */
  VPM_OP_KINETIC_ENERGY_GRAD = 11, /* gradient of the kinetic energy */
  VPM_OP_LES_STEP_SUMS = 12,       /* velocity, stretching, vorticity, enstrophy in one sweep */
  VPM_OP_LES_TEST_FILTER = 13      /* test-filter sums of the least-squares LES coefficient */
};

/* ---- library information ------------------------------------------------------------ */
int vpm_abi_version(void);
const char* vpm_last_error(void);
/* Check that the current device is sm_100 (B200); VPM_ERR_ARCH otherwise. */
int vpm_check_device(void);
/* The compute capability the library's kernels were compiled for on the current device
 * (cudaFuncGetAttributes binaryVersion / ptxVersion, e.g. 100 for sm_100a). */
int vpm_binary_info(int* binary_version, int* ptx_version);
/* Read (and optionally clear) the device error word: bit 0 = a bounded wait timed out (the
 * sweep that gave up wrote no partial sums, so that call's outputs are not valid), bit 1 =
 * VPM_UNIFORM_CORE was passed for radii that are not all equal.  The word is sticky until
 * cleared. */
int vpm_device_errors(int* out, int clear);
/* Failure-detection self-test: one block waits on an mbarrier phase that never completes; the
 * bounded wait gives up after ~1 s, sets bit 0 of the device error word, writes 1 to the
 * device int `timed_out` and the kernel returns (no fault, the context stays usable). */
int vpm_selftest_bounded_wait(int* timed_out, void* stream);
/* Scratch bytes `op` needs for m targets and n sources (m = n for self sums). */
size_t vpm_workspace_bytes(int op, int precision, int64_t m, int64_t n);
/* Launch plan of `op`: target blocks, source splits, threads/block, targets/thread. */
int vpm_plan_info(int op, int precision, int64_t m, int64_t n, int64_t* target_blocks,
                  int* splits, int* threads, int* targets_per_thread);

/* ---- reference entry points ------------------------------------------------------------ */

/* get_induced_velocity_at (ParticlesPhysicsCuda.py:11-34, kernel :39-97):
 * velocity at m probe points from n particles, source core sigma_j, pairs r^2<=1e-8 skipped. */
int vpm_induced_velocity_at(const double* targets, int64_t m, const double* positions,
                            const double* strengths, const double* radii, int64_t n,
                            double* velocities, int precision, void* workspace,
                            size_t workspace_bytes, void* stream);

/* get_selfinduced_velocity (ParticlesPhysicsCuda.py:103-127, kernel :133-191):
 * j != i, pair core (sigma_i + sigma_j)/2. */
int vpm_selfinduced_velocity(const double* positions, const double* strengths,
                             const double* radii, int64_t n, double* velocities, int precision,
                             void* workspace, size_t workspace_bytes, void* stream);

/* get_vorticity_field_at (ParticlesPhysicsCuda.py:198-219, kernel :291-346): zeta-kernel
 * vorticity at m probe points.  One output row per target (the reference sizes its output by
 * n and is only correct for m == n; for m == n the results agree). */
int vpm_vorticity_field_at(const double* targets, int64_t m, const double* positions,
                           const double* strengths, const double* radii, int64_t n,
                           double* vorticities, int precision, void* workspace,
                           size_t workspace_bytes, void* stream);

/* get_strength_gradients (ParticlesPhysicsCuda.py:351-370, kernel :375-445): vortex
 * stretching, transpose scheme. */
int vpm_strength_gradients(const double* positions, const double* strengths,
                           const double* radii, int64_t n, double* dalpha_dt, int precision,
                           void* workspace, size_t workspace_bytes, void* stream);

/* get_strength_gradients_PSE (ParticlesPhysicsCuda.py:452-473, kernel :478-530):
 * PSE diffusion with the target's viscosity nu_i. */
int vpm_strength_gradients_pse(const double* positions, const double* strengths,
                               const double* radii, const double* viscosities, int64_t n,
                               double* dalpha_dt, int precision, void* workspace,
                               size_t workspace_bytes, void* stream);

/* get_total_kinetic_energy (ParticlesPhysicsCuda.py:537-558, kernel :563-642).
 * The accumulator starts at zero (the reference never clears it). */
int vpm_total_kinetic_energy(const double* positions, const double* strengths,
                             const double* radii, int64_t n, double* energy, int precision,
                             void* workspace, size_t workspace_bytes, void* stream);

/* get_total_helicity (ParticlesPhysicsCuda.py:647-668, kernel :673-750).
 * ref_extra_4pi != 0 keeps the wrapper's second division by 4*pi (:668). */
int vpm_total_helicity(const double* positions, const double* strengths, const double* radii,
                       int64_t n, int ref_extra_4pi, double* helicity, int precision,
                       void* workspace, size_t workspace_bytes, void* stream);

/* get_total_enstrophy (ParticlesPhysicsCuda.py:756-777, kernel :867-920), all pairs.
 * ref_extra_4pi != 0 keeps the wrapper's second division by 4*pi (:777). */
int vpm_total_enstrophy(const double* positions, const double* strengths, const double* radii,
                        int64_t n, int ref_extra_4pi, double* enstrophy, int precision,
                        void* workspace, size_t workspace_bytes, void* stream);

/* get_selfinduced_velocity + get_strength_gradients (vpmModule.py:704 and :753-774 call
 * them on the same positions/strengths/radii) fused into one sweep. */
int vpm_velocity_and_strength_gradients(const double* positions, const double* strengths,
                                        const double* radii, int64_t n, double* velocities,
                                        double* dalpha_dt, int precision, void* workspace,
                                        size_t workspace_bytes, void* stream);

/* FP32-compensated self sums of velocity + stretching, velocity alone, PSE and the LES step
 * sums, the adjoint of (u, S [+ P]), and the FP64 self sums of velocity + stretching, velocity
 * alone, PSE and the LES step (vpm_velocity_and_strength_gradients, vpm_selfinduced_velocity,
 * vpm_strength_gradients_pse, vpm_les_step_sums, vpm_rhs_vjp, and vpm_sweep_records over all
 * records) with n >= this value evaluate each unordered pair once for both particles
 * (deterministic tile-pair schedule, about n / (2 T m) launches for tiles of T = 512 or 768
 * particles and m diagonal pairs per launch).  Where those launches are short (up to ~150000
 * particles), the diagonal tiles run on a second stream of the library's, forked from and
 * joined to the caller's stream by events inside the call, so stream order and CUDA-graph
 * capture see one call as before; that stream is created by the first such call in a context
 * (make it before any stream capture).  Sets the threshold and returns the previous one
 * (default 24576).  No counterpart in the reference. */
int64_t vpm_set_symmetric_min_n(int64_t n);
/* Kernel launches of one sweep of `op` (sweep and finalize, not the packing of the inputs)
 * for m targets and n sources under the current plan; -1 on error. */
int64_t vpm_sweep_launches(int op, int precision, int64_t m, int64_t n);

/* The four pair sums of one dynamic-LES time step on the same state, in one sweep:
 * get_selfinduced_velocity, get_strength_gradients, get_vorticity_field_at(positions, ...)
 * and get_total_enstrophy (vpmModule.py:704, :753, :640, :644).  `enstrophy` is a device
 * scalar; ref_extra_4pi as in vpm_total_enstrophy.  Workspace: VPM_OP_LES_STEP_SUMS. */
int vpm_les_step_sums(const double* positions, const double* strengths, const double* radii,
                      int64_t n, double* velocities, double* dalpha_dt, double* vorticity,
                      double* enstrophy, int ref_extra_4pi, int precision, void* workspace,
                      size_t workspace_bytes, void* stream);

/* ---- adjoint (differentiation form; no counterpart in the reference) ------------------ */
/* Vector-Jacobian product of the right-hand side F = (u, S [+ P]) of the coupled ODE
 * dx/dt = u, dalpha/dt = S + P, where u, S, P are the sums of vpm_selfinduced_velocity,
 * vpm_strength_gradients and vpm_strength_gradients_pse: given cotangents grad_velocities
 * and grad_rates (n,3), writes (dL/dx, dL/dalpha) (n,3), dL/dsigma (n,) and, when
 * `viscosities` is not NULL (PSE included), dL/dnu (n,) into grad_viscosities (may be NULL).
 * One deterministic sweep over all pairs; workspace from vpm_workspace_bytes(VPM_OP_RHS_VJP
 * or VPM_OP_RHS_VJP_PSE, precision, n, n). */
int vpm_rhs_vjp(const double* positions, const double* strengths, const double* radii,
                const double* viscosities, int64_t n, const double* grad_velocities,
                const double* grad_rates, double* grad_positions, double* grad_strengths,
                double* grad_radii, double* grad_viscosities, int precision, void* workspace,
                size_t workspace_bytes, void* stream);
/* Gradient of vpm_total_kinetic_energy w.r.t. positions, strengths and radii. */
int vpm_kinetic_energy_grad(const double* positions, const double* strengths,
                            const double* radii, int64_t n, double* grad_positions,
                            double* grad_strengths, double* grad_radii, int precision,
                            void* workspace, size_t workspace_bytes, void* stream);

/* ---- pre-packed records (device-resident state, target shards) ----------------------- */
/* Bytes of one packed particle record (64; FP32 records hold every value twice). */
size_t vpm_record_bytes(int precision);
/* Pack n particles from the reference layout into records {x,y,z,sigma,ax,ay,az,nu} of the
 * compute precision (viscosities may be NULL: nu = 0).  `records` is 16-byte aligned. */
int vpm_pack_records(const double* positions, const double* strengths, const double* radii,
                     const double* viscosities, int64_t n, int precision, void* records,
                     void* stream);
/* Self sum `op` (any VPM_OP_* except the two probes) for the m targets
 * records[target_begin, target_begin + m) against all n source records; outputs hold m
 * rows (out2 is the stretching output of VPM_OP_VELOCITY_AND_STRENGTH_GRADIENTS, scalars
 * are partial sums over the m targets).  This is the unit of work one rank runs when the
 * targets are sharded across GPUs.  Same workspace rule as the reference entry points. */
int vpm_sweep_records(int op, const void* records, int64_t n, int64_t target_begin, int64_t m,
                      int ref_extra_4pi, double* out, double* out2, int precision,
                      void* workspace, size_t workspace_bytes, void* stream);

/* ---- pair shards across GPUs (VPM_OP_VELOCITY_AND_STRENGTH_GRADIENTS, every precision) --
 * The both-sides schedule of a self sum over n records split between ranks by tiles: rank r
 * runs the diagonal tiles [tile_begin, tile_end) and the diagonal pairs [pair_begin,
 * pair_end) of the plan every rank makes for n, over all n gathered records, and sums its
 * accumulator sets into `rows` (n, values) FP64 -- one particle's sums per row, in a fixed
 * order.  The sum of all ranks' rows (a reduce-scatter between the GPUs, by row ranges) is
 * what the single-GPU sweep sums; vpm_finalize_pairs_partial turns a rank's summed rows into
 * its velocities and stretching.  Replaces, per rank, the target-shard sweep
 * vpm_sweep_records, which cannot evaluate a pair once for both particles when the two
 * particles sit on different ranks. */
/* Tiles, diagonal pairs and diagonal pairs per launch of the plan for n, values per row,
 * workspace bytes of one vpm_sweep_pairs_partial call (VPM_ERR_ARG if n does not take the
 * both-sides schedule).  Any output pointer may be NULL. */
int vpm_pairs_layout(int op, int precision, int64_t n, int64_t* tiles, int64_t* pairs,
                     int* pairs_per_launch, int* values, size_t* workspace_bytes);
int vpm_sweep_pairs_partial(int op, const void* records, int64_t n, int64_t tile_begin,
                            int64_t tile_end, int64_t pair_begin, int64_t pair_end,
                            double* rows, int precision, void* workspace,
                            size_t workspace_bytes, void* stream);
/* Outputs of targets records[target_begin, target_begin + m) from their summed rows (m,
 * values): out = velocities (m,3), out2 = stretching (m,3). */
int vpm_finalize_pairs_partial(int op, const double* rows, const void* records,
                               int64_t target_begin, int64_t m, double* out, double* out2,
                               int precision, void* stream);

/* ---- device-resident time step (vpmModule.ParticleSystem), element-wise, HBM-bound ------ */
/* out = x + c k over `count` doubles: RK stages (vpmModule.py:580,604,637,641,676,680,684). */
int vpm_axpy(const double* x, const double* k, double c, int64_t count, double* out,
             void* stream);
/* out = x + dt/6 (k1 + 2 k2 + 2 k3 + k4): RK4 combine (vpmModule.py:688). */
int vpm_rk4_combine(const double* x, const double* k1, const double* k2, const double* k3,
                    const double* k4, double dt, int64_t count, double* out, void* stream);
/* Strengths <- BDF ladder step `time_step` with rate coefficient `coef` (dt, 2/3 dt, 6/11 dt,
 * 12/25 dt) and the reference's history rotation, in place (vpmModule.py:751-787, 801-841). */
int vpm_bdf_update(double* strengths, double* hist1, double* hist2, double* hist3,
                   const double* rate, int64_t count, int time_step, double coef, void* stream);
/* sigma <- sqrt(sigma^2 + C (nu + nu_t) dt), in place (vpmModule.py:853-860). */
int vpm_core_spreading(double* radii, const double* viscosities, const double* viscosities_t,
                       int64_t n, double C, double dt, void* stream);
/* Dynamic LES update (vpmModule.py:887-962): when advance_constant != 0, les_state =
 * {Cnu, enstrophy_ref, initialised} (device doubles) is advanced with the device scalar
 * `enstrophy` (vpmModule.py:887-909); then, for n > 0, nu_t is recomputed from the vorticity
 * with the current Cnu and committed when its maximum exceeds 1e-9 (vpmModule.py:916-962;
 * the maximum is written to nut_max when it is not NULL). */
size_t vpm_les_workspace_bytes(int64_t n);
int vpm_les_update(const double* vorticity, const double* radii, const double* enstrophy,
                   int64_t n, int advance_constant, double* les_state, double* viscosities_t,
                   double* nut_max, void* workspace, size_t workspace_bytes, void* stream);
/* Least-squares dynamic LES coefficient, FP64 (no counterpart in the reference, which only
 * rescales Cnu by its enstrophy ratio, vpmModule.py:887-909).  Germano identity for the
 * sub-filter kinetic energy k(D) = C^2 D^2 |w_D|^2 between the particle filter (core sigma) and
 * a test filter of core 2 sigma:
 *   L_i = (hat(|u|^2)_i - |hat u_i|^2) / 2,   M_i = (2 sigma_i)^2 |hat w_i|^2 - hat(sigma^2|w|^2)_i,
 *   Cnu = clip(sqrt(sum L M / sum M M), 1e-9, 0.0761)  (unchanged when either sum is <= 0).
 * vpm_les_lsq_weights writes the per-particle fields the test filter acts on, times the particle
 * volume |alpha|/|w|: weights (n,3) = (|u|^2 v, sigma^2 |w|^2 v, 0).  The caller forms, with the
 * pair-sum entry points and radii 2 sigma: hat u = vpm_selfinduced_velocity, and hat w with
 * hat f from one vpm_les_test_filter sweep (equal to vpm_vorticity_field_at(x, x, alpha,
 * 2 sigma) and vpm_vorticity_field_at(x, x, weights, 2 sigma)).  vpm_les_lsq_update reduces both sums in one block in a fixed order, writes them to
 * `sums` (2 device doubles, may be NULL) and updates les_state[0] (= Cnu) on the device. */
/* The two test-filter sums of the least-squares coefficient in one sweep (no counterpart in
 * the reference): the vorticity filter sum of vpm_vorticity_field_at(x, x, alpha, test_radii)
 * into test_vorticity (n,3), and the same filter applied to the first two columns of `fields`
 * (n,3; the weights of vpm_les_lsq_weights) into test_filtered (n,3, third column 0).
 * Workspace: vpm_workspace_bytes(VPM_OP_LES_TEST_FILTER, precision, n, n). */
int vpm_les_test_filter(const double* positions, const double* strengths,
                        const double* test_radii, const double* fields, int64_t n,
                        double* test_vorticity, double* test_filtered, int precision,
                        void* workspace, size_t workspace_bytes, void* stream);
int vpm_les_lsq_weights(const double* velocities, const double* vorticity,
                        const double* strengths, const double* radii, int64_t n,
                        double* weights, void* stream);
int vpm_les_lsq_update(const double* test_velocities, const double* test_vorticity,
                       const double* test_filtered, const double* radii, int64_t n,
                       double* les_state, double* sums, void* stream);
/* Strength relaxation towards the vorticity direction, in place (vpmModule.py:867-883). */
int vpm_relax_strengths(double* strengths, const double* vorticity, int64_t n, double alpha,
                        void* stream);
/* FP64 O(N) diagnostics (vpmModule.py:264-284): out10 = [sum|a|, sum a (3),
 * linear impulse 1/2 sum x x a (3), angular impulse 1/3 sum x x (x x a) (3)]. */
int vpm_particle_diagnostics(const double* positions, const double* strengths, int64_t n,
                             double* out10, void* stream);

/* ---- initial conditions and lattices on the device ------------------------------------
 * Restate OpenONDA/utilities/vpm_flow_models.py and vpm_solver_helper.py; the reference builds
 * these fields with host numpy/numba.  All arrays are device, FP64, AoS (n,3) or (n,). */

/* Workspace (256-byte aligned) needed by vpm_ic_vortex_ring for n particles. */
size_t vpm_ic_workspace_bytes(int64_t n);
/* vortex_ring_vpm (vpm_flow_models.py:87-163): Gaussian-core ring of radius ring_radius in the
 * y-z plane around center, Widnall-type core displacement epsilon_w cos/sin(phase_w + n_w
 * theta); strengths = omega * volume, rescaled so that sum|alpha| = 2 pi R Gamma; radii and
 * viscosities filled with the particle values.  Velocities (zero in the reference) are the
 * caller's.  A field whose total |alpha| is zero gives non-finite strengths (the reference
 * raises ZeroDivisionError). */
int vpm_ic_vortex_ring(const double* positions, const double* volumes, int64_t n,
                       double particle_radius, double particle_viscosity, double center_x,
                       double center_y, double center_z, double ring_radius,
                       double ring_strength, double ring_thickness, double epsilon_w,
                       double phase_w, double n_w, double* strengths, double* radii,
                       double* viscosities, void* workspace, size_t workspace_bytes,
                       void* stream);
/* lamb_oseen_vpm (vpm_flow_models.py:14-83): axial (z) vorticity of a Gaussian core around
 * (center_x + eps sin(phase + N z), center_y + eps cos(phase + N z)). */
int vpm_ic_lamb_oseen(const double* positions, const double* volumes, int64_t n,
                      double particle_radius, double particle_viscosity, double center_x,
                      double center_y, double center_z, double vortex_strength,
                      double core_radius, double epsilon_w, double phase_w, double n_w,
                      double* strengths, double* radii, double* viscosities, void* stream);
/* Lattices.  box_limits / center are HOST arrays ([xmin,xmax,ymin,ymax,zmin,zmax] / 3).  The
 * point count is written to *count; with points == volumes == NULL nothing is launched (size
 * query), otherwise capacity (points) must be >= *count.
 * get_rectangular_point_distribuition (dims 3) / get_2D_rectangular_point_distribuition
 * (dims 2, z = 0), vpm_solver_helper.py:21-117: */
int vpm_lattice_rectangular(const double* box_limits, double spacing, int dims,
                            double* points, double* volumes, int64_t capacity, int64_t* count,
                            void* stream);
/* get_hexagonal_point_distribution, vpm_solver_helper.py:120-161: */
int vpm_lattice_hexagonal(const double* box_limits, double spacing, double* points,
                          double* volumes, int64_t capacity, int64_t* count, void* stream);
/* get_cylindrical_point_distribuition, vpm_solver_helper.py:164-253; axis 0/1/2 = 'x'/'y'/'z': */
int vpm_lattice_cylindrical(double particle_distance, double radius, double height,
                            const double* center, int axis, double* points, double* volumes,
                            int64_t capacity, int64_t* count, void* stream);

/* ---- no-allocation variant ------------------------------------------------------------ */
#define VPM_NOALLOC_MAX_N 32768
#define VPM_NOALLOC_SCRATCH_BYTES (8u << 20)
/* Self-induced velocity (same inputs, output and precisions as vpm_selfinduced_velocity) for
 * callers that may not allocate device memory, e.g. a plugin inside a host application that
 * owns the GPU's memory through its own pool.  No counterpart in the reference.  It takes no
 * workspace and calls no allocator: its scratch is a static 8 MiB device array inside the
 * library (reserved on every GPU that loads it), so n <= VPM_NOALLOC_MAX_N (larger n returns
 * VPM_ERR_ARG).  All calls share that array: calls that overlap on the GPU race.  The array
 * has one address per CUDA context; the first call in a context (per device) looks that
 * address up (and, for sizes whose sweep runs its diagonal tiles on a second stream, creates
 * that stream and its two events), so make it before any stream capture.  If a sweep's
 * bounded wait gives up
 * (bit 0 of the vpm_device_errors word), the output is built from the previous call's
 * partial sums: check the device error word where that matters. */
int vpm_selfinduced_velocity_noalloc(const double* positions, const double* strengths,
                                     const double* radii, int64_t n, double* velocities,
                                     int precision, void* stream);

/* ---- measurement helpers -------------------------------------------------------------- */
/* Pipe throughput kernels: blocks x threads threads each run `iters` iterations of 16
 * independent chains; one value per thread lands in `sink` (blocks*threads floats, or doubles
 * for FP64).  fp64 = 0: FP32 FMA, 1: FP64 FMA, 2: FP32 MUFU rsqrt (SFU), 3: packed FP32x2
 * FMA (FFMA2), 4: 8 FFMA2 + 16 FFMA chains.  Operation count = blocks*threads*iters*16 (lane
 * FMAs: twice that for 3 and 4). */
int vpm_launch_fma_peak(int fp64, int blocks, int threads, int iters, void* sink, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* VPM_B200_H */
