"""GPU parity: the CUDA library, called through its C ABI (via the drop-in module and the
tensor API), against the golden vectors of the reference and against the pinned oracle.

Tolerances: FP64 path <= 1e-12 normwise relative (max|d|/max|ref|) -- the reference
routine's own bar; FP32-compensated path <= 1e-6 normwise relative against the FP64 path
on the same FP32-rounded inputs."""
import numpy as np
import pytest

import oracle
from conftest import golden, normwise, pair_scale, scalar_close

pytestmark = pytest.mark.gpu

FP64_TOL = 1e-12
FP32C_TOL = 1e-6  # velocity (and PSE, vorticity, enstrophy)
# Stretching on ring-shaped fields is a small residual of cancelling near-neighbour
# terms, which amplifies the ulp-level FP32 pair error; its error is stated, bounded here.
FP32C_STRETCH_TOL = 2e-6


@pytest.fixture(scope="module")
def pp():
    from openonda_b200.vpm import ParticlesPhysicsB200 as m

    m.set_precision("fp64")
    m.set_reference_scaling(True)
    return m


def _cases(npz):
    return sorted({k.split("/")[0] for k in npz.files})


GPU_G = golden("gpu_kernels.npz")


@pytest.mark.parametrize("case", _cases(GPU_G))
def test_fp64_dropin_vs_reference_numba_cuda(pp, case):
    g = GPU_G
    x, a, s, v, t = (g[f"{case}/{k}"] for k in
                     ("positions", "strengths", "radii", "viscosities", "targets"))
    assert normwise(pp.get_induced_velocity_at(t, x, a, s), g[f"{case}/induced_velocity_at"]) \
        <= FP64_TOL
    assert normwise(pp.get_selfinduced_velocity(x, a, s), g[f"{case}/selfinduced_velocity"]) \
        <= FP64_TOL
    assert normwise(pp.get_vorticity_field_at(x, x, a, s), g[f"{case}/vorticity_field_at"]) \
        <= FP64_TOL
    assert normwise(pp.get_strength_gradients(x, a, s), g[f"{case}/strength_gradients"]) \
        <= FP64_TOL
    assert normwise(pp.get_strength_gradients_PSE(x, a, s, v),
                    g[f"{case}/strength_gradients_PSE"]) <= FP64_TOL
    scale = pair_scale(a, s)
    for fn in ("total_helicity", "total_enstrophy"):
        got = getattr(pp, "get_" + fn)(x, a, s)
        assert scalar_close(got, float(g[f"{case}/{fn}"]), FP64_TOL, scale), fn
    ke_ref = float(g[f"{case}/total_kinetic_energy"])
    ke = pp.get_total_kinetic_energy(x, a, s)
    if np.isnan(ke_ref):
        # Two distinct particles at one point: the reference divides 0/0; the B200 kernel
        # evaluates the finite limit of the same pair term.
        assert case == "coincident24" and np.isfinite(ke)
        x2 = x.copy()
        x2[17] += 1e-7
        assert abs(ke - oracle.gpu.get_total_kinetic_energy(x2, a, s)) <= 1e-5 * abs(ke)
    else:
        assert scalar_close(ke, ke_ref, FP64_TOL, scale)


def test_fp64_ring8192_vs_reference(pp):
    g = golden("ring8192.npz")
    x, a, s, v, t = g["positions"], g["strengths"], g["radii"], g["viscosities"], g["targets"]
    assert normwise(pp.get_induced_velocity_at(t, x, a, s), g["induced_velocity_at"]) <= FP64_TOL
    assert normwise(pp.get_strength_gradients(x, a, s), g["strength_gradients"]) <= FP64_TOL
    assert normwise(pp.get_selfinduced_velocity(x, a, s),
                    oracle.gpu.get_selfinduced_velocity(x, a, s)) <= FP64_TOL
    assert normwise(pp.get_strength_gradients_PSE(x, a, s, v),
                    oracle.gpu.get_strength_gradients_PSE(x, a, s, v)) <= FP64_TOL
    assert normwise(pp.get_vorticity_field_at(x, x, a, s),
                    oracle.gpu.get_vorticity_field_at(x, x, a, s)) <= FP64_TOL
    for fn in ("total_kinetic_energy", "total_helicity", "total_enstrophy"):
        got = getattr(pp, "get_" + fn)(x, a, s)
        ref = getattr(oracle.gpu, "get_" + fn)(x, a, s)
        assert scalar_close(got, ref, FP64_TOL, pair_scale(a, s)), fn


def test_fused_matches_separate_and_oracle(pp):
    from openonda_b200 import configs

    f = configs.random_cloud(3001, seed=7)  # ragged size
    x, a, s = f.positions, f.strengths, f.radii
    u, g = pp.get_selfinduced_velocity_and_strength_gradients(x, a, s)
    assert normwise(u, oracle.gpu.get_selfinduced_velocity(x, a, s)) <= FP64_TOL
    assert normwise(g, oracle.gpu.get_strength_gradients(x, a, s)) <= FP64_TOL
    assert normwise(u, pp.get_selfinduced_velocity(x, a, s)) <= 1e-14
    assert normwise(g, pp.get_strength_gradients(x, a, s)) <= 1e-14


def _round32(*arrs):
    return [np.asarray(z, dtype=np.float32).astype(np.float64) for z in arrs]


@pytest.mark.parametrize("precision", ["fp32c", "fp32c_refined"])
@pytest.mark.parametrize("field", ["ring8192", "cloud16384"])
def test_fp32c_error_vs_fp64(pp, precision, field):
    from openonda_b200 import configs

    f = configs.ring_8192() if field == "ring8192" else configs.random_cloud(16384, seed=3)
    x, a, s, v = _round32(f.positions, f.strengths, f.radii, f.viscosities)
    us = pp.get_selfinduced_velocity(x, a, s, precision=precision)
    gs = pp.get_strength_gradients(x, a, s, precision=precision)
    u64, g64 = pp.get_selfinduced_velocity_and_strength_gradients(x, a, s, precision="fp64")
    u32, g32 = pp.get_selfinduced_velocity_and_strength_gradients(x, a, s, precision=precision)
    eu, eg = normwise(u32, u64), normwise(g32, g64)
    print(f"{field} {precision}: velocity {eu:.2e} stretching {eg:.2e}")
    assert normwise(us, u64) <= FP32C_TOL and normwise(gs, g64) <= FP32C_STRETCH_TOL
    assert eu <= FP32C_TOL and eg <= FP32C_STRETCH_TOL
    p64 = pp.get_strength_gradients_PSE(x, a, s, v, precision="fp64")
    p32 = pp.get_strength_gradients_PSE(x, a, s, v, precision=precision)
    assert normwise(p32, p64) <= FP32C_TOL
    w64 = pp.get_vorticity_field_at(x, x, a, s, precision="fp64")
    w32 = pp.get_vorticity_field_at(x, x, a, s, precision=precision)
    assert normwise(w32, w64) <= FP32C_TOL
    e64 = pp.get_total_enstrophy(x, a, s, precision="fp64")
    e32 = pp.get_total_enstrophy(x, a, s, precision=precision)
    assert abs(e32 - e64) <= FP32C_TOL * abs(e64)


def test_empty_and_single(pp):
    z = np.zeros((0, 3))
    assert pp.get_selfinduced_velocity(z, z, np.zeros(0)).shape == (0, 3)
    assert pp.get_strength_gradients(z, z, np.zeros(0)).shape == (0, 3)
    assert pp.get_total_kinetic_energy(z, z, np.zeros(0)) == 0.0
    x = np.array([[0.1, 0.2, 0.3]])
    a = np.array([[1e-3, 2e-3, -1e-3]])
    s = np.array([0.05])
    assert np.all(pp.get_selfinduced_velocity(x, a, s) == 0.0)
    assert np.all(pp.get_strength_gradients(x, a, s) == 0.0)
    assert np.all(pp.get_strength_gradients_PSE(x, a, s, np.array([1e-4])) == 0.0)
    assert pp.get_total_kinetic_energy(x, a, s) == 0.0
    assert pp.get_total_enstrophy(x, a, s) == pytest.approx(
        oracle.gpu.get_total_enstrophy(x, a, s), rel=1e-14)
    # probes with no sources, and no probes
    assert np.all(pp.get_induced_velocity_at(np.ones((5, 3)), z, z, np.zeros(0)) == 0.0)
    assert pp.get_induced_velocity_at(z, x, a, s).shape == (0, 3)


@pytest.mark.parametrize("m", [1, 37, 513, 2049])
def test_probe_sizes(pp, m):
    from openonda_b200 import configs

    f = configs.random_cloud(1500, seed=21)
    t = np.random.default_rng(m).uniform(-1.2, 1.2, size=(m, 3))
    t[0] = f.positions[3]  # exactly on a source
    x, a, s = f.positions, f.strengths, f.radii
    assert normwise(pp.get_induced_velocity_at(t, x, a, s),
                    oracle.gpu.get_induced_velocity_at(t, x, a, s)) <= FP64_TOL
    assert normwise(pp.get_vorticity_field_at(t, x, a, s),
                    oracle.gpu.get_vorticity_field_at(t, x, a, s)) <= FP64_TOL


@pytest.mark.parametrize("n", [2, 31, 32, 33, 255, 257, 1023, 4097])
def test_ragged_sizes(pp, n):
    from openonda_b200 import configs

    f = configs.random_cloud(n, seed=n)
    f.radii *= 8  # overlapping cores
    x, a, s, v = f.positions, f.strengths, f.radii, f.viscosities
    assert normwise(pp.get_selfinduced_velocity(x, a, s),
                    oracle.gpu.get_selfinduced_velocity(x, a, s)) <= FP64_TOL
    assert normwise(pp.get_strength_gradients(x, a, s),
                    oracle.gpu.get_strength_gradients(x, a, s)) <= FP64_TOL
    assert normwise(pp.get_strength_gradients_PSE(x, a, s, v),
                    oracle.gpu.get_strength_gradients_PSE(x, a, s, v)) <= FP64_TOL
    assert scalar_close(pp.get_total_kinetic_energy(x, a, s),
                        oracle.gpu.get_total_kinetic_energy(x, a, s), FP64_TOL, pair_scale(a, s))


def test_deterministic_bitwise(pp):
    import torch

    from openonda_b200 import configs, kernels

    f = configs.random_cloud(20000, seed=5)
    x = torch.from_numpy(f.positions).cuda()
    a = torch.from_numpy(f.strengths).cuda()
    s = torch.from_numpy(f.radii).cuda()
    for prec in ("fp64", "fp32c"):
        u1, g1 = kernels.velocity_and_strength_gradients(x, a, s, precision=prec)
        u2, g2 = kernels.velocity_and_strength_gradients(x, a, s, precision=prec)
        assert torch.equal(u1, u2) and torch.equal(g1, g2)
        e1 = kernels.total_kinetic_energy(x, a, s, precision=prec)
        e2 = kernels.total_kinetic_energy(x, a, s, precision=prec)
        assert torch.equal(e1, e2)
    assert kernels.device_errors() == 0


def test_abi_workspace_and_argument_errors():
    import torch

    from openonda_b200 import _lib, kernels

    lib = _lib.load()
    n = 1000
    x = torch.rand((n, 3), dtype=torch.float64, device="cuda")
    s = torch.full((n,), 0.05, dtype=torch.float64, device="cuda")
    out = torch.empty((n, 3), dtype=torch.float64, device="cuda")
    need = kernels.workspace_bytes("selfinduced_velocity", "fp64", n, n)
    ws = torch.empty(need, dtype=torch.uint8, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    rc = lib.vpm_selfinduced_velocity(x.data_ptr(), x.data_ptr(), s.data_ptr(), n,
                                      out.data_ptr(), 0, ws.data_ptr(), need - 1, st)
    assert rc == _lib.VPM_ERR_WORKSPACE
    rc = lib.vpm_selfinduced_velocity(x.data_ptr(), x.data_ptr(), s.data_ptr(), n,
                                      out.data_ptr(), 0, ws.data_ptr() + 8, need, st)
    assert rc == _lib.VPM_ERR_ALIGN
    rc = lib.vpm_selfinduced_velocity(x.data_ptr(), x.data_ptr(), s.data_ptr(), n,
                                      out.data_ptr(), 0, ws.data_ptr(), need, st)
    assert rc == _lib.VPM_OK
    assert lib.vpm_check_device() == _lib.VPM_OK
    with pytest.raises(_lib.VPMError):
        _lib.check(lib.vpm_sweep_records(0, x.data_ptr(), n, n - 5, 10, 0, out.data_ptr(), None,
                                         0, ws.data_ptr(), need, st))


def test_records_target_shards_reassemble():
    """Target shards computed from packed records equal the full sweep (multi-GPU unit)."""
    import torch

    from openonda_b200 import _lib, configs, kernels

    f = configs.random_cloud(5000, seed=9)
    x = torch.from_numpy(f.positions).cuda()
    a = torch.from_numpy(f.strengths).cuda()
    s = torch.from_numpy(f.radii).cuda()
    v = torch.from_numpy(f.viscosities).cuda()
    lib = _lib.load()
    st = torch.cuda.current_stream().cuda_stream
    for prec in ("fp64", "fp32c"):
        pc = _lib.precision_code(prec)
        rb = lib.vpm_record_bytes(pc)
        rec = torch.empty(5000 * rb, dtype=torch.uint8, device="cuda")
        _lib.check(lib.vpm_pack_records(x.data_ptr(), a.data_ptr(), s.data_ptr(), v.data_ptr(),
                                        5000, pc, rec.data_ptr(), st))
        u_full, g_full = kernels.velocity_and_strength_gradients(x, a, s, precision=prec)
        ke_full = kernels.total_kinetic_energy(x, a, s, precision=prec)
        parts_u, parts_g, ke = [], [], 0.0
        for b, e in [(0, 1700), (1700, 3333), (3333, 5000)]:
            m = e - b
            u = torch.empty((m, 3), dtype=torch.float64, device="cuda")
            g = torch.empty((m, 3), dtype=torch.float64, device="cuda")
            need = kernels.workspace_bytes("velocity_and_strength_gradients", prec, m, 5000)
            ws = torch.empty(need, dtype=torch.uint8, device="cuda")
            _lib.check(lib.vpm_sweep_records(8, rec.data_ptr(), 5000, b, m, 0, u.data_ptr(),
                                             g.data_ptr(), pc, ws.data_ptr(), need, st))
            parts_u.append(u)
            parts_g.append(g)
            e_out = torch.empty((), dtype=torch.float64, device="cuda")
            need = kernels.workspace_bytes("total_kinetic_energy", prec, m, 5000)
            ws = torch.empty(need, dtype=torch.uint8, device="cuda")
            _lib.check(lib.vpm_sweep_records(5, rec.data_ptr(), 5000, b, m, 0, e_out.data_ptr(),
                                             None, pc, ws.data_ptr(), need, st))
            ke += float(e_out)
        assert normwise(torch.cat(parts_u).cpu().numpy(), u_full.cpu().numpy()) <= 1e-14
        assert normwise(torch.cat(parts_g).cpu().numpy(), g_full.cpu().numpy()) <= 1e-14
        assert abs(ke - float(ke_full)) <= 1e-12 * abs(float(ke_full))


def test_loaded_kernels_are_sm100a_binaries():
    """The kernels the runtime loaded on this device were compiled for compute capability 10.0
    (the library embeds sm_100a code only)."""
    import ctypes

    from openonda_b200 import _lib

    b, p = ctypes.c_int(), ctypes.c_int()
    _lib.check(_lib.load().vpm_binary_info(ctypes.byref(b), ctypes.byref(p)))
    assert b.value == 100, b.value
    assert _lib.load().vpm_check_device() == 0


@pytest.mark.parametrize("n", [1, 97, 2048, 5000])
def test_les_step_sums_vs_oracle(n):
    """One sweep = get_selfinduced_velocity + get_strength_gradients +
    get_vorticity_field_at(x, x, ...) + get_total_enstrophy (reference GPU semantics)."""
    import torch

    from openonda_b200 import configs, kernels

    f = configs.random_cloud(n, seed=n)
    f.radii *= 4
    x, a, s = (torch.from_numpy(np.ascontiguousarray(z)).cuda()
               for z in (f.positions, f.strengths, f.radii))
    u, g, w, e = kernels.les_step_sums(x, a, s, ref_extra_4pi=True, precision="fp64")
    o = oracle.gpu
    assert normwise(u.cpu().numpy(), o.get_selfinduced_velocity(f.positions, f.strengths,
                                                                f.radii)) <= FP64_TOL
    assert normwise(g.cpu().numpy(), o.get_strength_gradients(f.positions, f.strengths,
                                                              f.radii)) <= FP64_TOL
    assert normwise(w.cpu().numpy(), o.get_vorticity_field_at(f.positions, f.positions,
                                                              f.strengths, f.radii)) <= FP64_TOL
    ref_e = o.get_total_enstrophy(f.positions, f.strengths, f.radii)
    assert abs(float(e) - ref_e) <= 1e-12 * abs(ref_e)
    # FP32-compensated against FP64 on the same FP32-rounded inputs
    r32 = lambda z: z.float().double()
    x, a, s = r32(x), r32(a), r32(s)
    ref = kernels.les_step_sums(x, a, s, precision="fp64")
    got = kernels.les_step_sums(x, a, s, precision="fp32c")
    for k, tol in zip(range(3), (FP32C_TOL, FP32C_STRETCH_TOL, FP32C_TOL)):
        assert normwise(got[k].cpu().numpy(), ref[k].cpu().numpy()) <= tol, k
    assert abs(float(got[3]) - float(ref[3])) <= FP32C_TOL * abs(float(ref[3]))


def test_les_step_sums_empty_and_errors():
    import torch

    from openonda_b200 import _lib, kernels

    z = torch.zeros((0, 3), dtype=torch.float64, device="cuda")
    u, g, w, e = kernels.les_step_sums(z, z, torch.zeros(0, dtype=torch.float64,
                                                         device="cuda"))
    assert u.shape == (0, 3) and float(e) == 0.0
    lib = _lib.load()
    assert lib.vpm_les_step_sums(None, None, None, 4, None, None, None, None, 1, 0, None, 0,
                                 None) == _lib.VPM_ERR_ARG


@pytest.mark.parametrize("precision", ["fp64", "fp32c"])
def test_uniform_core_form_matches_general_form(precision):
    """VPM_UNIFORM_CORE: with all cores equal the pair core is sigma_i, so the specialised
    sweeps must give the general sweeps' values (same pair terms; only the launch plan, and
    with it the FP64 summation order, may differ)."""
    import torch

    from openonda_b200 import configs, kernels

    f = configs.vortex_ring(32, 64, 1.0, 1.0, 0.1, nu=1e-3)  # N = 2048, one core
    assert np.all(f.radii == f.radii[0])
    x, a, s, nu = (torch.from_numpy(np.ascontiguousarray(z)).cuda()
                   for z in (f.positions, f.strengths, f.radii, f.viscosities))
    kernels.device_errors()
    tol = 1e-14 if precision == "fp64" else 1e-7
    pairs = [
        (kernels.selfinduced_velocity, (x, a, s)),
        (kernels.strength_gradients, (x, a, s)),
        (kernels.velocity_and_strength_gradients, (x, a, s)),
        (kernels.strength_gradients_pse, (x, a, s, nu)),
        (kernels.les_step_sums, (x, a, s)),
        (kernels.total_enstrophy, (x, a, s)),
    ]
    for fn, args in pairs:
        ref = fn(*args, precision=precision)
        got = fn(*args, precision=precision, uniform_core=True)
        ref = ref if isinstance(ref, tuple) else (ref,)
        got = got if isinstance(got, tuple) else (got,)
        for r, g in zip(ref, got):
            assert normwise(g.cpu().numpy(), r.cpu().numpy()) <= tol, fn.__name__
    assert kernels.device_errors() == 0
    # a false claim is flagged (bit 1), not silently accepted
    s2 = s.clone()
    s2[5] *= 1.5
    kernels.selfinduced_velocity(x, a, s2, precision=precision, uniform_core=True)
    assert kernels.device_errors() & 2
    assert kernels.device_errors() == 0


def test_non_finite_input_propagates_like_reference(pp):
    """A NaN position reaches every target of the self sums (as in the reference, which has
    no guard), while the probe sums skip the pair (their r^2 > 1e-8 test is false for NaN,
    ParticlesPhysicsCuda.py:77) -- same NaN pattern as the oracle, no fault."""
    from openonda_b200 import configs

    f = configs.random_cloud(300, seed=8)
    x = f.positions.copy()
    x[17, 1] = np.nan
    t = f.positions[:40] * 0.9
    o = oracle.gpu
    for name in ("get_selfinduced_velocity", "get_strength_gradients"):
        got = getattr(pp, name)(x, f.strengths, f.radii)
        ref = getattr(o, name)(x, f.strengths, f.radii)
        assert np.array_equal(np.isnan(got), np.isnan(ref)), name
        assert np.isnan(got).all(), name
    got = pp.get_induced_velocity_at(t, x, f.strengths, f.radii)
    ref = o.get_induced_velocity_at(t, x, f.strengths, f.radii)
    assert np.array_equal(np.isnan(got), np.isnan(ref))
    assert normwise(got, ref) <= FP64_TOL
    from openonda_b200 import kernels

    assert kernels.device_errors() == 0
