"""The no-allocation entry point, vpm_selfinduced_velocity_noalloc, through the C ABI.

It serves callers that may not allocate device memory themselves (for example a plugin
inside a host application that owns the GPU's memory budget through its own pool): they
hand over only inputs and outputs, and the library works in a static scratch array of its
own.  This test compares it with the workspace entry point, vpm_selfinduced_velocity, and
with the oracle (the reference's GPU semantics restated in C) on two calls in a row with
different inputs (the shared array keeps the first call's contents), checks that a call
changes the device's free memory by nothing, and that sizes above the limit are refused.
The file name sorts last so that a run stopping at the first failure has already run every
other test."""
import numpy as np
import pytest
import torch

import oracle
from conftest import normwise

pytestmark = pytest.mark.gpu

TOL = {0: 1e-12, 1: 1e-6}  # FP64 drop-in bar; FP32-compensated velocity bar


def _field(n, seed):
    from openonda_b200 import configs

    f = configs.random_cloud(n, seed=seed)
    f.radii *= 4
    return f


def _cuda(f):
    dev = torch.device("cuda", 0)
    return [torch.from_numpy(z).to(dev) for z in (f.positions, f.strengths, f.radii)]


def _with_workspace(lib, x, a, s, precision, stream):
    from openonda_b200 import _lib, kernels

    n = x.shape[0]
    prec = {0: "fp64", 1: "fp32c"}[precision]
    need = kernels.workspace_bytes("selfinduced_velocity", prec, n, n)
    ws = torch.empty(max(need, 256), dtype=torch.uint8, device=x.device)
    out = torch.empty((n, 3), dtype=torch.float64, device=x.device)
    _lib.check(lib.vpm_selfinduced_velocity(x.data_ptr(), a.data_ptr(), s.data_ptr(), n,
                                            out.data_ptr(), precision, ws.data_ptr(),
                                            ws.numel(), stream))
    return out


@pytest.mark.parametrize("precision", [0, 1])
def test_noalloc_matches_workspace_entry_point_and_oracle_twice(precision):
    from openonda_b200 import _lib

    lib = _lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    for call, (n, seed) in enumerate([(32768, 1), (5000, 2)]):
        f = _field(n, seed)
        x, a, s = _cuda(f)
        out = torch.full((n, 3), float("nan"), dtype=torch.float64, device=x.device)
        _lib.check(lib.vpm_selfinduced_velocity_noalloc(x.data_ptr(), a.data_ptr(), s.data_ptr(),
                                                        n, out.data_ptr(), precision, stream))
        ref = _with_workspace(lib, x, a, s, precision, stream)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.all(np.isfinite(got)), f"call {call}"
        err = normwise(got, ref.cpu().numpy())
        assert err <= TOL[precision], (call, err)
        # against the oracle (FP64; for the FP32-compensated form on the FP32-rounded inputs
        # that form computes with): all targets of the small call, a window of the large one
        r = (lambda z: z.astype(np.float32).astype(np.float64)) if precision else np.asarray
        t0, t1 = (0, n) if n <= 5000 else (n // 2 - 256, n // 2 + 256)
        want = oracle.gpu.selfinduced_velocity_range(r(f.positions), r(f.strengths),
                                                     r(f.radii), t0, t1)
        err_o = normwise(got[t0:t1], want)
        assert err_o <= TOL[precision], (call, err_o)


def test_noalloc_call_changes_free_device_memory_by_nothing():
    from openonda_b200 import _lib

    lib = _lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    x, a, s = _cuda(_field(20000, 4))
    out = torch.empty((x.shape[0], 3), dtype=torch.float64, device=x.device)

    def call(precision):
        _lib.check(lib.vpm_selfinduced_velocity_noalloc(x.data_ptr(), a.data_ptr(), s.data_ptr(),
                                                        x.shape[0], out.data_ptr(), precision,
                                                        stream))

    for precision in (0, 1):
        call(precision)  # warm-up: address lookup, kernel attributes
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for precision in (0, 1, 0, 1):
        call(precision)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, (free0, free1)


def test_noalloc_refuses_sizes_above_the_limit():
    from openonda_b200 import _lib

    lib = _lib.load()
    n = 32769
    x, a, s = _cuda(_field(n, 3))
    out = torch.empty((n, 3), dtype=torch.float64, device=x.device)
    rc = lib.vpm_selfinduced_velocity_noalloc(x.data_ptr(), a.data_ptr(), s.data_ptr(), n,
                                              out.data_ptr(), 0,
                                              torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.VPM_ERR_ARG
    assert b"32768" in lib.vpm_last_error()
