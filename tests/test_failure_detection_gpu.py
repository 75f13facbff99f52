"""Failure detection without a GPU fault: a kernel waits on an mbarrier phase that nothing
completes; the library's bounded wait gives up after ~1 s, records the timeout in the device
error word and returns, and the context stays usable for the next computation."""
import time

import numpy as np
import pytest
import torch

import oracle
from conftest import normwise

pytestmark = pytest.mark.gpu


def test_bounded_wait_times_out_and_reports():
    from openonda_b200 import _lib, configs, kernels

    lib = _lib.load()
    kernels.device_errors(clear=True)
    flag = torch.zeros(1, dtype=torch.int32, device="cuda")
    t0 = time.perf_counter()
    _lib.check(lib.vpm_selftest_bounded_wait(flag.data_ptr(),
                                             torch.cuda.current_stream().cuda_stream))
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    assert int(flag.item()) == 1
    assert 0.5 <= dt <= 10.0
    assert kernels.device_errors(clear=True) & 1 == 1
    assert kernels.device_errors(clear=False) == 0
    # the context still computes correctly
    f = configs.random_cloud(500, seed=1)
    x, a, s = (torch.from_numpy(z).cuda() for z in (f.positions, f.strengths, f.radii))
    u = kernels.selfinduced_velocity(x, a, s)
    assert normwise(u.cpu().numpy(),
                    oracle.gpu.get_selfinduced_velocity(f.positions, f.strengths, f.radii)) <= 1e-12
    assert kernels.device_errors() == 0


def test_host_side_errors_raise():
    from openonda_b200 import _lib, kernels

    x = torch.zeros((4, 3), dtype=torch.float64, device="cuda")
    with pytest.raises(ValueError):
        kernels.selfinduced_velocity(x, torch.zeros((5, 3), dtype=torch.float64, device="cuda"),
                                     torch.ones(4, dtype=torch.float64, device="cuda"))
    with pytest.raises(TypeError):
        kernels.selfinduced_velocity(x.float(), x.float(),
                                     torch.ones(4, dtype=torch.float32, device="cuda"))
    with pytest.raises(_lib.VPMError):
        _lib.check(_lib.load().vpm_sweep_records(99, x.data_ptr(), 4, 0, 4, 0, x.data_ptr(),
                                                 None, 0, x.data_ptr(), 0, None))
