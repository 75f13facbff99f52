import os
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if REPO not in sys.path:
    sys.path.insert(0, REPO)

GOLDEN = os.path.join(REPO, "tests", "golden")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")
    config.addinivalue_line("markers", "slow: longer CPU test")


def pytest_collection_modifyitems(config, items):
    # GPU tests are skipped (not failed) when no device is present, so `-m "not gpu"`
    # and plain runs both work on a CPU-only host.
    try:
        import torch

        has_gpu = torch.cuda.is_available()
    except Exception:  # pragma: no cover
        has_gpu = False
    if has_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


def normwise(got, ref):
    """max|got - ref| / max|ref| (NaN-aware: NaN positions must coincide)."""
    import numpy as np

    got = np.asarray(got, dtype=np.float64)
    ref = np.asarray(ref, dtype=np.float64)
    assert got.shape == ref.shape, (got.shape, ref.shape)
    nan_g, nan_r = np.isnan(got), np.isnan(ref)
    assert np.array_equal(nan_g, nan_r), "NaN pattern differs"
    g, r = got[~nan_r], ref[~nan_r]
    if r.size == 0:
        return 0.0
    scale = np.max(np.abs(r))
    diff = np.max(np.abs(g - r))
    if scale == 0.0:
        return float(diff)
    return float(diff / scale)


def golden(name):
    import numpy as np

    return np.load(os.path.join(GOLDEN, name))


def pair_scale(strengths, radii):
    """Magnitude bound for a pair-summed scalar: (sum |alpha|)^2 / min(sigma)."""
    import numpy as np

    a = np.sqrt(np.sum(np.asarray(strengths) ** 2, axis=1))
    if a.size == 0:
        return 0.0
    return float(np.sum(a) ** 2 / np.min(radii))


def scalar_close(got, ref, rel, scale, abs_frac=1e-15):
    """True when got matches ref to `rel` relative, or to abs_frac * scale absolute.

    The absolute branch covers sums that cancel to ~0 (e.g. the helicity of a planar
    ring), where a relative test only measures rounding noise."""
    import numpy as np

    if np.isnan(ref):
        return bool(np.isnan(got))
    d = abs(got - ref)
    return d <= rel * abs(ref) or d <= abs_frac * scale


def ic_cases():
    """The seeded initial-condition / lattice cases that tests/golden/ic.npz was made from."""
    import importlib.util

    spec = importlib.util.spec_from_file_location(
        "make_golden", os.path.join(GOLDEN, "make_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.ic_cases()
