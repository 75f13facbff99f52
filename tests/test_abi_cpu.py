"""CPU-only checks of the C-ABI library: it is built for sm_100a, loads, and exports every
entry point declared in include/vpm_b200.h with a ctypes signature.  No compute calls."""
import os
import re
import subprocess

import pytest

from conftest import REPO

HEADER = os.path.join(REPO, "include", "vpm_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(vpm_[a-z0-9_]+)\s*\(", text)))


def test_header_declares_reference_entry_points():
    syms = declared_symbols()
    for name in ["vpm_induced_velocity_at", "vpm_selfinduced_velocity", "vpm_vorticity_field_at",
                 "vpm_strength_gradients", "vpm_strength_gradients_pse",
                 "vpm_total_kinetic_energy", "vpm_total_helicity", "vpm_total_enstrophy"]:
        assert name in syms


def test_library_builds_and_exports_every_declared_symbol():
    from openonda_b200 import _lib, build

    build.build()
    assert os.path.exists(_lib.LIB_PATH)
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\bT (vpm_[a-z0-9_]+)\b", out))
    missing = [s for s in declared_symbols() if s not in exported]
    assert not missing, missing
    lib = _lib.load()
    for s in declared_symbols():
        assert hasattr(lib, s)
        assert s in _lib.SIGNATURES, f"{s} has no ctypes signature"


def test_library_is_built_for_sm100a_only():
    """The build recipe passes exactly one -gencode, for sm_100a (a runtime check of the loaded
    kernels' binary version is in the GPU tests)."""
    from openonda_b200 import build

    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]
    assert not any(f.startswith(("-arch", "--gpu-architecture", "-gencode", "--generate-code"))
                   for f in build.FLAGS)


def test_abi_version_and_errors_without_device():
    from openonda_b200 import _lib

    lib = _lib.load()
    assert lib.vpm_abi_version() == 1
    # Invalid arguments are rejected before any CUDA call.
    rc = lib.vpm_selfinduced_velocity(None, None, None, -1, None, 0, None, 0, None)
    assert rc == _lib.VPM_ERR_ARG
    assert b"negative" in lib.vpm_last_error()
    rc = lib.vpm_selfinduced_velocity(None, None, None, 4, None, 0, None, 0, None)
    assert rc == _lib.VPM_ERR_ARG
    rc = lib.vpm_selfinduced_velocity(None, None, None, 0, None, 7, None, 0, None)
    assert rc == _lib.VPM_ERR_ARG  # unknown precision


def test_python_layer_rejects_host_tensors():
    import torch

    from openonda_b200 import kernels

    x = torch.zeros((4, 3), dtype=torch.float64)
    with pytest.raises(ValueError):
        kernels.selfinduced_velocity(x, x, torch.ones(4, dtype=torch.float64))
    with pytest.raises(ValueError):
        kernels.selfinduced_velocity(x, x, torch.ones(4, dtype=torch.float64), precision="fp16")
