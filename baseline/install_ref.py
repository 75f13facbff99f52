"""Install the reference's VPM physics modules into ``baseline/_ref`` (run once, on the host
that has the reference checkout; ``baseline/_ref`` is kept out of version control).

    python baseline/install_ref.py [--reference /path/to/OpenONDA-checkout]

First it tries the package install the reference documents:

    pip install --no-index --no-build-isolation --find-links /opt/wheelhouse \
        --target baseline/_ref <reference>

That install needs an OpenFOAM environment (the package's setup.py compiles the FVM solver
extension and raises without FOAM_SRC), so where it fails, the recipe places the two
pure-Python modules of the VPM pair-sum path -- ``OpenONDA/solvers/VPM/ParticlesPhysicsCuda.py``
(Numba-CUDA) and ``OpenONDA/solvers/VPM/ParticlesPhysics.py`` (Numba CPU) -- unmodified under
``baseline/_ref/OpenONDA_VPM/``, which is all that path imports.  The CPU module's Numba
``np.dot`` on arrays needs SciPy's BLAS bindings, so SciPy (its wheel from the same offline
wheelhouse, no dependencies) goes to ``baseline/_ref/deps``, for hosts whose Python lacks it;
``load_reference_module`` appends that folder to ``sys.path``, after any installed SciPy.
The outcome is written to ``baseline/_ref/INSTALL.json``.  Measurement code loads the modules
by file path from there (see ``load_reference_module``) and reports them unavailable when the
folder is absent.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
VPM_DIR = os.path.join(REF_DIR, "OpenONDA_VPM")
DEPS_DIR = os.path.join(REF_DIR, "deps")
MODULES = ("ParticlesPhysicsCuda.py", "ParticlesPhysics.py")


def load_reference_module(name: str):
    """Import ``ParticlesPhysicsCuda`` or ``ParticlesPhysics`` from ``baseline/_ref`` by file
    path; raises FileNotFoundError when the reference is not installed."""
    path = os.path.join(VPM_DIR, name + ".py")
    if os.path.isdir(DEPS_DIR) and DEPS_DIR not in sys.path:
        sys.path.append(DEPS_DIR)
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is not installed (python baseline/install_ref.py)")
    spec = importlib.util.spec_from_file_location(f"openonda_ref_{name}", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default="/root/reference")
    args = ap.parse_args()
    ref = os.path.abspath(args.reference)
    os.makedirs(REF_DIR, exist_ok=True)
    record = {"reference": ref}
    cmd = [sys.executable, "-m", "pip", "install", "--no-index", "--no-build-isolation",
           "--find-links", "/opt/wheelhouse", "--target", REF_DIR, ref]
    res = subprocess.run(cmd, capture_output=True, text=True)
    record["pip_rc"] = res.returncode
    if res.returncode == 0:
        record["how"] = "pip install"
    else:
        tail = [ln.strip() for ln in (res.stdout + res.stderr).splitlines() if "Error" in ln]
        record["pip_error"] = tail[-1] if tail else "pip install failed"
        os.makedirs(VPM_DIR, exist_ok=True)
        for name in MODULES:
            shutil.copyfile(os.path.join(ref, "OpenONDA", "solvers", "VPM", name),
                            os.path.join(VPM_DIR, name))
        record["how"] = "VPM physics modules placed unmodified (package install failed)"
        record["modules"] = [os.path.join("OpenONDA", "solvers", "VPM", m) for m in MODULES]
    dep = [sys.executable, "-m", "pip", "install", "--no-index", "--no-deps", "--find-links",
           "/opt/wheelhouse", "--target", DEPS_DIR, "scipy"]
    res = subprocess.run(dep, capture_output=True, text=True)
    record["deps"] = {"scipy": "installed" if res.returncode == 0 else
                      (res.stdout + res.stderr).strip().splitlines()[-1:]}
    with open(os.path.join(REF_DIR, "INSTALL.json"), "w") as fh:
        json.dump(record, fh, indent=1)
    print(json.dumps(record))
    return 0


if __name__ == "__main__":
    sys.exit(main())
