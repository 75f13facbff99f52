"""Build recipe for the CPU oracle (test infrastructure).

``python -m oracle.build`` compiles ``vpm_oracle.c`` twice into ``oracle/_build/``:
a strict -O2 build (the parity oracle) and a -O3 -ffast-math build (the timed CPU
baseline).  Both target generic x86-64-v2 so the same binary runs on any host it is
copied to.
"""
from __future__ import annotations

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "vpm_oracle.c")
OUT = os.path.join(HERE, "_build")

_COMMON = ["gcc", "-shared", "-fPIC", "-fopenmp", "-march=x86-64-v2", "-std=gnu11", "-Wall"]
_VARIANTS = {
    "libvpm_oracle.so": ["-O2", "-fno-fast-math", "-ffp-contract=off"],
    "libvpm_oracle_fast.so": ["-O3", "-ffast-math"],
}


def build(force: bool = False) -> None:
    os.makedirs(OUT, exist_ok=True)
    src_mtime = os.path.getmtime(SRC)
    for name, flags in _VARIANTS.items():
        dst = os.path.join(OUT, name)
        if not force and os.path.exists(dst) and os.path.getmtime(dst) >= src_mtime:
            continue
        cmd = _COMMON + flags + ["-o", dst, SRC, "-lm"]
        subprocess.run(cmd, check=True)


if __name__ == "__main__":
    build(force=True)
