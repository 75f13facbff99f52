"""B200-native engine for the all-pairs particle sums of OpenONDA's vortex particle method.

Public entry points:

* :mod:`openonda_b200.vpm.ParticlesPhysicsB200` -- drop-in for the reference's physics
  modules (``ParticlesPhysicsCuda`` / ``ParticlesPhysics``): same function names and
  arguments, backed by the sm_100a CUDA library through its C ABI.
* :mod:`openonda_b200.vpm.vpmModule` -- ``ParticleSystem`` with the reference's
  constructor and methods, keeping particle state resident on the GPU.
* :mod:`openonda_b200.kernels` -- tensor-level access to every kernel (FP64 drop-in
  form, FP32-compensated form, adjoint).
"""
from .version import __version__  # noqa: F401
