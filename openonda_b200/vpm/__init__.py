"""VPM solver pieces mirroring ``OpenONDA.solvers.VPM``."""
from . import ParticlesPhysicsB200  # noqa: F401
