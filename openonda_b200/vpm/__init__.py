"""VPM solver pieces mirroring ``OpenONDA.solvers.VPM``."""
from . import ParticlesPhysicsB200  # noqa: F401
from . import vpmModule  # noqa: F401
