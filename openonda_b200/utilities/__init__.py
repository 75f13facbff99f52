"""Initial conditions and particle lattices built on the B200 (mirrors OpenONDA/utilities)."""
from . import vpm_flow_models, vpm_solver_helper  # noqa: F401
