"""Native propagator modules with the reference's function signatures
(drop-ins for torchwi.propagator.td2d_cuda, td2d_forward_cuda and
td2d_exa_cuda)."""
from . import td2d_b200, td2d_exa_b200, td2d_forward_b200  # noqa: F401
