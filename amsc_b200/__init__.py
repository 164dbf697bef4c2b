"""dampm-b200: the depth-averaged MPM time step of dampm (lucadiprofio/AMSC)
as hand-written sm_100a CUDA behind a C ABI (include/dampm_cuda.h)."""
from .data import DATA, from_json, to_json  # noqa: F401

__all__ = ["DATA", "from_json", "to_json"]
