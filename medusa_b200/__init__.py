"""medusa_b200: the MEDUSA/Fornax hydrodynamic sweep as B200-native CUDA behind a C ABI.

- ``medusa_b200.problems``: problem setups (the reference's problems/init_*.c hooks).
- ``medusa_b200.solver``: the reference-shaped host interface (estimate_dt, step,
  update_cpu) over libmedusa_b200.so.
- ``medusa_b200.eos_table``: the tabulated nuclear EOS zone update on the device
  (eos_given_rex_per_zone) and a synthetic table in the reference's layout.
- ``medusa_b200.build``: in-tree nvcc build of libmedusa_b200.so for sm_100a.
"""
from . import problems  # noqa: F401
from .solver import Solver, Server, MdgError, PREC_FP64, PREC_MIXED, library  # noqa: F401

__all__ = ["problems", "Solver", "Server", "MdgError", "PREC_FP64", "PREC_MIXED", "library"]
