"""mcmax_b200 -- B200-native (sm_100a) library for the MCMax hot path:
the DHS/Mie opacity stage (ComputePart) and the photon-packet transport
(MCRadiation), behind the C-ABI of include/mcmax_gpu.h.

    from mcmax_b200 import Context, ComputePart, MCRadiation
"""
from .api import Context, McgError, ComputePart, MCRadiation, Diffuse, Particle, bb_table, planck  # noqa: F401

__all__ = ["Context", "McgError", "ComputePart", "MCRadiation", "Diffuse", "Particle", "bb_table", "planck"]
