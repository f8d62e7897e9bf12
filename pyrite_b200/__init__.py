"""pyrite_b200: PyRITE's electron-transport and radiation-scoring hot path on B200.

Hand-written sm_100a CUDA behind a C ABI (``include/pyrite_b200.h``), loaded
with ctypes; this package holds the host-side mirror of the reference's calls
and the tables they need. There is no CPU fallback.
"""

from .api import (  # noqa: F401
    BeamSpec,
    CharacteristicLines,
    LineTables,
    mc_brem_spectrum,
    mc_characteristic_spectrum,
    mc_cxr_spectrum,
    retry_step_budget,
    simulate_trajectories,
    TransportStepLimitError,
)
from ._lib import PyriteB200Error, load  # noqa: F401
from .summary import tally_tables  # noqa: F401

__all__ = [
    "BeamSpec",
    "CharacteristicLines",
    "LineTables",
    "PyriteB200Error",
    "load",
    "mc_brem_spectrum",
    "mc_characteristic_spectrum",
    "mc_cxr_spectrum",
    "retry_step_budget",
    "simulate_trajectories",
    "TransportStepLimitError",
    "tally_tables",
]
