"""``gbasis.integrals.electron_repulsion`` (``electron_repulsion.py:20-504``) on the engine."""
from ..electron_repulsion import (  # noqa: F401
    ElectronRepulsionIntegral,
    ElectronRepulsionIntegralImproved,
    electron_repulsion_integral,
    electron_repulsion_integral_improved,
)

__all__ = ["ElectronRepulsionIntegral", "ElectronRepulsionIntegralImproved",
           "electron_repulsion_integral", "electron_repulsion_integral_improved"]
