"""``gbasis.integrals.nuclear_electron_attraction`` (``nuclear_electron_attraction.py:6-42``) on
the engine."""
from ..point_charge import nuclear_electron_attraction_integral  # noqa: F401

__all__ = ["nuclear_electron_attraction_integral"]
