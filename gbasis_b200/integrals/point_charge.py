"""``gbasis.integrals.point_charge.point_charge_integral`` (``point_charge.py:271-325``) on the
engine."""
from ..point_charge import point_charge_integral  # noqa: F401

__all__ = ["point_charge_integral"]
