"""Base class of four-index arrays with the eight-fold symmetry of the two-electron integrals,
mirroring ``gbasis.base_four_symm``.

``BaseFourIndexSymmetric`` takes one shell list for all four axes (``gbasis/base_four_symm.py:
70-93``: constructor and ``contractions`` property).  The reference evaluates its whole arrays
with host loops over ``construct_array_contraction``; here the only four-index array is the
electron-repulsion tensor, whose class evaluates them on the device, so the array methods stay
abstract.

``register_with_gbasis`` makes the engine's classes virtual subclasses of gbasis's own base
classes when gbasis can be imported, so that code checking
``isinstance(obj, gbasis.base.BaseGaussianRelatedArray)`` or ``BaseFourIndexSymmetric`` accepts
the engine's objects; nothing of gbasis runs.
"""
from __future__ import annotations

from .base import BaseGaussianRelatedArray

__all__ = ["BaseFourIndexSymmetric", "register_with_gbasis"]


class BaseFourIndexSymmetric(BaseGaussianRelatedArray):
    """Four-index array over one list of shells, symmetric under (ab|cd) = (ba|cd) = (cd|ab)."""

    def __init__(self, contractions):
        super().__init__(contractions)

    @property
    def contractions(self):
        """The shells of all four axes (a tuple)."""
        return self._axes_contractions[0]


def register_with_gbasis(*classes):
    """Register ``classes`` as virtual subclasses of ``gbasis.base_four_symm.
    BaseFourIndexSymmetric`` (and so of ``gbasis.base.BaseGaussianRelatedArray``) when gbasis is
    importable; returns whether it was."""
    try:
        from gbasis.base_four_symm import BaseFourIndexSymmetric as _Reference
    except Exception:  # gbasis absent (or without that module): nothing to register with
        return False
    for c in classes:
        _Reference.register(c)
    return True
