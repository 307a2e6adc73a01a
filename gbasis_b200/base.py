"""Base class of arrays built over contracted Gaussian shells, mirroring ``gbasis.base``.

``BaseGaussianRelatedArray`` keeps the reference's constructor contract
(``gbasis/base.py:32-65``): one list or tuple of shells per array axis, each non-empty and
made of ``GeneralizedContractionShell`` instances, stored as ``_axes_contractions`` (a tuple of
tuples); the same ``TypeError`` / ``ValueError`` messages for bad input.  The array methods are
abstract, as in the reference (``gbasis/base.py:67-160``); the engine's subclasses evaluate them
on the device.
"""
from __future__ import annotations

import abc

from .contractions import is_shell

__all__ = ["BaseGaussianRelatedArray", "check_shell_list"]


def check_shell_list(axis):
    """The reference's checks of one axis's shells (a non-empty list or tuple of shells)."""
    if not isinstance(axis, (list, tuple)):
        raise TypeError("Contractions must be given as a list or tuple of "
                        "`GeneralizedContractionShell` instance")
    if not axis:
        raise ValueError("At least one `GeneralizedContractionShell` must be given.")
    if not all(is_shell(c) for c in axis):
        raise TypeError("Given contractions must be instances of the "
                        "`GeneralizedContractionShell` class.")


class BaseGaussianRelatedArray(abc.ABC):
    """Array whose axes are associated with contracted Gaussian shells."""

    def __init__(self, *contractions):
        for axis in contractions:
            check_shell_list(axis)
        self._axes_contractions = tuple(tuple(axis) for axis in contractions)

    @abc.abstractmethod
    def construct_array_contraction(self, *contractions, **kwargs):
        """Block of the array for one shell per axis."""

    @abc.abstractmethod
    def construct_array_cartesian(self, **kwargs):
        """Whole array over Cartesian functions."""

    @abc.abstractmethod
    def construct_array_spherical(self, **kwargs):
        """Whole array over real solid harmonics."""

    @abc.abstractmethod
    def construct_array_mix(self, coord_types, **kwargs):
        """Whole array with each shell in its own coordinate type."""

    @abc.abstractmethod
    def construct_array_lincomb(self, *transform, coord_type, **kwargs):
        """Whole array over linear combinations of the shells' functions."""
