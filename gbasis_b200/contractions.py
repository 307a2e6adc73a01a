"""Host-side shell data model: a drop-in for ``gbasis.contractions.GeneralizedContractionShell``.

The engine only reads shells; it never needs gbasis to be importable.  Shells built by
gbasis itself (or a subclass such as one with a HORTON component order) are accepted
everywhere this class is: :func:`is_shell` checks the class hierarchy by name.

Reference: ``gbasis/contractions.py:8-572`` (validation in the property setters,
component orders at ``:379-385`` / ``:426-432``, ``norm_cont`` at ``:503-524``).
"""
from __future__ import annotations

from numbers import Integral

import numpy as np

__all__ = ["GeneralizedContractionShell", "is_shell", "default_cart_components",
           "default_sph_components"]


def default_cart_components(l):
    """Cartesian order ``for x in l..0: for y in l-x..0: (x, y, l-x-y)`` (``contractions.py:379-385``)."""
    return np.array([(x, y, l - x - y) for x in range(l, -1, -1) for y in range(l - x, -1, -1)])


def default_sph_components(l):
    """Spherical order: l=1 -> (c1, s1, c0); else s_l..s_1, c_0..c_l (``contractions.py:426-432``)."""
    if l == 1:
        return ("c1", "s1", "c0")
    return tuple([f"s{m}" for m in range(l, 0, -1)] + [f"c{m}" for m in range(l + 1)])


def _double_factorial(n):
    r = 1.0
    while n > 1:
        r *= n
        n -= 2
    return r


def is_shell(obj) -> bool:
    """True for this class, gbasis's ``GeneralizedContractionShell`` and their subclasses."""
    for klass in type(obj).__mro__:
        if klass.__name__ == "GeneralizedContractionShell":
            return True
    return False


class GeneralizedContractionShell:
    """Contracted Cartesian Gaussians sharing centre, angular momentum and exponents.

    Same constructor, attributes and errors as gbasis
    (``GeneralizedContractionShell(angmom, coord, coeffs, exps, coord_type, icenter=None)``).
    """

    def __init__(self, angmom, coord, coeffs, exps, coord_type, icenter=None):
        self.angmom = angmom
        self.coord = coord
        self.coeffs = coeffs
        self.exps = exps
        self.assign_norm_cont()
        self.coord_type = coord_type
        self.icenter = icenter

    # ----------------------------------------------------------------- properties
    @property
    def icenter(self):
        return self._icenter

    @icenter.setter
    def icenter(self, icenter):
        if isinstance(icenter, Integral):
            self._icenter = int(icenter)
        elif icenter is None:
            self._icenter = None
        else:
            raise TypeError(f"Center should be of `numbers.Integral` type. Got {type(icenter)}")

    @property
    def coord(self):
        return self._coord

    @coord.setter
    def coord(self, coord):
        if not (isinstance(coord, np.ndarray) and coord.size == 3):
            raise TypeError("Coordinate must be given as a `numpy` array of dimension 3.")
        if coord.dtype == int:
            coord = coord.astype(float)
        if coord.dtype != float:
            raise TypeError("The data type of the coordinate must be int or float.")
        self._coord = coord

    @property
    def angmom(self):
        return self._angmom

    @angmom.setter
    def angmom(self, angmom):
        if not isinstance(angmom, int):
            raise TypeError("Angular momentum must be given as an integer")
        if angmom < 0:
            raise ValueError("Angular momentum must be a positive integer.")
        self._angmom = angmom

    @property
    def exps(self):
        return self._exps

    @exps.setter
    def exps(self, exps):
        if not (isinstance(exps, np.ndarray) and exps.dtype == float):
            raise TypeError("Exponents must be given as a `numpy` array of data type float.")
        if hasattr(self, "_coeffs") and self.coeffs.shape[0] != exps.size:
            raise ValueError(
                "Exponents array must have the same number of elements as the number of rows "
                "in the two-dimensional coefficient matrix (for the generalized contractions)."
            )
        self._exps = exps

    @property
    def coeffs(self):
        return self._coeffs

    @coeffs.setter
    def coeffs(self, coeffs):
        if not (isinstance(coeffs, np.ndarray) and coeffs.dtype == float):
            raise TypeError("Contraction coefficients must be a `numpy` array of data type float.")
        if coeffs.ndim not in [1, 2]:
            raise ValueError("Coefficients array must be given as a one- or two-dimensional array.")
        if hasattr(self, "_exps"):
            if coeffs.ndim == 2 and coeffs.shape[0] != self.exps.shape[0]:
                raise ValueError(
                    "Coefficients array for generalized contractions must be given as a two-"
                    "dimensional array with the same number of rows as the size of the exponents "
                    "array."
                )
            if coeffs.ndim == 1 and coeffs.shape != self.exps.shape:
                raise ValueError(
                    "Coefficients array for segmented contractions must be given as a one-"
                    "dimensional array with the same size as the exponents array."
                )
        self._coeffs = coeffs[:, np.newaxis] if coeffs.ndim == 1 else coeffs

    @property
    def angmom_components_cart(self):
        return default_cart_components(self.angmom)

    @property
    def angmom_components_sph(self):
        return default_sph_components(self.angmom)

    @property
    def norm_prim_cart(self):
        """(L, K) primitive normalisation (``contractions.py:434-461``)."""
        comps = self.angmom_components_cart
        df = np.array([np.prod([_double_factorial(2 * int(v) - 1) for v in c]) for c in comps])
        e = self.exps
        return (2 * e / np.pi) ** 0.75 * (4 * e) ** (self.angmom / 2) / np.sqrt(df)[:, None]

    @property
    def num_cart(self):
        return (self.angmom + 1) * (self.angmom + 2) // 2

    @property
    def num_sph(self):
        return 1 + 2 * self.angmom

    @property
    def num_seg_cont(self):
        return self.coeffs.shape[1]

    def assign_norm_cont(self):
        """norm_cont (M, L_cart) = (self overlap)^-1/2.

        The one-centre overlap of two normalised Cartesian primitives of the same
        component is (2a/pi)^{3/4}(4a)^{l/2}(2b/pi)^{3/4}(4b)^{l/2} (pi/s)^{3/2}/(2s)^l with
        s = a + b (the (2a_i-1)!! factors cancel), so every component of a segmented
        contraction gets the same constant.  Same quantity as ``contractions.py:503-524``.
        """
        e = self.exps
        l = self.angmom
        radial = (2 * e / np.pi) ** 0.75 * (4 * e) ** (l / 2.0)
        s = e[:, None] + e[None, :]
        kern = (np.pi / s) ** 1.5 / (2 * s) ** l
        c = self.coeffs * radial[:, None]
        ov = np.einsum("km,kq,qm->m", c, kern, c)
        self.norm_cont = np.repeat((ov ** -0.5)[:, None], self.num_cart, axis=1)

    @property
    def coord_type(self):
        return self._coord_type

    @coord_type.setter
    def coord_type(self, coord_type):
        if not isinstance(coord_type, str):
            raise TypeError("Coordinate type must be given as a string.")
        if coord_type not in ["c", "cartesian", "p", "spherical"]:
            raise ValueError(
                "`coord_type` is incorrectly specified. It must be either 'c' "
                "or 'cartesian' for Cartesian coordinates, or 'p' or 'spherical' "
                "for spherical coordinates."
            )
        self._coord_type = {"c": "cartesian", "cartesian": "cartesian",
                            "spherical": "spherical", "p": "spherical"}[coord_type]
