"""Shared test helpers: fixture loading and shell reconstruction."""
import json
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)
GOLDEN = os.path.join(ROOT, "tests", "golden")

from gbasis_b200.contractions import GeneralizedContractionShell  # noqa: E402


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built engine")


class OrderedShell(GeneralizedContractionShell):
    """Shell with explicit Cartesian / spherical component orders (e.g. HORTON's)."""

    def __init__(self, *args, cart_order=None, sph_order=None, **kw):
        self._cart_order = None if cart_order is None else np.asarray(cart_order)
        self._sph_order = None if sph_order is None else tuple(sph_order)
        super().__init__(*args, **kw)

    @property
    def angmom_components_cart(self):
        if self._cart_order is not None:
            return self._cart_order
        return super().angmom_components_cart

    @property
    def angmom_components_sph(self):
        if self._sph_order is not None:
            return self._sph_order
        return super().angmom_components_sph


def shell_from_record(rec):
    coeffs = np.asarray(rec["coeffs"], dtype=float)
    args = (int(rec["angmom"]), np.asarray(rec["coord"], dtype=float), coeffs,
            np.asarray(rec["exps"], dtype=float), rec["coord_type"])
    if "cart_order" in rec or "sph_order" in rec:
        return OrderedShell(*args, cart_order=rec.get("cart_order"), sph_order=rec.get("sph_order"))
    return GeneralizedContractionShell(*args)


def load_npz(name):
    return np.load(os.path.join(GOLDEN, name), allow_pickle=False)


def shells_from_json(s):
    return [shell_from_record(r) for r in json.loads(str(s))]


def unique_index(n):
    return np.array([(i, j, k, l) for i in range(n) for j in range(i + 1)
                     for k in range(n) for l in range(k + 1)
                     if i * (i + 1) // 2 + j >= k * (k + 1) // 2 + l], dtype=np.int64)


def expand_unique(n, values):
    """Rebuild the full 8-fold symmetric array from its unique elements."""
    idx = unique_index(n)
    out = np.zeros((n, n, n, n))
    i, j, k, l = idx.T
    for (a, b, c, d) in [(i, j, k, l), (j, i, k, l), (i, j, l, k), (j, i, l, k),
                         (k, l, i, j), (l, k, i, j), (k, l, j, i), (l, k, j, i)]:
        out[a, b, c, d] = values
    return out


@pytest.fixture(scope="session")
def golden():
    return load_npz


def horton_overflow_case():
    """Shells, component indices and values of the large-exponent (ss|ff) known answer
    (``horton_overflow.json``, from gbasis ``tests/test_two_elec_int.py``)."""
    rec = json.load(open(os.path.join(GOLDEN, "horton_overflow.json")))
    shells, idx = [], []
    for s in rec["shells"]:
        g = GeneralizedContractionShell(int(s["angmom"]), np.array(s["coord"], dtype=float),
                                        np.array(s["coeffs"], dtype=float),
                                        np.array(s["exps"], dtype=float), "cartesian")
        comps = [tuple(int(v) for v in row) for row in g.angmom_components_cart]
        idx.append(comps.index(tuple(s["components"][0])))
        shells.append(g)
    return shells, idx, rec
