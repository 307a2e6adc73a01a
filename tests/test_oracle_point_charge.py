"""The point-charge oracle (CPU) against the reference's own outputs (golden fixtures)."""
import numpy as np

from conftest import load_npz, shells_from_json
from oracle import point_charge_oracle as pco

G = load_npz("point_charge.npz")


def _basis(name):
    return shells_from_json(load_npz(name)["shells"])


def test_oracle_matches_reference_point_charges():
    for name, key in (("mixed.npz", "mixed"), ("tiny4.npz", "tiny4")):
        got = pco.point_charge_integral(_basis(name), G[f"{key}_coords"], G[f"{key}_charges"])
        ref = G[f"{key}_pc"]
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-12 * max(1.0, np.abs(ref).max()))


def test_oracle_matches_reference_lincomb_and_nuclear_sum():
    basis = _basis("mixed.npz")
    c, q = G["mixed_coords"], G["mixed_charges"]
    T = load_npz("mixed.npz")["transform"]
    np.testing.assert_allclose(pco.point_charge_integral(basis, c, q, transform=T),
                               G["mixed_pc_lincomb"], rtol=0, atol=1e-12)
    np.testing.assert_allclose(pco.nuclear_electron_attraction_integral(basis, c, q),
                               G["mixed_nuc"], rtol=0, atol=1e-11)
