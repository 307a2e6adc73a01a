"""GPU tests of the point-charge kernel (through the C ABI) against the reference's outputs
(golden fixtures) and the CPU oracle, at the FP64 bar of 1e-12 relative to the largest value."""
import numpy as np
import pytest

from conftest import load_npz, shells_from_json
from gbasis_b200 import point_charge as pc
from gbasis_b200.synthetic import batch_molecule
from oracle import point_charge_oracle as pco

pytestmark = pytest.mark.gpu
G = load_npz("point_charge.npz")


def _close(got, ref):
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-12 * max(1.0, np.abs(ref).max()))


def test_point_charges_match_reference():
    for name, key in (("mixed.npz", "mixed"), ("tiny4.npz", "tiny4")):
        basis = shells_from_json(load_npz(name)["shells"])
        _close(pc.point_charge_integral(basis, G[f"{key}_coords"], G[f"{key}_charges"]),
               G[f"{key}_pc"])


def test_lincomb_and_nuclear_attraction_match_reference():
    basis = shells_from_json(load_npz("mixed.npz")["shells"])
    c, q = G["mixed_coords"], G["mixed_charges"]
    _close(pc.point_charge_integral(basis, c, q, transform=load_npz("mixed.npz")["transform"]),
           G["mixed_pc_lincomb"])
    _close(pc.nuclear_electron_attraction_integral(basis, c, q), G["mixed_nuc"])


@pytest.mark.parametrize("m", [2, 8, 15])
def test_molecules_against_oracle(m):
    """Batch molecules (s to d shells, contracted) with their nuclei as the point charges."""
    basis = batch_molecule(m)
    coords = np.unique(np.array([s.coord for s in basis]), axis=0)
    charges = np.arange(1, coords.shape[0] + 1, dtype=float)
    ref = pco.point_charge_integral(basis, coords, charges)
    _close(pc.point_charge_integral(basis, coords, charges), ref)
    _close(pc.nuclear_electron_attraction_integral(basis, coords, charges), ref.sum(axis=2))


def test_rejects_bad_points():
    basis = shells_from_json(load_npz("tiny4.npz")["shells"])
    with pytest.raises(TypeError):
        pc.point_charge_integral(basis, np.zeros((2, 2)), np.ones(2))
    with pytest.raises(TypeError):
        pc.point_charge_integral(basis, np.zeros((2, 3)), np.ones((2, 1)))
    with pytest.raises(ValueError):
        pc.point_charge_integral(basis, np.zeros((2, 3)), np.ones(3))
    with pytest.raises(ValueError):
        pc.point_charge_integral(basis, np.array([[0.0, 0.0, np.nan]]), np.ones(1))
