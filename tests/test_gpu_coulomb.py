"""Direct Coulomb matrix (through the C ABI) against the contraction of the full tensor."""
import numpy as np
import pytest

from conftest import load_npz, shells_from_json
from gbasis_b200 import electron_repulsion as er
from gbasis_b200.coulomb import coulomb_matrix
from gbasis_b200.synthetic import density_matrix, make_workload

pytestmark = pytest.mark.gpu


def _check(shells, thr):
    eri = er.electron_repulsion_integral(shells, notation="chemist")
    n = eri.shape[0]
    D = density_matrix(n, seed=n)
    J = coulomb_matrix(shells, D, schwarz_threshold=0.0)
    ref = np.einsum("abcd,cd->ab", eri, D)
    np.testing.assert_allclose(J, ref, rtol=0, atol=1e-12 * max(1.0, np.abs(ref).max()))
    np.testing.assert_allclose(J, J.T, rtol=0, atol=1e-13)
    if thr:
        Jt = coulomb_matrix(shells, D, schwarz_threshold=thr)
        eri_t = er.electron_repulsion_integral_improved(shells, notation="chemist",
                                                        schwarz_threshold=thr)
        np.testing.assert_allclose(Jt, np.einsum("abcd,cd->ab", eri_t, D), rtol=0,
                                   atol=1e-12 * max(1.0, np.abs(ref).max()))


def test_coulomb_tiny4():
    _check(make_workload("tiny4"), 1e-4)


def test_coulomb_mixed_with_f_shells():
    z = load_npz("mixed.npz")
    _check(shells_from_json(z["shells"]), 1e-3)


def test_coulomb_medium8():
    _check(make_workload("medium8")[:18], 1e-8)
