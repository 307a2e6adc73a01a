"""GPU tests of the range-separated operators erf(omega r)/r and erfc(omega r)/r (through the
C ABI): against the oracle (same recursion order, FP64 bar 1e-12) and against the reference's
own outputs (tolerances of tests/test_oracle_range_separated.py)."""
import numpy as np
import pytest

from conftest import load_npz, shells_from_json
from gbasis_b200 import _engine
from gbasis_b200 import electron_repulsion as er
from gbasis_b200.synthetic import make_workload
from oracle import eri_oracle as orc

pytestmark = pytest.mark.gpu
G = load_npz("range_separated.npz")
CASES = (("erf", 1, 0.4, 5e-12), ("erfc", 2, 1.7, 1e-12))


def test_mixed_basis_against_reference_and_oracle():
    basis = shells_from_json(load_npz("mixed.npz")["shells"])
    idx = G["index"]
    for kind, code, omega, tol in CASES:
        t = er.electron_repulsion_integral(basis, notation="chemist", potential=kind, omega=omega)
        ref = G[f"{kind}_{omega}"]
        got = t[idx[:, 0], idx[:, 1], idx[:, 2], idx[:, 3]]
        np.testing.assert_allclose(got, ref, rtol=0, atol=tol * max(1.0, np.abs(ref).max()))
        o = orc.electron_repulsion_integral(basis, notation="chemist", reorder="exponent",
                                            potential=(code, omega))
        np.testing.assert_allclose(t, o, rtol=0, atol=1e-12 * max(1.0, np.abs(o).max()))


def test_tiny4_erf_plus_erfc_is_coulomb_and_oracle():
    basis = make_workload("tiny4")
    c = er.electron_repulsion_integral(basis, notation="chemist")
    e = er.electron_repulsion_integral(basis, notation="chemist", potential="erf", omega=0.9)
    f = er.electron_repulsion_integral(basis, notation="chemist", potential="erfc_coulomb",
                                       omega=0.9)
    np.testing.assert_allclose(e + f, c, rtol=0, atol=1e-12)
    o = orc.electron_repulsion_integral(basis, notation="chemist", reorder="exponent",
                                        potential=(1, 0.9))
    np.testing.assert_allclose(e, o, rtol=0, atol=1e-12 * max(1.0, np.abs(o).max()))
    # the same basis afterwards at 1/r again: the operator is per call
    np.testing.assert_array_equal(er.electron_repulsion_integral(basis, notation="chemist"), c)


def test_screened_and_lincomb_forms():
    basis = shells_from_json(load_npz("mixed.npz")["shells"])
    T = load_npz("mixed.npz")["transform"]
    full = er.electron_repulsion_integral(basis, notation="chemist", potential="erfc", omega=1.7)
    lin = er.electron_repulsion_integral(basis, transform=T, notation="chemist",
                                         potential="erfc", omega=1.7)
    ref = np.einsum("ia,jb,kc,ld,abcd->ijkl", T, T, T, T, full, optimize=True)
    np.testing.assert_allclose(lin, ref, rtol=0, atol=1e-12 * max(1.0, np.abs(ref).max()))
    scr = er.electron_repulsion_integral_improved(basis, notation="chemist",
                                                  schwarz_threshold=1e-30, potential="erfc",
                                                  omega=1.7)
    np.testing.assert_allclose(scr, full, rtol=0, atol=1e-15)


def test_rejects_bad_operators():
    basis = make_workload("tiny4")
    with pytest.raises(ValueError):
        er.electron_repulsion_integral(basis, potential="erf")
    with pytest.raises(ValueError):
        er.electron_repulsion_integral(basis, potential="yukawa", omega=1.0)
    db = _engine.DeviceBasis(basis)
    try:
        with pytest.raises(ValueError):
            db.set_potential(1, 0.0)
        with pytest.raises(ValueError):
            db.set_potential(3, 1.0)
    finally:
        db.close()
