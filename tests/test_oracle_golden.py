"""Pin the CPU oracle against vectors produced by the gbasis reference itself.

The fixtures in ``tests/golden`` were written by ``tests/golden/make_golden.py`` from the
reference (HORTON-derived scalars from its test suite, its stored HORTON tensor and its own
outputs).  Tolerances: the reference's own noise floor is ~1e-15 absolute; the bar is
1e-12 absolute unless stated.
"""
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN, expand_unique, load_npz, shells_from_json
from gbasis_b200.contractions import GeneralizedContractionShell
from oracle import eri_oracle as orc

ATOL = 1e-12


def test_boys_matches_reference():
    z = load_npz("boys.npz")
    F = orc.boys(z["m"][:, None], z["T"][None, :])
    np.testing.assert_allclose(F, z["F"], rtol=1e-14, atol=0)


def test_norm_cont_matches_reference():
    z = load_npz("norm_cont.npz")
    shells = shells_from_json(z["shells"])
    vals = np.split(z["values"], np.cumsum(z["sizes"])[:-1])
    for s, v in zip(shells, vals):
        np.testing.assert_allclose(np.asarray(s.norm_cont).ravel(), v, rtol=1e-13)
        np.testing.assert_allclose(orc.norm_cont(s.angmom, s.exps, s.coeffs).ravel(), v, rtol=1e-13)


def test_horton_scalars():
    """HORTON-derived primitive ERIs from gbasis tests/test_two_elec_int.py:1111-1365."""
    recs = json.load(open(os.path.join(GOLDEN, "horton_scalars.json")))
    assert len(recs) >= 50
    coords = [np.array(c) for c in ((0.2, 0.4, 0.6), (1.0, 1.5, 2.0), (0.1, 0.3, 0.5), (1.1, 1.6, 2.1))]
    for rec in recs:
        args = rec["args"]
        comps = [tuple(args[3 * n: 3 * n + 3]) for n in range(4)]
        assert args[12] == 0
        kw = rec.get("kwargs", {})
        exps = list(args[13:17]) + [0.1, 0.2, 0.3, 0.4][len(args[13:17]):]
        for n, name in enumerate(("alpha", "beta", "gamma", "delta")):
            exps[n] = kw.get(name, exps[n])
        cents = [np.array(kw.get(name, c), dtype=float)
                 for name, c in zip(("coord_a", "coord_b", "coord_c", "coord_d"), coords)]
        shells = []
        for comp, e, c in zip(comps, exps, cents):
            shells.append(GeneralizedContractionShell(int(sum(comp)), c.copy(), np.array([1.0]),
                                                      np.array([float(e)]), "cartesian"))
        blk = orc.quartet_cartesian(*shells)
        idx = []
        for comp, s in zip(comps, shells):
            cc = [tuple(int(v) for v in row) for row in s.angmom_components_cart]
            idx.append(cc.index(comp))
        val = blk[idx[0], idx[1], idx[2], idx[3], 0, 0, 0, 0]
        np.testing.assert_allclose(val, rec["expected"], rtol=1e-9, atol=1e-14)


def test_quartet_blocks_all_classes():
    """Every class with l <= 3.  Both gbasis paths lose digits on some diffuse high-l
    quartets (up to ~1e-6 absolute against 40-digit values), so the bar is
    1e-12 absolute or four times the reference's own error against the 40-digit value,
    whichever is larger."""
    z = load_npz("quartets.npz")
    recs = json.loads(str(z["shells"]))
    split = np.cumsum(z["sizes"])[:-1]
    blocks, truth, improved = (np.split(z[k], split) for k in ("blocks", "truth", "improved"))
    assert len(recs) == len(blocks) >= 50
    from conftest import shell_from_record
    for rq, ref, tru, imp in zip(recs, blocks, truth, improved):
        sh = [shell_from_record(r) for r in rq]
        plain = orc.construct_array_contraction(*sh).ravel()
        tol = max(ATOL, 4 * float(np.max(np.abs(ref - tru))))
        assert np.max(np.abs(plain - ref)) <= tol, [s.angmom for s in sh]
        reord = orc.construct_array_contraction(*sh, reorder=True).ravel()
        tol = max(ATOL, 4 * float(np.max(np.abs(imp - tru))))
        assert np.max(np.abs(reord - tru)) <= tol, [s.angmom for s in sh]
        assert np.max(np.abs(reord - imp)) <= 2 * tol, [s.angmom for s in sh]
        # the engine's recursion order (tighter shell first, bra by angular momentum) is
        # accurate to 1e-12 against the 40-digit values on every fixture quartet
        expo = orc.construct_array_contraction(*sh, reorder="exponent").ravel()
        assert np.max(np.abs(expo - tru)) <= ATOL, [s.angmom for s in sh]


def test_horton_bec_sto6g():
    z = load_npz("horton_bec_sto6g.npz")
    shells = shells_from_json(z["shells"])
    got = orc.electron_repulsion_integral(shells)
    np.testing.assert_allclose(got, z["reference"], rtol=0, atol=ATOL)
    np.testing.assert_allclose(got, z["horton"], rtol=1e-10, atol=1e-15)


def test_tiny4_full_tensor():
    z = load_npz("tiny4.npz")
    shells = shells_from_json(z["shells"])
    got = orc.electron_repulsion_integral(shells, notation="chemist")
    idx = z["index"].astype(int)
    np.testing.assert_allclose(got[idx[:, 0], idx[:, 1], idx[:, 2], idx[:, 3]], z["values"],
                               rtol=0, atol=ATOL)
    full = expand_unique(got.shape[0], z["values"])
    np.testing.assert_allclose(got, full, rtol=0, atol=ATOL)


@pytest.mark.parametrize("kind", ["cart", "sph", "mix", "lincomb", "screened"])
def test_mixed_basis(kind):
    z = load_npz("mixed.npz")
    shells = shells_from_json(z["shells"])
    cts = [s.coord_type for s in shells]
    for reorder in (False, True):
        if kind == "cart":
            got = orc.construct_array(shells, ["cartesian"] * len(shells), reorder=reorder)
        elif kind == "sph":
            got = orc.construct_array(shells, ["spherical"] * len(shells), reorder=reorder)
        elif kind == "mix":
            got = orc.construct_array(shells, cts, reorder=reorder)
        elif kind == "lincomb":
            got = orc.electron_repulsion_integral(shells, transform=z["transform"],
                                                  notation="chemist", reorder=reorder)
        else:
            got = orc.electron_repulsion_integral_screened(shells, 1e-3, notation="chemist",
                                                           reorder=reorder)
        n = int(z[kind + "_n"])
        assert got.shape == (n,) * 4
        ref = expand_unique(n, z[kind])
        truth = expand_unique(n, z[kind + "_truth"])
        ref_err = float(np.max(np.abs(ref - truth)))
        # Both paths agree with the reference to within its own rounding noise (its
        # distance from the 40-digit values); the reordered one (recursions from the
        # higher-l centres) is also that close to the 40-digit values.
        assert np.max(np.abs(got - ref)) <= max(ATOL, 8 * ref_err)
        if reorder:
            assert np.max(np.abs(got - truth)) <= max(ATOL, 4 * ref_err)


def test_horton_large_exponent_quartet():
    """gbasis tests/test_two_elec_int.py ``test_compute_two_elec_integrals_overflow_horton``
    (xfail in the reference): an (ss|ff) quartet of tightly contracted, alternating-sign s
    shells.  The reference's double path, which transfers angular momentum from the s pair,
    misses HORTON's value entirely; the 40-digit evaluator reproduces it, and so does the
    oracle in the recursion order of the engine (the f pair as the bra, no transfer)."""
    from conftest import horton_overflow_case
    shells, i, rec = horton_overflow_case()
    truth, horton = rec["truth_40_digits"], rec["horton"]
    # HORTON's value to the reference test's own tolerance (np.allclose defaults)
    assert np.allclose(truth, horton)
    assert abs(rec["reference_double"] - horton) > 1e-3  # the reference's known failure
    blk = orc.construct_array_contraction(*shells, reorder="exponent")
    got = blk[0, i[0], 0, i[1], 0, i[2], 0, i[3]]
    assert abs(got - truth) <= ATOL
    # the same integral with the pairs exchanged, (ff|ss)
    blk = orc.construct_array_contraction(shells[2], shells[3], shells[0], shells[1],
                                          reorder="exponent")
    assert abs(blk[0, i[2], 0, i[3], 0, i[0], 0, i[1]] - truth) <= ATOL


def test_heavily_contracted_quartet_pins_the_primitive_wise_checker():
    """A (dd|dd) quartet of the batch workload with d shells of 4-6 primitives spanning tight
    and diffuse exponents (``heavy_contraction.npz``, written from gbasis itself and from
    40-digit arithmetic).  The reference's own block misses the 40-digit values by about 5e-10,
    and the oracle in the reference's order by the same order of magnitude (the two differ by
    rounding, which this quartet amplifies a millionfold); the primitive-by-primitive form,
    the checker of the GPU test on such quartets, matches the 40-digit values."""
    from gbasis_b200.synthetic import batch_molecule
    z = load_npz("heavy_contraction.npz")
    shells = [batch_molecule(int(z["molecule"]))[int(i)] for i in z["quartet"]]
    ref, truth = z["reference"], z["truth_40_digits"]
    assert 1e-11 < float(np.abs(ref - truth).max()) < 1e-8
    plain = orc.construct_array_contraction(*shells)
    assert 1e-11 < float(np.abs(plain - truth).max()) < 1e-8
    by_prim = orc.construct_array_contraction_by_primitive(*shells)
    np.testing.assert_allclose(by_prim, truth, rtol=0, atol=1e-15)
