"""Schwarz screening interface on the CPU: primitive pair screening and argument checks of
``gbasis_b200.schwarz_screening`` (no device call), and the oracle's bounds pinned to the
reference's own ``SchwarzScreener`` bounds (``schwarz.npz``, written from gbasis by
``tests/golden/make_schwarz_golden.py``)."""
import numpy as np
import pytest

from conftest import load_npz, shells_from_json
from gbasis_b200 import schwarz_screening as sz
from gbasis_b200.contractions import GeneralizedContractionShell
from oracle import eri_oracle as orc


def _fixture():
    z = load_npz("schwarz.npz")
    return z, shells_from_json(z["shells"])


def test_shell_pair_significant_matches_reference():
    # gbasis/integrals/_schwarz_screening.py:93-128
    z, shells = _fixture()
    for t in z["thresholds"]:
        got = [sz.shell_pair_significant(shells[i], shells[j], t) for i, j in z["pairs"]]
        np.testing.assert_array_equal(got, z[f"pair_{t:g}"])


def test_shell_pair_significant_cases():
    # the cases of gbasis tests/test_schwarz_screening.py:79-118
    def s(c, e):
        return GeneralizedContractionShell(0, np.array(c, dtype=float), np.array([1.0]),
                                           np.array([e]), "cartesian")
    assert sz.shell_pair_significant(s([0, 0, 0], 1.0), s([0, 0, 0], 1.0))
    assert sz.shell_pair_significant(s([0, 0, 0], 1.0), s([1, 0, 0], 1.0))
    assert not sz.shell_pair_significant(s([0, 0, 0], 10.0), s([50, 0, 0], 10.0))
    assert sz.shell_pair_significant(s([0, 0, 0], 0.01), s([5, 0, 0], 0.01))
    a, b = s([0, 0, 0], 1.0), s([3, 0, 0], 1.0)  # decay exp(-4.5) = 1.1e-2
    assert sz.shell_pair_significant(a, b, threshold=1e-3)
    assert not sz.shell_pair_significant(a, b, threshold=0.1)


def test_oracle_bounds_match_reference():
    z, shells = _fixture()
    np.testing.assert_allclose(orc.schwarz_bounds(shells), z["bounds"], rtol=1e-10, atol=1e-14)


def test_argument_checks():
    with pytest.raises(TypeError):
        sz.compute_schwarz_bounds("not a list")
    with pytest.raises(ValueError):
        sz.compute_schwarz_bounds([])
    with pytest.raises(TypeError):
        sz.SchwarzScreener([object()])


def test_improved_contraction_screening_hook_without_device():
    # gbasis/integrals/electron_repulsion.py:340-360: a rejected quartet is zeros of the
    # block's shape, (M1, L1, M2, L2, M3, L3, M4, L4); nothing reaches the device
    from gbasis_b200.electron_repulsion import ElectronRepulsionIntegralImproved as Imp
    z, shells = _fixture()

    class Reject:
        calls = []

        def is_significant(self, i, j, k, l_shell):
            self.calls.append((i, j, k, l_shell))
            return False
    scr = Reject()
    index_map = {id(s): i for i, s in enumerate(shells)}
    blk = Imp.construct_array_contraction(shells[2], shells[3], shells[1], shells[0],
                                          screener=scr, contraction_index_map=index_map)
    m = [np.asarray(s.coeffs).shape[1] for s in shells]
    assert blk.shape == (m[2], 6, m[3], 10, m[1], 3, m[0], 1)
    assert not blk.any()
    assert scr.calls == [(2, 3, 1, 0)]
    with pytest.raises(TypeError):
        Imp.construct_array_contraction(None, shells[0], shells[0], shells[0], screener=scr,
                                        contraction_index_map=index_map)


def test_whole_array_screener_counts_match_reference():
    # the whole-array methods with the reference's hook count as the reference's loop over
    # unique shell quartets (base_four_symm.py:189-191) counts: the reference's own screener
    # statistics on the fixture's bounds, and a brute-force loop on random bounds
    from gbasis_b200.electron_repulsion import ElectronRepulsionIntegralImproved as Imp
    z, shells = _fixture()
    index_map = {id(s): i for i, s in enumerate(shells)}

    class Stub:
        def __init__(self, bounds, t):
            self.bounds, self.threshold = bounds, t
            self.n_screened = self.n_computed = 0
    obj = Imp(shells)
    for t in z["thresholds"]:
        st = Stub(z["bounds"], t)
        assert obj._screen_from({"screener": st, "contraction_index_map": index_map}) == t
        np.testing.assert_array_equal([st.n_screened, st.n_computed], z[f"stats_{t:g}"])
    rng = np.random.default_rng(7)
    n = 9
    q = rng.lognormal(-3.0, 3.0, size=(n, n))
    q = np.triu(q) + np.triu(q, 1).T
    pairs = [(i, j) for i in range(n) for j in range(i, n)]
    s0 = shells[0]
    many = [type(s0)(s0.angmom, s0.coord + i, s0.coeffs, s0.exps, s0.coord_type)
            for i in range(n)]
    objn = Imp(many)
    many_map = {id(s): i for i, s in enumerate(many)}
    for t in (1e-10, 1e-6, 1e-3, 0.0):
        brute = sum(q[i, j] * q[k, l] >= t for p, (i, j) in enumerate(pairs)
                    for (k, l) in pairs[p:])
        st = Stub(q, t)
        objn._screen_from({"screener": st, "contraction_index_map": many_map})
        assert st.n_computed == brute
        assert st.n_screened == len(pairs) * (len(pairs) + 1) // 2 - brute
    with pytest.raises(NotImplementedError):
        obj._screen_from({"screener": Stub(z["bounds"], 1e-3),
                          "contraction_index_map": {id(s): len(shells) - 1 - i
                                                    for i, s in enumerate(shells)}})
    with pytest.raises(TypeError):
        obj._screen_from({"bad_keyword": 3})
