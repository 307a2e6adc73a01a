"""Schwarz bounds and screener of ``gbasis_b200.schwarz_screening`` on the GPU against the
reference's own ``SchwarzScreener`` (``schwarz.npz``: the shells of ``mixed.npz``, with a
generalized d shell and an f shell, plus copies of the first shell 3.5 and 30 bohr away) and
against the oracle."""
import numpy as np
import pytest

from conftest import load_npz, shells_from_json
from gbasis_b200 import schwarz_screening as sz
from oracle import eri_oracle as orc

pytestmark = pytest.mark.gpu


def test_bounds_match_reference_and_oracle():
    z = load_npz("schwarz.npz")
    shells = shells_from_json(z["shells"])
    q = sz.compute_schwarz_bounds(shells)
    assert q.shape == (len(shells),) * 2
    np.testing.assert_array_equal(q, q.T)
    np.testing.assert_allclose(q, z["bounds"], rtol=1e-10, atol=1e-14)
    # the FP64 form's bar, 1e-12 absolute (measured: at most 1.3e-13 from the oracle)
    np.testing.assert_allclose(q, orc.schwarz_bounds(shells), rtol=1e-12, atol=1e-12)
    assert sz.compute_schwarz_bound_shell_pair(None, shells[1], shells[2]) == \
        pytest.approx(q[1, 2], rel=1e-12)


def test_screener_counts_match_reference():
    z = load_npz("schwarz.npz")
    shells = shells_from_json(z["shells"])
    pairs = [tuple(p) for p in z["pairs"]]
    for t in z["thresholds"]:
        scr = sz.SchwarzScreener(shells, None, None, t)
        for pi, (i, j) in enumerate(pairs):
            for (k, l) in pairs[:pi + 1]:
                scr.is_significant(i, j, k, l)
        np.testing.assert_array_equal([scr.n_screened, scr.n_computed], z[f"stats_{t:g}"])
        st = scr.get_statistics()
        assert st["total"] == len(pairs) * (len(pairs) + 1) // 2
        scr.reset_counters()
        assert scr.get_statistics()["total"] == 0


def test_improved_contraction_with_screener():
    """The screening hook of ``ElectronRepulsionIntegralImproved.construct_array_contraction``
    with the device screener: rejected quartets are zeros, the others equal the plain call."""
    from gbasis_b200.electron_repulsion import ElectronRepulsionIntegral
    from gbasis_b200.electron_repulsion import ElectronRepulsionIntegralImproved as Imp
    z = load_npz("schwarz.npz")
    shells = shells_from_json(z["shells"])
    scr = sz.SchwarzScreener(shells, None, None, 1e-3)
    index_map = {id(s): i for i, s in enumerate(shells)}
    q = scr.bounds
    for (i, j, k, l) in [(0, 1, 2, 3), (0, 4, 0, 5), (2, 2, 1, 0)]:
        sh = (shells[i], shells[j], shells[k], shells[l])
        blk = Imp.construct_array_contraction(*sh, screener=scr, contraction_index_map=index_map)
        if q[i, j] * q[k, l] < 1e-3:
            assert not blk.any()
        else:
            ref = ElectronRepulsionIntegral.construct_array_contraction(*sh)
            np.testing.assert_allclose(blk, ref, rtol=0, atol=1e-14)
    assert scr.get_statistics() == {"n_screened": 1, "n_computed": 2, "total": 3,
                                    "percent_screened": 100.0 / 3, "speedup_factor": 1.5}


def test_whole_array_screener_hook():
    """``construct_array_cartesian(screener=..., contraction_index_map=...)`` of the improved
    class: the same array as a Schwarz threshold equal to the screener's, and the screener's
    counts equal to those of the reference's own screener on this basis."""
    from gbasis_b200.electron_repulsion import ElectronRepulsionIntegralImproved as Imp
    z = load_npz("schwarz.npz")
    shells = shells_from_json(z["shells"])
    scr = sz.SchwarzScreener(shells, None, None, 1e-3)
    obj = Imp(shells)
    got = obj.construct_array_cartesian(screener=scr,
                                        contraction_index_map={id(s): i
                                                               for i, s in enumerate(shells)})
    assert obj._screen == 0.0
    ref = Imp(shells, 1e-3).construct_array_cartesian()
    np.testing.assert_array_equal(got, ref)
    np.testing.assert_array_equal([scr.n_screened, scr.n_computed], z["stats_0.001"])
