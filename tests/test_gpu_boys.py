"""The device Boys function on its own (``gbx_boys_eval``, the ``boys_eval`` the class kernels
run) against F_m(T) = 1F1(m+1/2; m+3/2; -T) / (2m+1) evaluated to 40 digits, the definition of
gbasis/integrals/boys_functions.py:26-63.

Orders m <= 13 (the highest any class with l <= 3 needs is 12), arguments on [0, 200] with the
grid points of the Taylor table, the midpoints between them (the largest Taylor step) and a band
around T = 40, where the device switches from the table to the asymptotic form
F_0 = sqrt(pi/T)/2 with upward recursion.  Bar: 1e-14 relative (the table's Taylor remainder is
below 1e-15 relative and the recursions add a few roundings per order)."""
import numpy as np
import pytest

from gbasis_b200 import _engine

RTOL = 1e-14
M_MAX = 13


def _arguments():
    rng = np.random.default_rng(7)
    T = np.concatenate([
        np.arange(0.0, 40.0, 0.1),                    # the table's grid points
        np.arange(0.05, 40.0, 0.1),                   # midpoints: |T - T_n| = 0.05
        40.0 + np.array([-1e-9, -1e-12, 0.0, 1e-12, 1e-9, -0.05, 0.05, -0.049, 0.049]),
        rng.uniform(39.0, 41.0, 60),
        rng.uniform(0.0, 200.0, 200),
        [1e-300, 1e-12, 1e-6, 123.456, 200.0],
    ])
    return np.clip(T, 0.0, None)


def _truth(T, m_max):
    import mpmath
    mpmath.mp.dps = 40
    out = np.empty((T.size, m_max + 1))
    for i, t in enumerate(T):
        x = mpmath.mpf(float(t))
        for m in range(m_max + 1):
            a = mpmath.mpf(m) + mpmath.mpf(1) / 2
            out[i, m] = float(mpmath.hyp1f1(a, a + 1, -x) / (2 * m + 1))
    return out


@pytest.mark.gpu
def test_device_boys_against_40_digit_values():
    T = _arguments()
    ref = _truth(T, M_MAX)
    for m_max in (0, 1, 4, 8, 12, M_MAX):
        got = _engine.boys_eval(m_max, T)
        rel = np.abs(got - ref[:, : m_max + 1]) / np.abs(ref[:, : m_max + 1])
        worst = np.unravel_index(np.argmax(rel), rel.shape)
        assert rel.max() <= RTOL, (m_max, float(rel.max()), float(T[worst[0]]), int(worst[1]))


def test_boys_entry_rejects_bad_arguments_without_a_device_call():
    with pytest.raises(ValueError):
        _engine.boys_eval(3, np.array([1.0, -0.5]))
    with pytest.raises(ValueError):
        _engine.boys_eval(3, np.array([np.nan]))
    with pytest.raises(ValueError):
        _engine.boys_eval(14, np.array([1.0]))
