"""Schwarz screening of shell quartets, with the interface of gbasis's
``gbasis/integrals/_schwarz_screening.py`` and the bounds computed on the device.

Q_ij = sqrt(max |(ij|ij)|) over the (ij|ij) block with primitive and Cartesian component norms
and without ``norm_cont``: the block ``compute_schwarz_bound_shell_pair`` takes the maximum of
(``_schwarz_screening.py:14-59``).  The engine evaluates every diagonal quartet (ij|ij) with its
class kernels in one pass (the kernels' Schwarz mode writes sqrt(max |.|) per shell pair), for
a generalized contraction the largest value over its segments.  ``boys_func`` and
``compute_integral_func`` are accepted where the reference takes them and are not called: the
device path evaluates the Coulomb operator with its own Boys function and recursions, as the
reference's improved path does when it builds its screener (``electron_repulsion.py:470-479``).
"""
from __future__ import annotations

import numpy as np

from . import _engine
from .contractions import is_shell

__all__ = ["compute_schwarz_bound_shell_pair", "compute_schwarz_bounds",
           "shell_pair_significant", "SchwarzScreener"]


def _check(contractions):
    if not isinstance(contractions, (list, tuple)):
        raise TypeError("`contractions` must be a list or tuple of `GeneralizedContractionShell`.")
    if not contractions:
        raise ValueError("At least one `GeneralizedContractionShell` must be given.")
    for c in contractions:
        if not is_shell(c):
            raise TypeError("Given contractions must be instances of the "
                            "`GeneralizedContractionShell` class.")


def compute_schwarz_bounds(contractions, boys_func=None, compute_integral_func=None, device=None):
    """(n_shells, n_shells) symmetric array of Q_ij = sqrt(max |(ij|ij)|)
    (``_schwarz_screening.py:62-90``), computed on ``device`` (default: the current one)."""
    _check(contractions)
    db = _engine.DeviceBasis(list(contractions), raw=True, device=device)
    try:
        q_seg = db.schwarz_bounds()  # one row and column per segmented contraction
        group = db.packed["group"]
    finally:
        db.close()
    n = len(contractions)
    q = np.zeros((n, n))
    # max over the segments of each shell: the largest element of a generalized block
    np.maximum.at(q, (group[:, None], group[None, :]), q_seg)
    return q


def compute_schwarz_bound_shell_pair(boys_func, cont_one, cont_two, compute_integral_func=None,
                                     device=None):
    """sqrt(max |(ab|ab)|) of one shell pair (``_schwarz_screening.py:14-59``)."""
    return float(compute_schwarz_bounds([cont_one, cont_two], device=device)[0, 1])


def shell_pair_significant(cont_one, cont_two, threshold=1e-12):
    """Primitive screening of a shell pair (``_schwarz_screening.py:93-128``): True if the
    centres coincide (|A-B|^2 < 1e-10) or any primitive pair has a Gaussian-product decay
    exp(-ab/(a+b) |A-B|^2) above ``threshold``."""
    r2 = float(np.sum((np.asarray(cont_one.coord, dtype=float)
                       - np.asarray(cont_two.coord, dtype=float)) ** 2))
    if r2 < 1e-10:
        return True
    a = np.asarray(cont_one.exps, dtype=float).ravel()[:, None]
    b = np.asarray(cont_two.exps, dtype=float).ravel()[None, :]
    return bool(np.any(np.exp(-a * b / (a + b) * r2) > threshold))


class SchwarzScreener:
    """Shell-quartet screening by |(ij|kl)| <= Q_ij Q_kl (``_schwarz_screening.py:131-218``).

    ``bounds`` come from :func:`compute_schwarz_bounds`; ``is_significant`` counts screened and
    computed quartets exactly as the reference's screener does.
    """

    def __init__(self, contractions, boys_func=None, compute_integral_func=None,
                 threshold=1e-12, device=None):
        self.threshold = threshold
        self.n_screened = 0
        self.n_computed = 0
        self.bounds = compute_schwarz_bounds(contractions, boys_func, compute_integral_func,
                                             device=device)

    def is_significant(self, i, j, k, l_shell):
        if self.bounds[i, j] * self.bounds[k, l_shell] < self.threshold:
            self.n_screened += 1
            return False
        self.n_computed += 1
        return True

    def get_statistics(self):
        total = self.n_screened + self.n_computed
        return {
            "n_screened": self.n_screened,
            "n_computed": self.n_computed,
            "total": total,
            "percent_screened": 0.0 if total == 0 else 100.0 * self.n_screened / total,
            "speedup_factor": total / max(self.n_computed, 1),
        }

    def reset_counters(self):
        self.n_screened = 0
        self.n_computed = 0
