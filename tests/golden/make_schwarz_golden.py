"""Regenerate ``schwarz.npz`` (this folder) from the gbasis reference itself.

    python tests/golden/make_schwarz_golden.py --reference /path/to/gbasis

Imports gbasis from ``--reference`` and, on the shells of ``mixed.npz`` plus two copies of its
first shell moved 3.5 and 30 bohr away (so that quartets fall below the thresholds), records:

* ``bounds``: ``SchwarzScreener(...).bounds`` built as ``electron_repulsion_integral_improved``
  builds it (``get_boys_function("coulomb")``, ``compute_two_electron_integrals_os_hgp``);
* ``stats_<t>``: ``n_screened``, ``n_computed`` of that screener after ``is_significant`` over
  every shell quartet (i <= j, k <= l, ij <= kl) at threshold ``t``;
* ``pair_<t>``: ``shell_pair_significant`` of every shell pair at threshold ``t``.

The tests only read the written file; they never import gbasis.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
THRESHOLDS = (1e-12, 1e-6, 1e-3)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="path of a gbasis source checkout")
    a = ap.parse_args()
    sys.path.insert(0, a.reference)
    from gbasis.contractions import GeneralizedContractionShell as RefShell
    from gbasis.integrals._schwarz_screening import SchwarzScreener, shell_pair_significant
    from gbasis.integrals._two_elec_int_improved import compute_two_electron_integrals_os_hgp
    from gbasis.integrals.boys_functions import get_boys_function

    z = np.load(os.path.join(HERE, "mixed.npz"), allow_pickle=False)
    recs = json.loads(str(z["shells"]))
    for shift in (3.5, 30.0):
        far = dict(recs[0])
        far["coord"] = (np.array(recs[0]["coord"]) + np.array([shift, 0.0, 0.0])).tolist()
        recs = recs + [far]
    basis = [RefShell(r["angmom"], np.array(r["coord"]), np.array(r["coeffs"]),
                      np.array(r["exps"]), r["coord_type"]) for r in recs]
    n = len(basis)
    pairs = [(i, j) for i in range(n) for j in range(i, n)]
    out = {"shells": json.dumps(recs), "thresholds": np.array(THRESHOLDS)}
    for t in THRESHOLDS:
        scr = SchwarzScreener(basis, get_boys_function("coulomb"),
                              compute_two_electron_integrals_os_hgp, t)
        out["bounds"] = scr.bounds
        for pi, (i, j) in enumerate(pairs):
            for (k, l) in pairs[:pi + 1]:
                scr.is_significant(i, j, k, l)
        out[f"stats_{t:g}"] = np.array([scr.n_screened, scr.n_computed])
        out[f"pair_{t:g}"] = np.array([shell_pair_significant(basis[i], basis[j], t)
                                       for i, j in pairs])
    out["pairs"] = np.array(pairs)
    np.savez_compressed(os.path.join(HERE, "schwarz.npz"), **out)
    print({k: (v if np.ndim(v) <= 1 and np.size(v) < 20 else np.shape(v)) for k, v in out.items()
           if k != "shells"})


if __name__ == "__main__":
    main()
