"""Regenerate ``range_separated.npz`` (this folder) from the gbasis reference itself.

    python tests/golden/make_range_separated_golden.py --reference /path/to/gbasis

Imports gbasis from ``--reference`` and evaluates ``electron_repulsion_integral_improved`` with
the class's ``boys_func`` set to ``get_boys_function("erf", 0.4)`` and ``("erfc", 1.7)`` (the reference's
way of selecting a range-separated operator, ``boys_functions.py:283-350``) on the shells of
``mixed.npz``.  Stores the unique elements of each chemist tensor.  The tests only read the
written file; they never import gbasis.
"""
from __future__ import annotations

import argparse
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="path of a gbasis source checkout")
    a = ap.parse_args()
    sys.path.insert(0, a.reference)
    from gbasis.contractions import GeneralizedContractionShell as RefShell
    from gbasis.integrals.boys_functions import get_boys_function
    from gbasis.integrals.electron_repulsion import (ElectronRepulsionIntegralImproved,
                                                     electron_repulsion_integral_improved)

    z = np.load(os.path.join(HERE, "mixed.npz"), allow_pickle=False)
    recs = json.loads(str(z["shells"]))
    basis = [RefShell(r["angmom"], np.array(r["coord"]), np.array(r["coeffs"]),
                      np.array(r["exps"]), r["coord_type"]) for r in recs]
    out = {}
    saved = ElectronRepulsionIntegralImproved.boys_func
    try:
        for kind, omega in (("erf", 0.4), ("erfc", 1.7)):
            ElectronRepulsionIntegralImproved.boys_func = get_boys_function(kind, omega=omega)
            t = electron_repulsion_integral_improved(basis, notation="chemist")
            n = t.shape[0]
            idx = np.array([(i, j, k, l) for i in range(n) for j in range(i + 1)
                            for k in range(n) for l in range(k + 1)
                            if i * (i + 1) // 2 + j >= k * (k + 1) // 2 + l])
            out["index"] = idx
            out[f"{kind}_{omega}"] = t[idx[:, 0], idx[:, 1], idx[:, 2], idx[:, 3]]
    finally:
        ElectronRepulsionIntegralImproved.boys_func = saved
    np.savez_compressed(os.path.join(HERE, "range_separated.npz"), **out)
    print({k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
