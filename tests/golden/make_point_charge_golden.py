"""Regenerate ``point_charge.npz`` (this folder) from the gbasis reference itself.

    python tests/golden/make_point_charge_golden.py --reference /path/to/gbasis

Imports gbasis from ``--reference``; the basis sets are the shells stored in ``mixed.npz``
(Cartesian and spherical shells, s to f, a generalized contraction) and ``tiny4.npz``.
Writes, for seeded point charges: ``point_charge_integral`` (K, K, N) of both bases, the
``transform`` (lincomb) form and ``nuclear_electron_attraction_integral`` of the mixed basis.
The tests only read the written file; they never import gbasis.
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
    from gbasis.integrals.nuclear_electron_attraction import nuclear_electron_attraction_integral
    from gbasis.integrals.point_charge import point_charge_integral

    def basis_of(name):
        z = np.load(os.path.join(HERE, name), allow_pickle=False)
        recs = json.loads(str(z["shells"]))
        return [RefShell(r["angmom"], np.array(r["coord"]), np.array(r["coeffs"]),
                         np.array(r["exps"]), r["coord_type"]) for r in recs], z

    rng = np.random.default_rng(2468)
    out = {}
    mixed, zm = basis_of("mixed.npz")
    coords = rng.uniform(-1.5, 1.5, size=(5, 3))
    charges = rng.uniform(0.5, 6.0, size=5)
    out["mixed_coords"], out["mixed_charges"] = coords, charges
    out["mixed_pc"] = point_charge_integral(mixed, coords, charges)
    out["mixed_pc_lincomb"] = point_charge_integral(mixed, coords, charges,
                                                    transform=zm["transform"])
    out["mixed_nuc"] = nuclear_electron_attraction_integral(mixed, coords, charges)
    tiny, _ = basis_of("tiny4.npz")
    coords = rng.uniform(-3.0, 3.0, size=(4, 3))
    charges = rng.uniform(1.0, 8.0, size=4)
    out["tiny4_coords"], out["tiny4_charges"] = coords, charges
    out["tiny4_pc"] = point_charge_integral(tiny, coords, charges)
    np.savez_compressed(os.path.join(HERE, "point_charge.npz"), **out)
    print({k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
