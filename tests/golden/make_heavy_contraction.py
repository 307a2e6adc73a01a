"""Write ``heavy_contraction.npz``: one heavily contracted (dd|dd) shell quartet of the batch
workload (molecule 371, shells 0, 6, 0, 18: d shells of 6, 4, 6 and 5 primitives with
exponents from 0.25 to 28.6 on three atoms), with

* the reference's own block: ``ElectronRepulsionIntegral.construct_array_contraction`` of
  gbasis (its contracted recursions run from one fixed centre per pair, and on this quartet
  they miss the 40-digit values by about 1e-9);
* the 40-digit values of ``oracle.eri_mp``.

Layout of both: (M1, L1, M2, L2, M3, L3, M4, L4), chemist, without ``norm_cont``, as the
reference's call returns it.

Run: ``python tests/golden/make_heavy_contraction.py --reference /path/to/gbasis``.
"""
from __future__ import annotations

import argparse
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
MOLECULE, QUARTET = 371, (0, 6, 0, 18)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="path of a gbasis source checkout")
    a = ap.parse_args()
    sys.path.insert(0, ROOT)
    from gbasis_b200.synthetic import batch_molecule
    from oracle import eri_mp
    shells = [batch_molecule(MOLECULE)[i] for i in QUARTET]
    sys.path.insert(0, a.reference)
    from gbasis.contractions import GeneralizedContractionShell as RefShell
    from gbasis.integrals.electron_repulsion import ElectronRepulsionIntegral
    ref_shells = [RefShell(s.angmom, np.asarray(s.coord), np.asarray(s.coeffs), np.asarray(s.exps),
                           "cartesian") for s in shells]
    reference = ElectronRepulsionIntegral.construct_array_contraction(*ref_shells)
    truth = eri_mp.quartet_cartesian_mp(*shells, dps=40)          # (La, Lb, Lc, Ld, M...)
    truth = np.transpose(truth, (4, 0, 5, 1, 6, 2, 7, 3))
    np.savez_compressed(os.path.join(HERE, "heavy_contraction.npz"), reference=reference,
                        truth_40_digits=truth, molecule=MOLECULE, quartet=np.array(QUARTET))
    print("reference vs 40 digits: %.3e" % np.abs(reference - truth).max())


if __name__ == "__main__":
    main()
