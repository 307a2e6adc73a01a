"""Write ``horton_overflow.json``: the large-exponent (ss|ff) known answer of gbasis's
``tests/test_two_elec_int.py`` (``test_compute_two_elec_integrals_overflow_horton``, marked
xfail there: "integrals with larger angular momentum and exponents results in an overflow").

The quartet's s shells are contracted over 8 and 9 primitives up to an exponent of 1149 with
alternating-sign coefficients, and the f shells have one primitive of exponent 0.725.  Built
from the s pair, the electron-transfer step multiplies by (zeta/eta)^6 and the double result
loses every digit; built from the f pair it needs no transfer.  The fixture records the
inputs and HORTON's value as the reference's test states them, the reference's own double
result (which misses), and the 40-digit value of ``oracle.eri_mp``.

Run in a checkout that has the reference: ``python tests/golden/make_horton_overflow.py``.
"""
from __future__ import annotations

import argparse
import ast
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
TEST = "test_compute_two_elec_integrals_overflow_horton"


def _literal(node):
    # np.array([...]) -> the list; plain literals as they are
    if isinstance(node, ast.Call) and getattr(node.func, "attr", "") == "array":
        return ast.literal_eval(node.args[0])
    return ast.literal_eval(node)


def parse(path):
    tree = ast.parse(open(path).read())
    fn = next(n for n in ast.walk(tree) if isinstance(n, ast.FunctionDef) and n.name == TEST)
    call = next(n for n in ast.walk(fn) if isinstance(n, ast.Call)
                and getattr(n.func, "attr", "") == "allclose")
    inner, expected = call.args
    args = [_literal(a) for a in inner.args[1:]]  # skip boys_func
    shells = []
    for n in range(4):  # coord, angmom, components, exps, coeffs per shell
        coord, l, comps, exps, coeffs = args[5 * n: 5 * n + 5]
        shells.append({"coord": coord, "angmom": l, "components": comps, "exps": exps,
                       "coeffs": coeffs})
    return shells, float(ast.literal_eval(expected))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="path of a gbasis source checkout")
    a = ap.parse_args()
    shells, expected = parse(os.path.join(a.reference, "tests", "test_two_elec_int.py"))

    sys.path.insert(0, a.reference)
    from gbasis.integrals._two_elec_int import _compute_two_elec_integrals
    from gbasis.integrals.point_charge import PointChargeIntegral
    flat = []
    for s in shells:
        flat += [np.array(s["coord"], dtype=float), s["angmom"], np.array(s["components"]),
                 np.array(s["exps"], dtype=float), np.array(s["coeffs"], dtype=float)]
    ref_value = float(np.ravel(_compute_two_elec_integrals(PointChargeIntegral.boys_func, *flat))[0])

    sys.path.insert(0, ROOT)
    from gbasis_b200.contractions import GeneralizedContractionShell
    from oracle import eri_mp
    gs = [GeneralizedContractionShell(s["angmom"], np.array(s["coord"], dtype=float),
                                      np.array(s["coeffs"], dtype=float),
                                      np.array(s["exps"], dtype=float), "cartesian")
          for s in shells]
    blk = eri_mp.quartet_cartesian_mp(*gs)  # (La, Lb, Lc, Ld, Ma, Mb, Mc, Md)
    idx = []
    for s, g in zip(shells, gs):
        comps = [tuple(int(v) for v in row) for row in g.angmom_components_cart]
        idx.append(comps.index(tuple(s["components"][0])))
    truth = float(blk[idx[0], idx[1], idx[2], idx[3], 0, 0, 0, 0])

    rec = {"source": f"gbasis tests/test_two_elec_int.py::{TEST}", "shells": shells,
           "horton": expected, "reference_double": ref_value, "truth_40_digits": truth}
    json.dump(rec, open(os.path.join(HERE, "horton_overflow.json"), "w"), indent=1)
    print(f"horton {expected!r}  reference {ref_value!r}  40-digit {truth!r}")


if __name__ == "__main__":
    main()
