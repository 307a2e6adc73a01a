"""Regenerate the golden fixtures in this folder from the gbasis reference itself.

Run in a checkout that has the reference sources (pure Python) on disk:

    python tests/golden/make_golden.py --reference /path/to/gbasis

It imports gbasis from ``--reference`` and writes small ``.npz``/``.json`` files next to
this script.  The tests only read the written fixtures; they never import gbasis.

Fixtures:
  * ``horton_scalars.json`` — the HORTON-derived primitive ERIs pinned by gbasis's
    ``tests/test_two_elec_int.py`` (``test_two_int_brute``), parsed from that file's
    ``assert np.allclose(two_int_brute(...), value)`` statements.
  * ``horton_bec_sto6g.npz`` — Be/C STO-6G shells (parsed by gbasis) with HORTON component
    order, gbasis's stored HORTON tensor (``tests/data_horton_bec_cart_elec_repulsion.npy``)
    and the reference's own ``electron_repulsion_integral`` output on the same basis.
  * ``quartets.npz`` — ``ElectronRepulsionIntegral.construct_array_contraction`` blocks for
    seeded random quartets covering every class with l <= 3, generalized contractions
    included; the improved path's blocks for the same quartets; and 40-digit values of the
    same blocks from ``oracle/eri_mp.py`` ("truth": both reference paths lose digits on some
    diffuse high-l quartets, by up to ~1e-6 absolute).
  * ``tiny4.npz`` — the full chemist tensor of the 4-atom workload (unique elements only).
  * ``mixed.npz`` — a small mixed Cartesian/spherical basis: cartesian, spherical, mix and
    lincomb arrays in both notations, and the Schwarz-screened improved path.
  * ``norm_cont.npz`` and ``boys.npz`` — shell normalisation and Boys values.
"""
from __future__ import annotations

import argparse
import ast
import itertools as it
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))


def shell_record(s, cart_order=None, sph_order=None):
    rec = {
        "angmom": int(s.angmom),
        "coord": [float(v) for v in s.coord],
        "exps": [float(v) for v in s.exps],
        "coeffs": np.asarray(s.coeffs, dtype=float).tolist(),
        "coord_type": s.coord_type,
    }
    if cart_order is not None:
        rec["cart_order"] = np.asarray(cart_order).tolist()
    if sph_order is not None:
        rec["sph_order"] = list(sph_order)
    return rec


def unique_index(n):
    """(i, j, k, l) with i >= j, k >= l, (ij) >= (kl): one representative per 8-fold orbit."""
    return np.array([(i, j, k, l) for i in range(n) for j in range(i + 1)
                     for k in range(n) for l in range(k + 1)
                     if i * (i + 1) // 2 + j >= k * (k + 1) // 2 + l], dtype=np.int16)


def parse_horton_scalars(path):
    """(args, kwargs, expected) of every ``two_int_brute(..., output=True)`` assertion."""
    tree = ast.parse(open(path).read())
    out = []
    for node in ast.walk(tree):
        if not (isinstance(node, ast.Call) and getattr(node.func, "attr", "") == "allclose"):
            continue
        call, expected = node.args[0], node.args[1]
        if not (isinstance(call, ast.Call) and getattr(call.func, "id", "") == "two_int_brute"):
            continue
        kw = {k.arg: ast.literal_eval(k.value) for k in call.keywords}
        if not kw.get("output", False):
            continue
        args = [ast.literal_eval(a) for a in call.args]
        kw.pop("output")
        out.append({"args": args, "kwargs": kw, "expected": float(ast.literal_eval(expected))})
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", required=True, help="path of a gbasis source checkout")
    a = ap.parse_args()
    sys.path.insert(0, a.reference)
    from gbasis.contractions import GeneralizedContractionShell as RefShell
    from gbasis.integrals.electron_repulsion import (
        ElectronRepulsionIntegral,
        ElectronRepulsionIntegralImproved,
        electron_repulsion_integral,
        electron_repulsion_integral_improved,
    )
    from gbasis.integrals.point_charge import PointChargeIntegral
    from gbasis.parsers import make_contractions, parse_nwchem

    class HortonShell(RefShell):
        @property
        def angmom_components_cart(self):
            return np.array([(c.count(0), c.count(1), c.count(2))
                             for c in it.combinations_with_replacement(range(3), self.angmom)])

        @property
        def angmom_components_sph(self):
            if self.angmom == 1:
                return ("c1", "s1", "c0")
            cos = [f"c{m}" for m in range(1, self.angmom + 1)]
            sin = [f"s{m}" for m in range(1, self.angmom + 1)]
            o = ["c0"] + [None] * (2 * self.angmom)
            o[1::2] = cos
            o[2::2] = sin
            return o

    # ---- HORTON scalars
    scal = parse_horton_scalars(os.path.join(a.reference, "tests", "test_two_elec_int.py"))
    json.dump(scal, open(os.path.join(HERE, "horton_scalars.json"), "w"), indent=0)
    print("horton scalars:", len(scal))

    # ---- Be/C STO-6G with HORTON order
    bd = parse_nwchem(os.path.join(a.reference, "tests", "data_sto6g.nwchem"))
    basis = make_contractions(bd, ["Be", "C"], np.array([[0, 0, 0], [1.0, 0, 0]]), "cartesian")
    basis = [HortonShell(s.angmom, s.coord, s.coeffs, s.exps, s.coord_type) for s in basis]
    horton = np.load(os.path.join(a.reference, "tests", "data_horton_bec_cart_elec_repulsion.npy"))
    ref = electron_repulsion_integral(basis)
    recs = [shell_record(s, s.angmom_components_cart, s.angmom_components_sph) for s in basis]
    np.savez_compressed(os.path.join(HERE, "horton_bec_sto6g.npz"),
                        shells=json.dumps(recs), horton=horton, reference=np.ascontiguousarray(ref))
    print("bec", ref.shape, np.abs(ref - horton).max())

    # ---- random quartets, every class with l <= 3
    rng = np.random.default_rng(12345)
    qrecs, blocks = [], []

    def rshell(l, K, M):
        exps = np.exp(rng.uniform(np.log(0.08), np.log(30.0), size=K))
        coeffs = rng.uniform(-0.2, 1.0, size=(K, M)) if M > 1 else rng.uniform(0.1, 1.0, size=K)
        return RefShell(l, rng.uniform(-2.0, 2.0, size=3), coeffs, exps, "cartesian")

    for la, lb, lc, ld in it.product(range(4), repeat=4):
        if rng.uniform() > 0.35 and (la, lb, lc, ld) != (0, 0, 0, 0) and max(la, lb, lc, ld) < 3:
            continue
        if max(la, lb, lc, ld) == 3 and rng.uniform() > 0.25:
            continue
        Ks = [int(rng.integers(1, 4)) for _ in range(4)]
        Ms = [1, 1, 1, 1]
        if rng.uniform() < 0.2:
            Ms[int(rng.integers(0, 4))] = 2
        sh = [rshell(l, K, M) for l, K, M in zip((la, lb, lc, ld), Ks, Ms)]
        blk = ElectronRepulsionIntegral.construct_array_contraction(*sh)
        qrecs.append([shell_record(s) for s in sh])
        blocks.append(np.ascontiguousarray(blk).ravel())
    # shared centres (AB = 0 and P = Q) and large exponents
    for ls in [(1, 1, 1, 1), (2, 0, 2, 0), (2, 2, 1, 0), (3, 1, 2, 0)]:
        c0 = rng.uniform(-1, 1, size=3)
        sh = []
        for l in ls:
            exps = np.array([0.3, 2.0, 40.0])[: 1 + l % 3]
            sh.append(RefShell(l, c0.copy(), rng.uniform(0.1, 1, size=len(exps)), exps,
                               "cartesian"))
        qrecs.append([shell_record(s) for s in sh])
        blocks.append(np.ascontiguousarray(
            ElectronRepulsionIntegral.construct_array_contraction(*sh)).ravel())
    # 40-digit values of the same blocks (the recursion is evaluated in mpmath)
    from oracle.eri_mp import quartet_cartesian_mp
    truth, improved = [], []
    for rq in qrecs:
        sh = [RefShell(r["angmom"], np.array(r["coord"]), np.array(r["coeffs"]),
                       np.array(r["exps"]), r["coord_type"]) for r in rq]
        truth.append(np.transpose(quartet_cartesian_mp(*sh), (4, 0, 5, 1, 6, 2, 7, 3)).ravel())
        improved.append(np.ascontiguousarray(
            ElectronRepulsionIntegralImproved.construct_array_contraction(*sh)).ravel())
    np.savez_compressed(os.path.join(HERE, "quartets.npz"), shells=json.dumps(qrecs),
                        blocks=np.concatenate(blocks), truth=np.concatenate(truth),
                        improved=np.concatenate(improved),
                        sizes=np.array([b.size for b in blocks]))
    print("quartets:", len(blocks))

    # ---- tiny4 workload full tensor (unique elements)
    from gbasis_b200.synthetic import make_workload
    mine = make_workload("tiny4")
    refb = [RefShell(s.angmom, s.coord, s.coeffs[:, 0], s.exps, s.coord_type) for s in mine]
    full = electron_repulsion_integral(refb, notation="chemist")
    n = full.shape[0]
    idx = unique_index(n)
    np.savez_compressed(os.path.join(HERE, "tiny4.npz"), index=idx,
                        values=full[idx[:, 0], idx[:, 1], idx[:, 2], idx[:, 3]],
                        shells=json.dumps([shell_record(s) for s in refb]))
    print("tiny4:", full.shape, len(idx))

    # ---- mixed small basis (unique elements of each 8-fold symmetric array)
    rng = np.random.default_rng(777)
    # compact exponents and short distances keep every path well conditioned here
    centers = [np.array([0.0, 0.0, 0.0]), np.array([0.7, -0.3, 0.4])]
    mixed = []
    for ci, (l, K, M, ct) in enumerate([(0, 3, 1, "spherical"), (1, 2, 1, "cartesian"),
                                        (2, 2, 2, "spherical"), (3, 1, 1, "spherical")]):
        exps = np.exp(rng.uniform(np.log(0.6), np.log(6.0), size=K))
        coeffs = rng.uniform(0.1, 1.0, size=(K, M)) if M > 1 else rng.uniform(0.1, 1.0, size=K)
        mixed.append(RefShell(l, centers[ci % 2] + rng.uniform(-0.3, 0.3, size=3), coeffs, exps, ct))
    erep = ElectronRepulsionIntegral(mixed)
    cts = [s.coord_type for s in mixed]
    arrays = {"mix": erep.construct_array_mix(cts), "cart": erep.construct_array_cartesian(),
              "sph": erep.construct_array_spherical()}
    nmix = arrays["mix"].shape[0]
    T = rng.normal(size=(nmix - 3, nmix))
    arrays["lincomb"] = electron_repulsion_integral(mixed, transform=T, notation="chemist")
    arrays["screened"] = electron_repulsion_integral_improved(mixed, notation="chemist",
                                                               schwarz_threshold=1e-3)
    phys = electron_repulsion_integral(mixed)
    assert np.array_equal(np.transpose(phys, (0, 2, 1, 3)), arrays["mix"])
    # 40-digit blocks assembled the same way ("truth")
    from oracle import eri_oracle as orc
    from oracle.eri_mp import quartet_cartesian_mp
    mp_block = lambda a_, b_, c_, d_: np.transpose(  # noqa: E731
        quartet_cartesian_mp(a_, b_, c_, d_), (4, 0, 5, 1, 6, 2, 7, 3))
    truth = {"mix": orc.construct_array(mixed, cts, quartet_fn=mp_block),
             "cart": orc.construct_array(mixed, ["cartesian"] * 4, quartet_fn=mp_block),
             "sph": orc.construct_array(mixed, ["spherical"] * 4, quartet_fn=mp_block)}
    truth["lincomb"] = orc.construct_array_lincomb(truth["mix"], T)
    Qm = orc.schwarz_bounds(mixed)
    truth["screened"] = orc.construct_array(
        mixed, cts, quartet_fn=mp_block, screen=lambda i, j, k, l: Qm[i, j] * Qm[k, l] >= 1e-3)
    out = {"shells": json.dumps([shell_record(s) for s in mixed]), "transform": T}
    for k, v in arrays.items():
        ix = unique_index(v.shape[0])
        out[k + "_n"] = np.array(v.shape[0])
        out[k] = v[ix[:, 0], ix[:, 1], ix[:, 2], ix[:, 3]]
        out[k + "_truth"] = truth[k][ix[:, 0], ix[:, 1], ix[:, 2], ix[:, 3]]
    np.savez_compressed(os.path.join(HERE, "mixed.npz"), **out)
    print("mixed:", {k: v.shape for k, v in arrays.items()})

    # ---- norm_cont and Boys
    nc_recs, nc_vals = [], []
    for l in range(5):
        for K, M in [(1, 1), (3, 1), (4, 2)]:
            s = rshell(l, K, M)
            nc_recs.append(shell_record(s))
            nc_vals.append(np.asarray(s.norm_cont).ravel())
    np.savez_compressed(os.path.join(HERE, "norm_cont.npz"), shells=json.dumps(nc_recs),
                        values=np.concatenate(nc_vals), sizes=np.array([v.size for v in nc_vals]))
    Tg = np.concatenate([np.linspace(0, 1, 41), np.linspace(1, 60, 237), [1e-12, 1e-8, 80.0, 200.0, 1500.0]])
    mg = np.arange(0, 25)
    F = PointChargeIntegral.boys_func(mg[:, None], Tg[None, :])
    np.savez_compressed(os.path.join(HERE, "boys.npz"), T=Tg, m=mg, F=F)
    print("done")


if __name__ == "__main__":
    main()
