"""CPU tests: the C-ABI library loads and exports every declared symbol; host-side packing;
the generated recursion code (run here as Python) against the oracle for every class."""
import ctypes
import os
import re
import sys

import numpy as np
import pytest

from conftest import ROOT, OrderedShell
from gbasis_b200 import _engine
from gbasis_b200.contractions import GeneralizedContractionShell
from oracle import eri_oracle as orc

sys.path.insert(0, os.path.join(ROOT, "gbasis_b200", "csrc"))
import gen_eri  # noqa: E402


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "gbx_eri.h")).read()
    return sorted(set(re.findall(r"^int (gbx_\w+)\(", txt, flags=re.M)))


def test_library_exports_every_declared_symbol():
    if not os.path.exists(_engine.LIB_PATH):
        pytest.skip("engine library not built")
    L = ctypes.CDLL(_engine.LIB_PATH)
    syms = header_symbols()
    assert len(syms) >= 12
    for s in syms:
        assert hasattr(L, s), s
    assert set(syms) == set(_engine.EXPORTED_SYMBOLS)


def test_last_error_roundtrip_without_gpu():
    if not os.path.exists(_engine.LIB_PATH):
        pytest.skip("engine library not built")
    L = _engine.lib()
    rc = L.gbx_basis_create(ctypes.byref(ctypes.c_void_p()), 0, None, None, None, None, None,
                            None, None, None, None, 0)
    assert rc == _engine.GBX_ERR_INVALID
    assert "null argument" in _engine.last_error()
    with pytest.raises(ValueError):
        _engine.check(rc)


def test_pack_cartesian_default_and_custom_order():
    s = GeneralizedContractionShell(2, np.zeros(3), np.array([0.5, 0.5]), np.array([1.0, 3.0]),
                                    "cartesian")
    pk = _engine.pack_basis([s])
    pos = pk["pos"].reshape(-1, 10)[0, :6]
    assert list(pos) == [0, 1, 2, 3, 4, 5]
    scl = pk["scl"].reshape(-1, 10)[0, :6]
    nc = s.norm_cont[0, 0]
    np.testing.assert_allclose(scl, nc * np.array([1 / np.sqrt(3), 1, 1, 1 / np.sqrt(3), 1,
                                                   1 / np.sqrt(3)]))
    rev = OrderedShell(2, np.zeros(3), np.array([1.0]), np.array([1.0]), "cartesian",
                       cart_order=orc.cart_components(2)[::-1])
    assert list(_engine.pack_basis([rev])["pos"][:6]) == [5, 4, 3, 2, 1, 0]


def test_pack_spherical_labels_signs_and_generalized():
    s = OrderedShell(2, np.zeros(3), np.array([[0.5, 0.2], [0.5, 0.9]]), np.array([1.0, 3.0]),
                     "spherical", sph_order=("c0", "-s1", "c1", "s2", "c2"))
    pk = _engine.pack_basis([s])
    assert list(pk["nout"]) == [5, 5]  # two segmented contractions
    assert list(pk["group"]) == [0, 0]
    pos = pk["pos"].reshape(-1, 10)[0, :5]
    # internal order s2 s1 c0 c1 c2 -> positions in ("c0","-s1","c1","s2","c2")
    assert list(pos) == [3, 1, 0, 2, 4]
    scl = pk["scl"].reshape(-1, 10)[1, :5]
    assert scl[1] < 0 and np.all(scl[[0, 2, 3, 4]] > 0)
    with pytest.raises(TypeError):
        _engine.pack_basis([s, "not a shell"])


def _pyexec(lines, env):
    code = []
    for ln in lines:
        ln = ln.strip().rstrip(";")
        ln = re.sub(r"^(const )?(R|double) ", "", ln)
        code.append(ln)
    exec("\n".join(code), env)


# The straight-line register code that the device compiles: every light class and the (ab|ss)
# structs of the point-charge kernel (the heavy classes run the line, split and cooperative
# kernels, whose generated code is checked in tests/test_lines_host.py and below); plus every
# class with l <= 2.
_REGISTER_CLASSES = sorted(
    set(gen_eri.canonical_classes(2))
    | {c for c in gen_eri.canonical_classes(3) if gen_eri.is_light(c)}
    | {(la, lb, 0, 0) for la in range(4) for lb in range(4)})


def test_register_emitter_refuses_classes_beyond_its_checked_range():
    assert max(sum(c) for c in _REGISTER_CLASSES) <= gen_eri.MAX_EMIT_L
    with pytest.raises(ValueError):
        gen_eri.emit_all(3, [(3, 3, 3, 3)])


@pytest.mark.parametrize("cls", _REGISTER_CLASSES)
def test_generated_recursions_match_oracle(cls):
    la, lb, lc, ld = cls
    rng = np.random.default_rng(sum((i + 1) * v for i, v in enumerate(cls)))
    shells = [GeneralizedContractionShell(l, rng.uniform(-1, 1, 3), np.array([1.0]),
                                          np.array([rng.uniform(0.3, 3.0)]), "cartesian")
              for l in cls]
    ref = orc.quartet_cartesian(*shells)[..., 0, 0, 0, 0]
    (a, A), (b, B), (c, C), (d, D) = [(float(s.exps[0]), s.coord) for s in shells]
    z, e = a + b, c + d
    P, Q = (a * A + b * B) / z, (c * C + d * D) / e
    rho = z * e / (z + e)
    PQ = P - Q
    T = rho * PQ @ PQ
    norm = np.prod([(2 * s.exps[0] / np.pi) ** 0.75 * (4 * s.exps[0]) ** (s.angmom / 2)
                    for s in shells])
    pref = 2 * np.pi ** 2.5 / (z * e * np.sqrt(z + e)) * np.exp(-a * b / z * (A - B) @ (A - B)) \
        * np.exp(-c * d / e * (C - D) @ (C - D)) * norm
    L = sum(cls)
    F = [pref * float(orc.boys(m, T)) for m in range(L + 1)]
    g = gen_eri.best_prim(la, lb, lc, ld)
    h = gen_eri.HrrGen(la, lb, lc, ld)
    acc = [0.0] * (len(g.E) * len(g.F))
    out = [0.0] * (gen_eri.ncart(la) * gen_eri.ncart(lb) * gen_eri.ncart(lc) * gen_eri.ncart(ld))
    PA, QC = P - A, Q - C
    rz = rho / z
    ze = z / e
    env = dict(fma=lambda x, y, w: x * y + w, R=float, F=F, acc=acc, out=out,
               PAx=PA[0], PAy=PA[1], PAz=PA[2], WPx=-rz * PQ[0], WPy=-rz * PQ[1], WPz=-rz * PQ[2],
               o2z=0.5 / z, rz=rz, CEx=QC[0] + ze * PA[0], CEy=QC[1] + ze * PA[1],
               CEz=QC[2] + ze * PA[2], ze=ze, o2e=0.5 / e)
    lines = []
    g.emit(lines)
    _pyexec(lines, env)
    AB, CD = A - B, C - D
    env.update(ABx=AB[0], ABy=AB[1], ABz=AB[2], CDx=CD[0], CDy=CD[1], CDz=CD[2])
    lines = []
    h.emit(lines)
    _pyexec(lines, env)
    got = np.array(out).reshape(ref.shape)
    cn = [1 / np.sqrt(np.prod(orc.factorial2(2 * orc.cart_components(l) - 1), axis=1)) for l in cls]
    got = np.einsum("abcd,a,b,c,d->abcd", got, *cn)
    np.testing.assert_allclose(got, ref, rtol=1e-11, atol=1e-14)


import gen_coop  # noqa: E402


def _run_coop_program(cls, shells):
    """Interpret one class's cooperative program (as the warp kernel does) for one primitive
    quartet, Cartesian output (component norms applied)."""
    prog = gen_coop.program(*cls)
    (a, A), (b, B), (c, C), (d, D) = [(float(s.exps[0]), s.coord) for s in shells]
    z, e = a + b, c + d
    P, Q = (a * A + b * B) / z, (c * C + d * D) / e
    rho = z * e / (z + e)
    PQ = P - Q
    T = rho * PQ @ PQ
    norm = np.prod([(2 * s.exps[0] / np.pi) ** 0.75 * (4 * s.exps[0]) ** (s.angmom / 2)
                    for s in shells])
    pref = 2 * np.pi ** 2.5 / (z * e * np.sqrt(z + e)) * np.exp(-a * b / z * (A - B) @ (A - B)) \
        * np.exp(-c * d / e * (C - D) @ (C - D)) * norm
    L = sum(cls)
    X = np.zeros(prog["nX"])
    X[:L + 1] = [pref * float(orc.boys(m, T)) for m in range(L + 1)]
    PA, QC = P - A, Q - C
    rz, ze = rho / z, z / e
    WP, CE = -rz * PQ, QC + ze * PA
    for (dst, s1, s2, s3, s4, i, k, _) in prog["vins"]:
        v = PA[i] * X[s1] + WP[i] * X[s2]
        if k:
            v += k * 0.5 / z * (X[s3] - rz * X[s4])
        X[dst] = v
    for (dst, s1, s2, s3, s4, i, k1, k2) in prog["tins"]:
        v = CE[i] * X[s1] - ze * X[s2]
        if k1:
            v += k1 * 0.5 / e * X[s3]
        if k2:
            v += k2 * 0.5 / e * X[s4]
        X[dst] = v
    NE, NF = prog["NE"], prog["NF"]
    acc = X[prog["targets"]].reshape(NE, NF)
    CD, AB = C - D, A - B
    NCD = len(prog["kfin"])
    HF = np.zeros((NE, NCD))
    for r in range(NE):
        K = np.zeros(prog["nK"])
        K[:NF] = acc[r]
        for (dst, s1, s2, _, _, i, _, _) in prog["kins"]:
            K[dst] = K[s1] + CD[i] * K[s2]
        HF[r] = K[prog["kfin"]]
    NAB = len(prog["bfin"])
    out = np.zeros((NAB, NCD))
    for col in range(NCD):
        Bn = np.zeros(prog["nB"])
        Bn[:NE] = HF[:, col]
        for (dst, s1, s2, _, _, i, _, _) in prog["bins"]:
            Bn[dst] = Bn[s1] + AB[i] * Bn[s2]
        out[:, col] = Bn[prog["bfin"]]
    la, lb, lc, ld = cls
    cn = [1 / np.sqrt(np.prod(orc.factorial2(2 * orc.cart_components(l) - 1), axis=1)) for l in cls]
    out = out.reshape(len(cn[0]), len(cn[1]), len(cn[2]), len(cn[3]))
    return np.einsum("abcd,a,b,c,d->abcd", out, *cn)


@pytest.mark.parametrize("cls", [(2, 2, 2, 2), (2, 2, 1, 2), (1, 2, 1, 2), (3, 3, 3, 3),
                                 (3, 0, 2, 2), (0, 3, 3, 1), (3, 2, 2, 3)])
def test_cooperative_programs_match_oracle(cls):
    rng = np.random.default_rng(7 + sum(cls))
    shells = [GeneralizedContractionShell(l, rng.uniform(-1, 1, 3), np.array([1.0]),
                                          np.array([rng.uniform(0.4, 2.5)]), "cartesian")
              for l in cls]
    ref = orc.quartet_cartesian(*shells)[..., 0, 0, 0, 0]
    got = _run_coop_program(cls, shells)
    np.testing.assert_allclose(got, ref, rtol=1e-10, atol=1e-13)
