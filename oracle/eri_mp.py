"""Arbitrary-precision ERI evaluator — TEST INFRASTRUCTURE ONLY.

Evaluates the same Obara-Saika / electron-transfer / horizontal recursions as
:mod:`oracle.eri_oracle` (which follows ``gbasis/integrals/_two_elec_int.py:149-814``)
on scalars in mpmath with 40 significant digits.  Every recursion path then gives
the same value to far below double precision, so this is the "true" value a double
implementation is measured against where the double-precision reference itself loses
digits (diffuse high-l quartets, where gbasis's two ERI paths disagree with each other).
"""
from __future__ import annotations

from functools import lru_cache

import mpmath as mp
import numpy as np

__all__ = ["quartet_cartesian_mp"]


def _boys(m, T):
    # F_m(T) = 1F1(m+1/2; m+3/2; -T) / (2m+1)   (gbasis/integrals/boys_functions.py:63)
    return mp.hyp1f1(m + mp.mpf(1) / 2, m + mp.mpf(3) / 2, -T) / (2 * m + 1)


def _dfact(n):
    r = 1
    while n > 1:
        r *= n
        n -= 2
    return r


def _triples(l):
    return [(x, y, l - x - y) for x in range(l, -1, -1) for y in range(l - x, -1, -1)]


def _prim_vrr_etr(ea, eb, ec, ed, A, B, C, D, L, lc_ld):
    """[e0|f0] for one primitive quartet (unnormalised), all e <= L - |f|, |f| <= lc+ld."""
    zeta, eta = ea + eb, ec + ed
    rho = zeta * eta / (zeta + eta)
    P = [(ea * A[i] + eb * B[i]) / zeta for i in range(3)]
    Q = [(ec * C[i] + ed * D[i]) / eta for i in range(3)]
    PA = [P[i] - A[i] for i in range(3)]
    QC = [Q[i] - C[i] for i in range(3)]
    PQ = [P[i] - Q[i] for i in range(3)]
    AB2 = sum((A[i] - B[i]) ** 2 for i in range(3))
    CD2 = sum((C[i] - D[i]) ** 2 for i in range(3))
    T = rho * sum(v * v for v in PQ)
    pref = 2 * mp.pi ** mp.mpf(2.5) / (zeta * eta * mp.sqrt(zeta + eta)) \
        * mp.exp(-ea * eb / zeta * AB2) * mp.exp(-ec * ed / eta * CD2)
    F = [pref * _boys(m, T) for m in range(L + 1)]
    WP = [-rho / zeta * PQ[i] for i in range(3)]

    @lru_cache(maxsize=None)
    def V(e, m):
        if min(e) < 0:
            return mp.mpf(0)
        if e == (0, 0, 0):
            return F[m]
        i = next(k for k in range(3) if e[k] > 0)
        e1 = list(e); e1[i] -= 1; e1 = tuple(e1)
        e2 = list(e1); e2[i] -= 1; e2 = tuple(e2)
        v = PA[i] * V(e1, m) + WP[i] * V(e1, m + 1)
        if e1[i] > 0:
            v += mp.mpf(e1[i]) / (2 * zeta) * (V(e2, m) - rho / zeta * V(e2, m + 1))
        return v

    @lru_cache(maxsize=None)
    def Et(e, f):
        if min(e) < 0 or min(f) < 0:
            return mp.mpf(0)
        if f == (0, 0, 0):
            return V(e, 0)
        i = next(k for k in range(3) if f[k] > 0)
        f1 = list(f); f1[i] -= 1; f1 = tuple(f1)
        ep = list(e); ep[i] += 1; ep = tuple(ep)
        em = list(e); em[i] -= 1; em = tuple(em)
        f2 = list(f1); f2[i] -= 1; f2 = tuple(f2)
        v = (QC[i] + zeta / eta * PA[i]) * Et(e, f1) - zeta / eta * Et(ep, f1)
        if e[i] > 0:
            v += mp.mpf(e[i]) / (2 * eta) * Et(em, f1)
        if f1[i] > 0:
            v += mp.mpf(f1[i]) / (2 * eta) * Et(e, f2)
        return v

    return Et


def quartet_cartesian_mp(sa, sb, sc, sd, dps=40):
    """Same layout as ``oracle.eri_oracle.quartet_cartesian`` (L_a,L_b,L_c,L_d,M_a,...), float64."""
    with mp.workdps(dps):
        shells = (sa, sb, sc, sd)
        ls = [s.angmom for s in shells]
        la, lb, lc, ld = ls
        L = sum(ls)
        X = [[mp.mpf(float(v)) for v in s.coord] for s in shells]
        A, B, C, D = X
        exps = [[mp.mpf(float(v)) for v in s.exps] for s in shells]
        coefs = []
        for s, l in zip(shells, ls):
            cf = np.asarray(s.coeffs, dtype=float)
            cf = cf[:, None] if cf.ndim == 1 else cf
            cc = []
            for k, e in enumerate(exps[len(coefs)]):
                nrm = (2 * e / mp.pi) ** mp.mpf(0.75) * (4 * e) ** (mp.mpf(l) / 2)
                cc.append([mp.mpf(float(cf[k, m])) * nrm for m in range(cf.shape[1])])
            coefs.append(cc)
        Ms = [len(c[0]) for c in coefs]
        es = [(e,) for e in []]  # placeholder to keep linters calm
        del es
        e_list = [e for n in range(la, la + lb + 1) for e in _triples(n)]
        f_list = [f for n in range(lc, lc + ld + 1) for f in _triples(n)]
        G = {}
        for ia, a_ in enumerate(exps[0]):
            for ib, b_ in enumerate(exps[1]):
                for ic, c_ in enumerate(exps[2]):
                    for id_, d_ in enumerate(exps[3]):
                        Et = _prim_vrr_etr(a_, b_, c_, d_, A, B, C, D, L, lc + ld)
                        for e in e_list:
                            for f in f_list:
                                v = Et(e, f)
                                for ma in range(Ms[0]):
                                    for mb in range(Ms[1]):
                                        for mc in range(Ms[2]):
                                            for md in range(Ms[3]):
                                                key = (e, f, ma, mb, mc, md)
                                                w = coefs[0][ia][ma] * coefs[1][ib][mb] \
                                                    * coefs[2][ic][mc] * coefs[3][id_][md]
                                                G[key] = G.get(key, 0) + v * w
        AB = [A[i] - B[i] for i in range(3)]
        CD = [C[i] - D[i] for i in range(3)]

        def hrr(e, f, c, d, ms):
            # (e | c d) from [e | f], then (a b | c d) from (e | c d)
            @lru_cache(maxsize=None)
            def H(ee, cc, dd):
                if dd == (0, 0, 0):
                    return G[(ee, cc) + ms]
                i = next(k for k in range(3) if dd[k] > 0)
                d1 = list(dd); d1[i] -= 1; d1 = tuple(d1)
                cp = list(cc); cp[i] += 1; cp = tuple(cp)
                return H(ee, cp, d1) + CD[i] * H(ee, cc, d1)
            return H

        comps = [np.asarray(s.angmom_components_cart) for s in shells]
        out = np.zeros([len(c) for c in comps] + Ms)
        for ma in range(Ms[0]):
            for mb in range(Ms[1]):
                for mc in range(Ms[2]):
                    for md in range(Ms[3]):
                        ms = (ma, mb, mc, md)
                        H = hrr(None, None, None, None, ms)

                        @lru_cache(maxsize=None)
                        def R(aa, bb, cc, dd):
                            if bb == (0, 0, 0):
                                return H(aa, cc, dd)
                            i = next(k for k in range(3) if bb[k] > 0)
                            b1 = list(bb); b1[i] -= 1; b1 = tuple(b1)
                            ap = list(aa); ap[i] += 1; ap = tuple(ap)
                            return R(ap, b1, cc, dd) + AB[i] * R(aa, b1, cc, dd)

                        for i0, a0 in enumerate(comps[0]):
                            for i1, a1 in enumerate(comps[1]):
                                for i2, a2 in enumerate(comps[2]):
                                    for i3, a3 in enumerate(comps[3]):
                                        t = [tuple(int(v) for v in x) for x in (a0, a1, a2, a3)]
                                        val = R(*t)
                                        nrm = 1
                                        for x in t:
                                            nrm *= _dfact(2 * x[0] - 1) * _dfact(2 * x[1] - 1) \
                                                * _dfact(2 * x[2] - 1)
                                        out[i0, i1, i2, i3, ma, mb, mc, md] = float(val / mp.sqrt(nrm))
        return out
