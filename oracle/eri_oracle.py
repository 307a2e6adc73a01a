"""CPU oracle for the electron-repulsion-integral path — TEST INFRASTRUCTURE ONLY.

This module is the checker that the CUDA engine is compared against.  It is a
NumPy restatement of the algorithm of gbasis (theochem/gbasis) for the ERI
path; nothing in the product imports it.  Only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl reference``
legs of ``bench.py`` may call it.

Algorithm followed (reference file:line, paths inside the gbasis project):

* Boys function F_m(T) = 1F1(m+1/2; m+3/2; -T) / (2m+1)
  — ``gbasis/integrals/boys_functions.py:26-63`` (called through
  ``gbasis/integrals/point_charge.py:69-118``).
* [00|00]^(m) prefactor 2 pi^{5/2} / (zeta eta sqrt(zeta+eta)) K_AB K_CD F_m(T)
  — ``gbasis/integrals/_two_elec_int.py:335-348``.
* Obara-Saika vertical recursion on centre A
  — ``gbasis/integrals/_two_elec_int.py:350-399``.
* Electron-transfer recursion onto centre C
  — ``gbasis/integrals/_two_elec_int.py:413-526``.
* Primitive contraction with (2a/pi)^{3/4} (4a)^{l/2}
  — ``gbasis/integrals/_two_elec_int.py:528-547``.
* Horizontal recursion on D then on B
  — ``gbasis/integrals/_two_elec_int.py:549-788``.
* Cartesian component norm 1/sqrt(prod (2a_i-1)!!)
  — ``gbasis/integrals/_two_elec_int.py:793-812``.
* Per-quartet transpose to (M1,L1,M2,L2,M3,L3,M4,L4)
  — ``gbasis/integrals/electron_repulsion.py:86-211``.
* norm_cont scaling, spherical transform and 8-fold placement
  — ``gbasis/base_four_symm.py:160-616``.
* Real-solid-harmonic transformation matrices
  — ``gbasis/spherical.py:10-340``.
* Contraction normalisation (self-overlap)^-1/2
  — ``gbasis/contractions.py:503-524``.
* Public entry ``electron_repulsion_integral``
  — ``gbasis/integrals/electron_repulsion.py:214-281``.

The recursions are written here independently (dictionaries of arrays keyed by
Cartesian exponent triples, vectorised over the flattened primitive quartets);
they evaluate the same mathematics as the reference, so results agree to
floating-point noise (pinned by ``tests/test_oracle_golden.py`` against vectors
produced by the reference itself).
"""
from __future__ import annotations

import itertools
import math

import numpy as np
from scipy.special import comb, factorial, hyp1f1

__all__ = [
    "boys",
    "factorial2",
    "cart_components",
    "sph_components",
    "norm_cont",
    "generate_transformation",
    "quartet_cartesian",
    "construct_array_contraction",
    "construct_array_contraction_by_primitive",
    "construct_array",
    "construct_array_lincomb",
    "electron_repulsion_integral",
    "schwarz_bounds",
    "electron_repulsion_integral_screened",
]


# --------------------------------------------------------------------------- helpers
def factorial2(n):
    """n!! with n <= 0 -> 1 (``gbasis/utils.py:7-22``)."""
    n = np.asarray(n)
    out = np.ones(n.shape, dtype=float)
    it_ = np.nditer(n, flags=["multi_index"])
    for v in it_:
        v = int(v)
        r = 1.0
        while v > 1:
            r *= v
            v -= 2
        out[it_.multi_index] = r
    return out


def boys(m, T):
    """F_m(T) through Kummer's function (``boys_functions.py:63``)."""
    m = np.asarray(m, dtype=float)
    return hyp1f1(m + 0.5, m + 1.5, -np.asarray(T)) / (2.0 * m + 1.0)


def cart_components(l):
    """Default Cartesian order (``contractions.py:379-385``)."""
    return np.array([(x, y, l - x - y) for x in range(l, -1, -1) for y in range(l - x, -1, -1)])


def sph_components(l):
    """Default spherical order (``contractions.py:426-432``)."""
    if l == 1:
        return ("c1", "s1", "c0")
    return tuple([f"s{m}" for m in range(l, 0, -1)] + [f"c{m}" for m in range(l + 1)])


def _comp_norm(comps):
    return 1.0 / np.sqrt(np.prod(factorial2(2 * np.asarray(comps) - 1), axis=1))


def norm_cont(angmom, exps, coeffs, comps=None):
    """(self-overlap)^-1/2 per (segmented contraction, Cartesian component).

    Same quantity as ``contractions.py:503-524`` (which evaluates the overlap via
    ``overlap.py:55``); here the one-centre overlap is written in closed form:
    <g_p|g_q> = N_p N_q prod_i (2a_i-1)!! / (2 s)^{a_i} (pi/s)^{3/2}, s = a_p + a_q.
    Returns (M, L_cart).
    """
    if comps is None:
        comps = cart_components(angmom)
    comps = np.asarray(comps)
    exps = np.asarray(exps, dtype=float)
    coeffs = np.asarray(coeffs, dtype=float)
    if coeffs.ndim == 1:
        coeffs = coeffs[:, None]
    nprim = (2 * exps / np.pi) ** 0.75 * (4 * exps) ** (angmom / 2.0)
    s = exps[:, None] + exps[None, :]
    # the component factor prod (2a_i-1)!! of the moment cancels the 1/sqrt(df)
    # of both primitive norms, so every Cartesian component gets the same value
    base = (np.pi / s) ** 1.5 / (2 * s) ** angmom  # (K,K)
    out = np.empty((coeffs.shape[1], comps.shape[0]))
    for m in range(coeffs.shape[1]):
        cm = coeffs[:, m] * nprim
        out[m, :] = (cm @ base @ cm) ** -0.5
    return out


# ------------------------------------------------------------- spherical transform
def _shift(mag):
    return 0.5 if mag < 0 else 0.0


def _expansion_coeff(l, mag, i, j, k):
    # (``spherical.py:40-117``)
    am = abs(mag)
    val = (0.25) ** i * comb(l, i) * comb(l - i, am + i) * comb(i, j) * comb(am, 2 * k)
    expo = i + k - _shift(mag)
    if mag < 0:
        return float(np.real(complex(-1) ** expo)) * val
    return (-1) ** int(round(expo)) * val


def _harmonic_norm(l, mag):
    # (``spherical.py:120-163``)
    am = abs(mag)
    return (1.0 / (2 ** am * factorial(l))) * math.sqrt(
        2 * factorial(l + am) * factorial(l - am) / (2 ** int(mag == 0))
    )


def _solid_harmonic(l, mag):
    # (``spherical.py:166-225``)
    am = abs(mag)
    out = {}
    norm = _harmonic_norm(l, mag)
    for i in range((l - am) // 2 + 1):
        for j in range(i + 1):
            for kk in range(am // 2 + 1):
                k = kk + _shift(mag)
                c = _expansion_coeff(l, mag, i, j, k) * norm
                ax = int(2 * i + am - 2 * (j + k))
                ay = int(2 * (j + k))
                az = int(l - 2 * i - am)
                if c != 0:
                    out[(ax, ay, az)] = out.get((ax, ay, az), 0.0) + c
    return out


def generate_transformation(l, cart_order, sph_order):
    """(2l+1, L_cart) matrix applied from the left (``spherical.py:229-340``)."""
    cart_order = np.asarray(cart_order)
    index = {tuple(int(v) for v in c): n for n, c in enumerate(cart_order)}
    tr = np.zeros((cart_order.shape[0], 2 * l + 1))
    for col, name in enumerate(sph_order):
        sign = 1.0
        if name[0] == "-":
            sign, name = -1.0, name[1:]
        mag = -int(name[1:]) if name[0] == "s" else int(name[1:])
        for comp, c in _solid_harmonic(l, mag).items():
            tr[index[comp], col] = sign * c
    tr *= np.sqrt(np.prod(factorial2(2 * cart_order - 1), axis=1))[:, None]
    tr /= math.sqrt(float(factorial2(2 * l - 1)))
    return tr.T


# ------------------------------------------------------------------ quartet kernel
def _triples(l):
    return [(x, y, l - x - y) for x in range(l, -1, -1) for y in range(l - x, -1, -1)]


def _minus(t, i, n=1):
    u = list(t)
    u[i] -= n
    return tuple(u)


def _plus(t, i):
    u = list(t)
    u[i] += 1
    return tuple(u)


def _first_dir(t):
    for i in range(3):
        if t[i] > 0:
            return i
    raise ValueError


def quartet_cartesian(sa, sb, sc, sd, potential=(0, 0.0)):
    """Contracted Cartesian block (L_a, L_b, L_c, L_d, M_a, M_b, M_c, M_d).

    Mirrors the output of ``_compute_two_elec_integrals`` (``_two_elec_int.py:149-814``):
    primitive and Cartesian-component normalisation applied, ``norm_cont`` not applied,
    component order taken from each shell's ``angmom_components_cart``.  ``potential`` = (1,
    omega) or (2, omega) selects erf(omega r)/r or erfc(omega r)/r through the modified Boys
    values of ``boys_functions.py:145-223`` (the ``boys_func(orders, T, rho=...)`` call of
    ``_two_elec_int_improved.py:697``).
    """
    la, lb, lc, ld = sa.angmom, sb.angmom, sc.angmom, sd.angmom
    L = la + lb + lc + ld
    A, B, C, D = (np.asarray(s.coord, dtype=float) for s in (sa, sb, sc, sd))
    ea, eb, ec, ed = (np.asarray(s.exps, dtype=float) for s in (sa, sb, sc, sd))
    # flattened primitive-quartet axis, index order (a, b, c, d)
    a, b, c, d = (x.ravel() for x in np.meshgrid(ea, eb, ec, ed, indexing="ij"))
    zeta, eta = a + b, c + d
    rho = zeta * eta / (zeta + eta)
    P = (a[:, None] * A + b[:, None] * B) / zeta[:, None]
    Q = (c[:, None] * C + d[:, None] * D) / eta[:, None]
    PA, QC, PQ = P - A, Q - C, P - Q
    AB, CD = A - B, C - D
    T = rho * np.sum(PQ * PQ, axis=1)
    kab = np.exp(-a * b / zeta * np.dot(AB, AB))
    kcd = np.exp(-c * d / eta * np.dot(CD, CD))
    pref = 2.0 * np.pi ** 2.5 / (zeta * eta * np.sqrt(zeta + eta)) * kab * kcd
    F = boys(np.arange(L + 1)[:, None], T[None, :])  # (L+1, nprim)
    if potential[0]:
        w2 = float(potential[1]) ** 2
        att = w2 / (w2 + rho)
        Fa = att[None, :] ** (np.arange(L + 1)[:, None] + 0.5) * boys(np.arange(L + 1)[:, None],
                                                                     (att * T)[None, :])
        F = Fa if potential[0] == 1 else F - Fa
    WP = -(rho / zeta)[:, None] * PQ
    r_z = rho / zeta
    o2z = 0.5 / zeta

    # vertical recursion on A: V[e] has shape (L+1-|e|, nprim), rows are m
    V = {(0, 0, 0): pref[None, :] * F}
    for n in range(1, L + 1):
        for e in _triples(n):
            i = _first_dir(e)
            e1 = _minus(e, i)
            mm = L + 1 - n
            v = PA[:, i] * V[e1][:mm] + WP[:, i] * V[e1][1 : mm + 1]
            if e1[i] > 0:
                e2 = _minus(e1, i)
                v = v + e1[i] * o2z * (V[e2][:mm] - r_z * V[e2][1 : mm + 1])
            V[e] = v
    # electron transfer onto C, m = 0 only: E[(e,f)]
    E = {}
    for n in range(L + 1):
        for e in _triples(n):
            E[(e, (0, 0, 0))] = V[e][0]
    z_e = zeta / eta
    o2e = 0.5 / eta
    for nf in range(1, lc + ld + 1):
        for f in _triples(nf):
            i = _first_dir(f)
            f1 = _minus(f, i)
            for ne in range(0, L - nf + 1):
                for e in _triples(ne):
                    v = (QC[:, i] + z_e * PA[:, i]) * E[(e, f1)] - z_e * E[(_plus(e, i), f1)]
                    if e[i] > 0:
                        v = v + e[i] * o2e * E[(_minus(e, i), f1)]
                    if f1[i] > 0:
                        v = v + f1[i] * o2e * E[(e, _minus(f1, i))]
                    E[(e, f)] = v
    # contraction with normalised coefficients
    def ncoef(s, l):
        e = np.asarray(s.exps, dtype=float)
        cf = np.asarray(s.coeffs, dtype=float)
        if cf.ndim == 1:
            cf = cf[:, None]
        return cf * ((2 * e / np.pi) ** 0.75 * (4 * e) ** (l / 2.0))[:, None]

    ca, cb, cc, cd = ncoef(sa, la), ncoef(sb, lb), ncoef(sc, lc), ncoef(sd, ld)
    Ka, Kb, Kc, Kd = len(ea), len(eb), len(ec), len(ed)
    Ma, Mb, Mc, Md = ca.shape[1], cb.shape[1], cc.shape[1], cd.shape[1]
    G = {}
    for ne in range(la, la + lb + 1):
        for e in _triples(ne):
            for nf in range(lc, lc + ld + 1):
                for f in _triples(nf):
                    x = E[(e, f)].reshape(Ka, Kb, Kc, Kd)
                    G[(e, f)] = np.einsum("abcd,aw,bx,cy,dz->wxyz", x, ca, cb, cc, cd)
    # horizontal recursion on D: H[(e, c, d)]
    H = {}
    for ne in range(la, la + lb + 1):
        for e in _triples(ne):
            for nf in range(lc, lc + ld + 1):
                for f in _triples(nf):
                    H[(e, f, (0, 0, 0))] = G[(e, f)]
            for nd in range(1, ld + 1):
                for dd in _triples(nd):
                    i = _first_dir(dd)
                    d1 = _minus(dd, i)
                    for nc in range(lc, lc + ld - nd + 1):
                        for cc_ in _triples(nc):
                            H[(e, cc_, dd)] = H[(e, _plus(cc_, i), d1)] + CD[i] * H[(e, cc_, d1)]
    # horizontal recursion on B: R[(a, b, c, d)]
    comps = [np.asarray(s.angmom_components_cart) for s in (sa, sb, sc, sd)]
    out = np.empty((len(comps[0]), len(comps[1]), len(comps[2]), len(comps[3]), Ma, Mb, Mc, Md))
    for ic, cc_ in enumerate(comps[2]):
        for id_, dd in enumerate(comps[3]):
            cc_t, dd_t = tuple(int(v) for v in cc_), tuple(int(v) for v in dd)
            R = {}
            for ne in range(la, la + lb + 1):
                for e in _triples(ne):
                    R[(e, (0, 0, 0))] = H[(e, cc_t, dd_t)]
            for nb in range(1, lb + 1):
                for bb in _triples(nb):
                    i = _first_dir(bb)
                    b1 = _minus(bb, i)
                    for na in range(la, la + lb - nb + 1):
                        for aa in _triples(na):
                            R[(aa, bb)] = R[(_plus(aa, i), b1)] + AB[i] * R[(aa, b1)]
            for ia, aa in enumerate(comps[0]):
                for ib, bb in enumerate(comps[1]):
                    out[ia, ib, ic, id_] = R[(tuple(int(v) for v in aa), tuple(int(v) for v in bb))]
    for axis, cmp_ in enumerate(comps):
        shape = [1] * 8
        shape[axis] = -1
        out = out * _comp_norm(cmp_).reshape(shape)
    return out


def construct_array_contraction(sa, sb, sc, sd, reorder=False, potential=(0, 0.0)):
    """(M1, L1, M2, L2, M3, L3, M4, L4), chemist (``electron_repulsion.py:86-211``).

    ``reorder=True`` first swaps shells so that l_a >= l_b, l_c >= l_d and l_a >= l_c and
    un-swaps the axes afterwards, as gbasis's improved path does
    (``electron_repulsion.py:363-408``).  Same integrals; the recursions then run from the
    higher-l centres, which loses far fewer digits for diffuse high-l quartets.
    """
    if not reorder:
        return np.transpose(quartet_cartesian(sa, sb, sc, sd, potential), (4, 0, 5, 1, 6, 2, 7, 3))
    if reorder == "exponent":
        return _exponent_oriented(sa, sb, sc, sd, potential)
    bra_sw = sa.angmom < sb.angmom
    if bra_sw:
        sa, sb = sb, sa
    ket_sw = sc.angmom < sd.angmom
    if ket_sw:
        sc, sd = sd, sc
    bk_sw = sa.angmom < sc.angmom
    if bk_sw:
        sa, sb, sc, sd = sc, sd, sa, sb
    x = quartet_cartesian(sa, sb, sc, sd, potential)  # (La, Lb, Lc, Ld, Ma, Mb, Mc, Md)
    if bk_sw:
        x = np.transpose(x, (2, 3, 0, 1, 6, 7, 4, 5))
    if ket_sw:
        x = np.swapaxes(np.swapaxes(x, 2, 3), 6, 7)
    if bra_sw:
        x = np.swapaxes(np.swapaxes(x, 0, 1), 4, 5)
    return np.transpose(x, (4, 0, 5, 1, 6, 2, 7, 3))


def _pair_key(a, b):
    return (a + b, max(a, b), a)


def _exponent_oriented(sa, sb, sc, sd, potential=(0, 0.0)):
    """Same integrals with the recursions run from the shell of larger maximum exponent of
    each pair and the bra being the pair of larger (l_a + l_b, max l, l_a) — the recursion
    order of the B200 engine (``gbasis_b200/csrc/runtime.cu``)."""
    def tight_first(x, y):
        ex, ey = float(np.max(x.exps)), float(np.max(y.exps))
        return (ey > ex) or (ey == ex and y.angmom > x.angmom)

    perm = [0, 1, 2, 3]
    s = [sa, sb, sc, sd]
    if tight_first(s[0], s[1]):
        s[0], s[1] = s[1], s[0]
        perm[0], perm[1] = perm[1], perm[0]
    if tight_first(s[2], s[3]):
        s[2], s[3] = s[3], s[2]
        perm[2], perm[3] = perm[3], perm[2]
    if _pair_key(s[2].angmom, s[3].angmom) > _pair_key(s[0].angmom, s[1].angmom):
        s = s[2:] + s[:2]
        perm = perm[2:] + perm[:2]
    x = quartet_cartesian(*s, potential)  # axes in the order of s
    inv = list(np.argsort(perm))
    x = np.transpose(x, inv + [4 + v for v in inv])
    return np.transpose(x, (4, 0, 5, 1, 6, 2, 7, 3))


def construct_array_contraction_by_primitive(sa, sb, sc, sd):
    """(M1, L1, M2, L2, M3, L3, M4, L4) as ``construct_array_contraction``, summed primitive
    quartet by primitive quartet, each with its own recursion order: within each pair the
    recursions run from the primitive of larger exponent (``_exponent_oriented`` on one-
    primitive shells), and the horizontal recursion is applied per primitive quartet before
    the sum.  Same mathematics as the contracted form (the contraction is linear); it is the
    checker for heavily contracted shells whose primitives span tight and diffuse exponents,
    where a contracted recursion run from one fixed centre per pair (the reference's form,
    ``_two_elec_int.py:350-788``) loses up to about 1e-9 absolute: a primitive pair whose
    other primitive is the tighter one puts the product centre P near the other atom, and the
    vertical recursion then builds high angular momentum on a centre far from P."""
    def one(shell, k):
        cf = np.asarray(shell.coeffs, dtype=float).reshape(len(shell.exps), -1)
        return _PrimShell(shell, k, cf[k])
    out = 0.0
    for i in range(len(sa.exps)):
        for j in range(len(sb.exps)):
            for k in range(len(sc.exps)):
                for l in range(len(sd.exps)):
                    out = out + _exponent_oriented(one(sa, i), one(sb, j), one(sc, k), one(sd, l))
    return out


class _PrimShell:
    """Primitive k of a shell as a one-primitive shell (same centre, angular momentum,
    component orders and coefficient row)."""

    def __init__(self, shell, k, coef_row):
        self.coord = shell.coord
        self.angmom = shell.angmom
        self.exps = np.asarray([float(np.asarray(shell.exps)[k])])
        self.coeffs = np.asarray(coef_row, dtype=float).reshape(1, -1)
        self.angmom_components_cart = shell.angmom_components_cart


# --------------------------------------------------------------------- assembly
def _shell_matrix(shell, ctype):
    """Per-shell matrix mapping Cartesian block components to output functions,
    including norm_cont (``base_four_symm.py:195-205``) and, for spherical shells,
    the transformation (``base_four_symm.py:280-349``).  Shape (M*n_out, M*L_cart)."""
    nc = np.asarray(shell.norm_cont)  # (M, L)
    M, Lc = nc.shape
    if ctype == "spherical":
        t = generate_transformation(shell.angmom, shell.angmom_components_cart,
                                    shell.angmom_components_sph)
    else:
        t = np.eye(Lc)
    n_out = t.shape[0]
    W = np.zeros((M * n_out, M * Lc))
    for m in range(M):
        W[m * n_out:(m + 1) * n_out, m * Lc:(m + 1) * Lc] = t * nc[m][None, :]
    return W


def construct_array(basis, coord_types, quartet_fn=None, screen=None, reorder=False,
                    potential=(0, 0.0)):
    """Full 4-index array in chemist order for per-shell coordinate types.

    Restates ``construct_array_cartesian/spherical/mix`` (``base_four_symm.py:160-557``):
    loop over shell pairs from ``combinations_with_replacement`` and pair-of-pairs
    (i<=j, k<=l, pair index p <= q), scale by norm_cont, transform spherical shells,
    place the 8 symmetric copies.  ``screen(i,j,k,l)`` returning False zeroes a block
    (the improved path, ``electron_repulsion.py:341-361``).
    """
    if quartet_fn is None:
        quartet_fn = lambda a, b, c, d: construct_array_contraction(a, b, c, d, reorder,  # noqa: E731
                                                                    potential)
    Ws = [_shell_matrix(s, t) for s, t in zip(basis, coord_types)]
    sizes = [W.shape[0] for W in Ws]
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(int)
    N = int(off[-1])
    out = np.zeros((N, N, N, N))
    pairs = list(itertools.combinations_with_replacement(range(len(basis)), 2))
    for p, (i, j) in enumerate(pairs):
        for (k, l) in pairs[p:]:
            if screen is not None and not screen(i, j, k, l):
                blk = np.zeros((sizes[i], sizes[j], sizes[k], sizes[l]))
            else:
                raw = quartet_fn(basis[i], basis[j], basis[k], basis[l])
                s = raw.shape
                blk = raw.reshape(s[0] * s[1], s[2] * s[3], s[4] * s[5], s[6] * s[7])
                blk = np.einsum("pa,qb,rc,sd,abcd->pqrs", Ws[i], Ws[j], Ws[k], Ws[l], blk)
            si, sj, sk, sl = (slice(off[x], off[x + 1]) for x in (i, j, k, l))
            out[si, sj, sk, sl] = blk
            out[si, sj, sl, sk] = blk.transpose(0, 1, 3, 2)
            out[sj, si, sk, sl] = blk.transpose(1, 0, 2, 3)
            out[sj, si, sl, sk] = blk.transpose(1, 0, 3, 2)
            out[sk, sl, si, sj] = blk.transpose(2, 3, 0, 1)
            out[sl, sk, si, sj] = blk.transpose(3, 2, 0, 1)
            out[sk, sl, sj, si] = blk.transpose(2, 3, 1, 0)
            out[sl, sk, sj, si] = blk.transpose(3, 2, 1, 0)
    return out


def construct_array_lincomb(array, transform):
    """Four-index transform (``base_four_symm.py:559-616``)."""
    t = np.asarray(transform)
    return np.einsum("ia,jb,kc,ld,abcd->ijkl", t, t, t, t, array, optimize=True)


def _coord_types(basis):
    out = []
    for s in basis:
        ct = s.coord_type
        out.append({"c": "cartesian", "p": "spherical"}.get(ct, ct))
    return out


def electron_repulsion_integral(basis, transform=None, notation="physicist", reorder=False,
                                potential=(0, 0.0)):
    """``electron_repulsion.py:214-281``: dispatch, then physicist = transpose(0,2,1,3)."""
    if notation not in ("physicist", "chemist"):
        raise ValueError("`notation` must be one of 'physicist' or 'chemist'")
    arr = construct_array(list(basis), _coord_types(basis), reorder=reorder, potential=potential)
    if transform is not None:
        arr = construct_array_lincomb(arr, transform)
    if notation == "physicist":
        arr = np.transpose(arr, (0, 2, 1, 3))
    return arr


def schwarz_bounds(basis, reorder=True):
    """Q_ij = sqrt(max |(ij|ij)|) on blocks without norm_cont
    (``_schwarz_screening.py:14-90``)."""
    n = len(basis)
    Qm = np.zeros((n, n))
    for i in range(n):
        for j in range(i, n):
            blk = construct_array_contraction(basis[i], basis[j], basis[i], basis[j], reorder)
            Qm[i, j] = Qm[j, i] = math.sqrt(float(np.max(np.abs(blk))))
    return Qm


def electron_repulsion_integral_screened(basis, threshold, transform=None, notation="physicist",
                                        reorder=True):
    """Schwarz-zeroed variant (``electron_repulsion.py:415-504``,
    ``_schwarz_screening.py:169-191``): blocks with Q_ij Q_kl < threshold are zero."""
    if notation not in ("physicist", "chemist"):
        raise ValueError("`notation` must be one of 'physicist' or 'chemist'")
    screen = None
    if threshold > 0:
        Qm = schwarz_bounds(basis)
        screen = lambda i, j, k, l: Qm[i, j] * Qm[k, l] >= threshold  # noqa: E731
    arr = construct_array(list(basis), _coord_types(basis), screen=screen, reorder=reorder)
    if transform is not None:
        arr = construct_array_lincomb(arr, transform)
    if notation == "physicist":
        arr = np.transpose(arr, (0, 2, 1, 3))
    return arr
