"""CPU oracle for point-charge (nuclear-attraction) integrals — TEST INFRASTRUCTURE ONLY.

The checker the CUDA point-charge kernel is compared against: a NumPy restatement of gbasis's
algorithm for this integral.  Nothing in the product imports it; only ``tests/`` may call it.

Algorithm followed (reference file:line, paths inside the gbasis project):

* [0|0]^(m) = 2 pi / zeta  exp(-ab/zeta |AB|^2)  F_m(zeta |PC|^2)
  — ``gbasis/integrals/_one_elec_int.py:117-124``.
* Obara-Saika vertical recursion on centre A, axis by axis
  [a+1_i]^(m) = PA_i [a]^(m) - PC_i [a]^(m+1) + a_i/(2 zeta) ([a-1_i]^(m) - [a-1_i]^(m+1))
  — ``_one_elec_int.py:126-170``.
* Primitive norms (2a/pi)^{3/4} (4a)^{l/2} and contraction — ``_one_elec_int.py:172-183``.
* Horizontal recursion [a, b+1_i] = [a+1_i, b] + AB_i [a, b] — ``_one_elec_int.py:185-232``.
* Cartesian component norms 1/sqrt(prod (2a_i-1)!!) — ``_one_elec_int.py:240-252``.
* Scaling by -charge, output (M_1, L_1, M_2, L_2, N) — ``gbasis/integrals/point_charge.py:219-268``.
* norm_cont, spherical transform and symmetric placement (K, K, N)
  — ``gbasis/base_two_symm.py`` (construct_array_cartesian/spherical/mix/lincomb), and the
  dispatch of ``point_charge.py:271-325``; nuclear attraction sums over the points
  (``gbasis/integrals/nuclear_electron_attraction.py:8-42``).

Parity is pinned against ``tests/golden/point_charge.npz`` (reference outputs, generated by
``tests/golden/make_point_charge_golden.py``).
"""
from __future__ import annotations

import itertools

import numpy as np

from .eri_oracle import _coord_types, _shell_matrix, boys, factorial2


def pair_contraction(sa, sb, coords, charges):
    """(M_a, L_a, M_b, L_b, N) block of -q_c (a| 1/|r - C_c| |b), Cartesian, component norms
    included, no norm_cont (``point_charge.py:165-268``)."""
    coords = np.asarray(coords, dtype=float).reshape(-1, 3)
    charges = np.asarray(charges, dtype=float).ravel()
    la, lb = int(sa.angmom), int(sb.angmom)
    L = la + lb
    A, B = np.asarray(sa.coord, float), np.asarray(sb.coord, float)
    ea, eb = np.asarray(sa.exps, float).ravel(), np.asarray(sb.exps, float).ravel()
    ca = np.asarray(sa.coeffs, float)
    cb = np.asarray(sb.coeffs, float)
    ca = ca[:, None] if ca.ndim == 1 else ca
    cb = cb[:, None] if cb.ndim == 1 else cb
    npt = coords.shape[0]
    AB = A - B
    # V[m, ax, ay, az, point, prim_b, prim_a], as _one_elec_int.py:86-104 lays it out
    V = np.zeros((L + 1, L + 1, L + 1, L + 1, npt, eb.size, ea.size))
    a_ = ea[None, None, :]
    b_ = eb[None, :, None]
    z = a_ + b_
    P = (a_[..., None] * A + b_[..., None] * B) / z[..., None]     # (1, Kb, Ka, 3)
    PA = P - A
    PC = P - coords[:, None, None, :]                               # (N, Kb, Ka, 3)
    K = np.exp(-(a_ * b_ / z) * np.dot(AB, AB))
    T = z * np.sum(PC ** 2, axis=-1)                                # (N, Kb, Ka)
    m = np.arange(L + 1)[:, None, None, None]
    V[:, 0, 0, 0] = 2.0 * np.pi / z * K * boys(m, T[None])
    for ax in range(3):
        pa = PA[..., ax]                                            # (1, Kb, Ka)
        pc = PC[..., ax]                                            # (N, Kb, Ka)
        for n in range(L):                                          # [n] -> [n+1] along ax
            src = [slice(None)] * 4
            for mm in range(L - n):
                idx_n = _axis_index(ax, n)
                idx_n1 = _axis_index(ax, n + 1)
                val = pa * V[(mm,) + idx_n] - pc * V[(mm + 1,) + idx_n]
                if n > 0:
                    idx_m1 = _axis_index(ax, n - 1)
                    val = val + n / (2.0 * z) * (V[(mm,) + idx_m1] - V[(mm + 1,) + idx_m1])
                V[(mm,) + idx_n1] = val
            del src
    I0 = V[0]                                                       # (L+1)^3, N, Kb, Ka
    na = (2.0 * ea / np.pi) ** 0.75 * (4.0 * ea) ** (la / 2.0)
    nb = (2.0 * eb / np.pi) ** 0.75 * (4.0 * eb) ** (lb / 2.0)
    C = np.einsum("xyznba,a,am,b,bk->xyznmk", I0, na, ca, nb, cb)   # contracted
    # horizontal recursion: H[bx, by, bz][ax, ay, az] (a index up to L - |b|)
    H = {(0, 0, 0): C}
    for bt in _triples_upto(lb):
        if bt == (0, 0, 0):
            continue
        i = next(k for k in (2, 1, 0) if bt[k] > 0)
        prev = tuple(bt[k] - (k == i) for k in range(3))
        src = H[prev]
        out = np.zeros_like(src)
        sl_hi = [slice(None)] * 3
        sl_lo = [slice(None)] * 3
        sl_hi[i] = slice(1, None)
        sl_lo[i] = slice(0, -1)
        out[tuple(sl_lo)] = src[tuple(sl_hi)] + AB[i] * src[tuple(sl_lo)]
        H[bt] = out
    comps_a = np.asarray(sa.angmom_components_cart)
    comps_b = np.asarray(sb.angmom_components_cart)
    Ma, Mb = ca.shape[1], cb.shape[1]
    blk = np.zeros((Ma, len(comps_a), Mb, len(comps_b), npt))
    for ja, ta in enumerate(comps_a):
        na_c = 1.0 / np.sqrt(np.prod(factorial2(2 * np.asarray(ta) - 1)))
        for jb, tb in enumerate(comps_b):
            nb_c = 1.0 / np.sqrt(np.prod(factorial2(2 * np.asarray(tb) - 1)))
            v = H[tuple(int(x) for x in tb)][int(ta[0]), int(ta[1]), int(ta[2])]   # (N, Ma, Mb)
            blk[:, ja, :, jb, :] = np.transpose(v, (1, 2, 0)) * na_c * nb_c
    return -charges * blk


def _axis_index(ax, n):
    idx = [0, 0, 0]
    idx[ax] = n
    # earlier axes keep every value (slices); later axes are still zero
    out = []
    for k in range(3):
        if k < ax:
            out.append(slice(None))
        else:
            out.append(idx[k])
    return tuple(out)


def _triples_upto(l):
    """All (bx, by, bz) with sum <= l, ordered so that each one's predecessor comes first."""
    out = []
    for s in range(l + 1):
        for bx in range(s, -1, -1):
            for by in range(s - bx, -1, -1):
                out.append((bx, by, s - bx - by))
    return out


def point_charge_integral(basis, coords, charges, transform=None, coord_types=None):
    """(K, K, N) array (``point_charge.py:271-325``); ``transform`` as construct_array_lincomb."""
    basis = list(basis)
    cts = _coord_types(basis) if coord_types is None else list(coord_types)
    Ws = [_shell_matrix(s, t) for s, t in zip(basis, cts)]
    sizes = [W.shape[0] for W in Ws]
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(int)
    n = int(off[-1])
    npt = np.asarray(charges).size
    out = np.zeros((n, n, npt))
    for i, j in itertools.combinations_with_replacement(range(len(basis)), 2):
        raw = pair_contraction(basis[i], basis[j], coords, charges)
        s = raw.shape
        blk = np.einsum("pa,qb,abn->pqn", Ws[i], Ws[j], raw.reshape(s[0] * s[1], s[2] * s[3], s[4]))
        out[off[i]:off[i + 1], off[j]:off[j + 1]] = blk
        out[off[j]:off[j + 1], off[i]:off[i + 1]] = blk.transpose(1, 0, 2)
    if transform is not None:
        t = np.asarray(transform)
        out = np.einsum("ia,jb,abn->ijn", t, t, out)
    return out


def nuclear_electron_attraction_integral(basis, coords, charges, transform=None):
    """Sum over the points (``nuclear_electron_attraction.py:38-42``)."""
    return point_charge_integral(basis, coords, charges, transform).sum(axis=2)
