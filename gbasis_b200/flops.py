"""Algorithmic FLOP and byte model of the ERI path (the numerator of every roofline figure).

Per primitive quartet of canonical class (la, lb | lc, ld), la >= lb, lc >= ld,
(la, lb) >= (lc, ld), L = la + lb + lc + ld (FMA = 2 flops, no padding):

* Boys + prefactor: 30 + 3L;
* VRR: sum_{e=1..L} ncart(e) (L - e + 1) (4 if e == 1 else 8);
* ETR: sum_{f=1..lc+ld} ncart(f) sum_{e=la..L-f} ncart(e) * 8;
* contraction: 2 * #[e0|f0] with e in [la, la+lb], f in [lc, lc+ld].

Per contracted quartet: HRR = 2 flops per element produced (ket, then bra).  (ss|ss) has no
HRR.  Unique contracted ERIs = P(P+1)/2 with P = N(N+1)/2.  Bytes of the full tensor:
8 N^4 written.
"""
from __future__ import annotations

import itertools
from functools import lru_cache

__all__ = ["prim_flops", "hrr_flops", "basis_flops", "unique_eris", "canonical"]


def ncart(l):
    return (l + 1) * (l + 2) // 2


def canonical(la, lb, lc, ld):
    a, b = max(la, lb), min(la, lb)
    c, d = max(lc, ld), min(lc, ld)
    if (a, b) < (c, d):
        a, b, c, d = c, d, a, b
    return a, b, c, d


@lru_cache(maxsize=None)
def prim_flops(la, lb, lc, ld):
    L = la + lb + lc + ld
    f = 30 + 3 * L
    for e in range(1, L + 1):
        f += ncart(e) * (L - e + 1) * (4 if e == 1 else 8)
    for ff in range(1, lc + ld + 1):
        f += ncart(ff) * sum(ncart(e) for e in range(la, L - ff + 1)) * 8
    ne = sum(ncart(e) for e in range(la, la + lb + 1))
    nf = sum(ncart(e) for e in range(lc, lc + ld + 1))
    return f + 2 * ne * nf


@lru_cache(maxsize=None)
def hrr_flops(la, lb, lc, ld):
    if la + lb + lc + ld == 0:
        return 0
    ne = sum(ncart(e) for e in range(la, la + lb + 1))
    k = sum(ncart(c) * ncart(dd) for dd in range(1, ld + 1) for c in range(lc, lc + ld - dd + 1))
    b = sum(ncart(a) * ncart(bb) for bb in range(1, lb + 1) for a in range(la, la + lb - bb + 1))
    return 2 * (k * ne + b * ncart(lc) * ncart(ld))


def basis_flops(shells):
    """Algorithmic FLOPs of one full-tensor call over the unique shell quartets of ``shells``
    (each segmented contraction counted as its own shell, as the engine computes them)."""
    seg = []
    for s in shells:
        m = s.coeffs.shape[1] if getattr(s.coeffs, "ndim", 1) == 2 else 1
        seg += [(int(s.angmom), len(s.exps))] * m
    pairs = list(itertools.combinations_with_replacement(range(len(seg)), 2))
    # group pairs by (la, lb, K) to count quartets per class without an O(P^2) loop
    from collections import Counter
    pc = Counter()
    for i, j in pairs:
        (li, ki), (lj, kj) = seg[i], seg[j]
        pc[(max(li, lj), min(li, lj), ki * kj)] += 1
    keys = sorted(pc)
    total = 0
    for x, kx in enumerate(keys):
        for y in range(x, len(keys)):
            ky = keys[y]
            nq = pc[kx] * pc[ky] if x != y else pc[kx] * (pc[kx] + 1) // 2
            a, b, c, d = canonical(kx[0], kx[1], ky[0], ky[1])
            total += nq * (kx[2] * ky[2] * prim_flops(a, b, c, d) + hrr_flops(a, b, c, d))
    return total


def unique_eris(n):
    p = n * (n + 1) // 2
    return p * (p + 1) // 2
