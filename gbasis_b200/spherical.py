"""Cartesian -> real-solid-harmonic transformation, host side.

Same conventions as ``gbasis/spherical.py:10-340`` (expansion coefficients, harmonic
normalisation, component normalisation sqrt((2a_x-1)!!(2a_y-1)!!(2a_z-1)!!)/sqrt((2l-1)!!),
labels ``c{m}``/``s{m}`` with an optional leading ``-`` for a sign flip).  The engine bakes
the default-order matrices into its kernels as constants (see ``csrc/gen_eri.py``) and
applies custom orders, signs and ``norm_cont`` as a per-function permutation and scale.
"""
from __future__ import annotations

import math
from fractions import Fraction

import numpy as np

__all__ = ["solid_harmonic", "generate_transformation", "engine_sph_matrix",
           "canonical_sph_labels"]


def _dfact(n):
    r = 1
    while n > 1:
        r *= n
        n -= 2
    return r


def _comb(n, k):
    if k < 0 or k > n or n < 0:
        return 0
    return math.comb(n, k)


def _harmonic_norm(l, m):
    am = abs(m)
    return math.sqrt(2 * math.factorial(l + am) * math.factorial(l - am) / (2 ** int(m == 0))) \
        / (2 ** am * math.factorial(l))


def solid_harmonic(l, m):
    """Coefficients {(ax, ay, az): c} of the real regular solid harmonic C_l^m (m >= 0) or
    S_l^|m| (m < 0), normalised as gbasis's ``real_solid_harmonic``."""
    am = abs(m)
    shift = Fraction(1, 2) if m < 0 else Fraction(0)
    norm = _harmonic_norm(l, m)
    out = {}
    for t in range((l - am) // 2 + 1):
        for u in range(t + 1):
            for v2 in range(am // 2 + 1):
                v = v2 + shift
                # (-1)^(t + v - shift) is real: t + v2 is an integer
                sign = -1 if (t + v2) % 2 else 1
                c = sign * (0.25 ** t) * _comb(l, t) * _comb(l - t, am + t) * _comb(t, u) \
                    * _comb(am, int(2 * v))
                if c == 0:
                    continue
                ax = int(2 * t + am - 2 * (u + v))
                ay = int(2 * (u + v))
                az = l - 2 * t - am
                out[(ax, ay, az)] = out.get((ax, ay, az), 0.0) + c * norm
    return out


def _parse_label(label):
    sign = 1.0
    if label[0] == "-":
        sign, label = -1.0, label[1:]
    m = int(label[1:])
    return sign, (-m if label[0] == "s" else m)


def generate_transformation(angmom, cartesian_order, spherical_order, apply_from="left"):
    """Transformation matrix with gbasis's signature and layout
    ((2l+1, L_cart) for ``apply_from='left'``)."""
    cart = np.asarray(cartesian_order)
    index = {tuple(int(v) for v in c): n for n, c in enumerate(cart)}
    tr = np.zeros((cart.shape[0], 2 * angmom + 1))
    for col, label in enumerate(spherical_order):
        sign, m = _parse_label(label)
        for comp, c in solid_harmonic(angmom, m).items():
            tr[index[comp], col] = sign * c
    df = np.array([_dfact(2 * a - 1) * _dfact(2 * b - 1) * _dfact(2 * c - 1) for a, b, c in cart])
    tr *= np.sqrt(df)[:, None]
    tr /= math.sqrt(_dfact(2 * angmom - 1))
    return tr.T if apply_from == "left" else tr


def canonical_sph_labels(l):
    """Engine-internal spherical order: s_l..s_1, c_0..c_l (gbasis's default for l != 1)."""
    return [f"s{m}" for m in range(l, 0, -1)] + [f"c{m}" for m in range(l + 1)]


def engine_sph_matrix(l):
    """(2l+1, L_cart) matrix from *unnormalised-component* Cartesian integrals (canonical
    order) to normalised spherical ones (canonical labels): the solid-harmonic coefficient
    divided by sqrt((2l-1)!!).  The component norms of gbasis's transform cancel against
    the Cartesian component normalisation of the block, so they do not appear."""
    from .contractions import default_cart_components
    cart = [tuple(int(v) for v in c) for c in default_cart_components(l)]
    K = np.zeros((2 * l + 1, len(cart)))
    for u, label in enumerate(canonical_sph_labels(l)):
        _, m = _parse_label(label)
        for comp, c in solid_harmonic(l, m).items():
            K[u, cart.index(comp)] = c
    return K / math.sqrt(_dfact(2 * l - 1))
