"""Seeded synthetic molecules for the five benchmark workloads.

No dataset is involved: every workload is a seeded random basis set with the shapes and
value distributions below, built with :class:`GeneralizedContractionShell`.

Shared distributions (per shell):
  * exponents a_k = a0 * beta**k, k = 0..K-1, a0 log-uniform in [0.1, 0.5], beta uniform
    in [2.5, 3.5];
  * contraction coefficients uniform in (0.1, 1), one segmented contraction (M = 1),
    normalised by the shell class as gbasis does.

Workloads:
  * ``tiny4``   — 4 atoms in a 6-bohr box (min separation 1.2), per atom s(3), s(1), p(3):
    12 shells, 20 Cartesian functions.  Seed 1.
  * ``medium8`` — 8 atoms in a 10-bohr box (min separation 1.2), per atom s(6), s(3), s(1),
    p(3), p(1), d(1): 48 shells, 120 Cartesian functions.  Seed 2.
  * ``chain20`` — 20-atom 3-D random walk (steps uniform 1.4-2.0 bohr, isotropic), per atom
    s(5), s(5), s(5), p(3), p(3), d(2), f(1), spherical: 140 shells, 420 functions.  Seed 3.
  * ``batch512`` — 512 molecules, molecule m seeded 4000+m: 2-14 atoms (uniform) in a box
    holding 54 bohr^3 per atom, 1-3 shells per atom drawn from {s, p, d} with K uniform in
    [1, 6], Cartesian.
  * ``large64`` — 64 atoms in a 20-bohr box, per atom s(8), s(4), s(2), s(1), p(3) x3,
    d(2) x2, f(1), spherical: 640 shells, 1920 functions.  Seed 5.
"""
from __future__ import annotations

import numpy as np

from .contractions import GeneralizedContractionShell

__all__ = ["random_shell", "box_atoms", "random_walk_atoms", "make_workload", "WORKLOADS",
           "batch_molecule", "density_matrix"]


def random_shell(rng, l, K, center, coord_type="cartesian"):
    a0 = float(np.exp(rng.uniform(np.log(0.1), np.log(0.5))))
    beta = float(rng.uniform(2.5, 3.5))
    exps = a0 * beta ** np.arange(K, dtype=float)
    coeffs = rng.uniform(0.1, 1.0, size=K)
    return GeneralizedContractionShell(int(l), np.asarray(center, dtype=float), coeffs, exps,
                                       coord_type)


def box_atoms(rng, n, box, min_sep=1.2, max_tries=100000):
    pts = []
    tries = 0
    while len(pts) < n:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("could not place atoms with the requested minimum separation")
        p = rng.uniform(0.0, box, size=3)
        if all(np.linalg.norm(p - q) >= min_sep for q in pts):
            pts.append(p)
    return np.array(pts)


def random_walk_atoms(rng, n, step_lo=1.4, step_hi=2.0):
    pts = [np.zeros(3)]
    while len(pts) < n:
        v = rng.normal(size=3)
        v /= np.linalg.norm(v)
        pts.append(pts[-1] + v * rng.uniform(step_lo, step_hi))
    return np.array(pts)


_PER_ATOM = {
    "tiny4": [(0, 3), (0, 1), (1, 3)],
    "medium8": [(0, 6), (0, 3), (0, 1), (1, 3), (1, 1), (2, 1)],
    "chain20": [(0, 5), (0, 5), (0, 5), (1, 3), (1, 3), (2, 2), (3, 1)],
    "large64": [(0, 8), (0, 4), (0, 2), (0, 1), (1, 3), (1, 3), (1, 3), (2, 2), (2, 2), (3, 1)],
}

WORKLOADS = ("tiny4", "medium8", "chain20", "batch512", "large64")


def make_workload(name):
    """Return the shell list of a named workload (``batch512`` returns a list of molecules)."""
    if name == "tiny4":
        rng = np.random.default_rng(1)
        atoms, ctype = box_atoms(rng, 4, 6.0), "cartesian"
    elif name == "medium8":
        rng = np.random.default_rng(2)
        atoms, ctype = box_atoms(rng, 8, 10.0), "cartesian"
    elif name == "chain20":
        rng = np.random.default_rng(3)
        atoms, ctype = random_walk_atoms(rng, 20), "spherical"
    elif name == "large64":
        rng = np.random.default_rng(5)
        atoms, ctype = box_atoms(rng, 64, 20.0), "spherical"
    elif name == "batch512":
        return [batch_molecule(m) for m in range(512)]
    else:
        raise ValueError(f"unknown workload {name!r}; expected one of {WORKLOADS}")
    shells = []
    for center in atoms:
        for l, K in _PER_ATOM[name]:
            shells.append(random_shell(rng, l, K, center, ctype))
    return shells


def batch_molecule(m, max_atoms=14):
    """Molecule ``m`` of the 512-molecule batch (seed 4000+m)."""
    rng = np.random.default_rng(4000 + m)
    n_atoms = int(rng.integers(2, max_atoms + 1))
    box = (54.0 * n_atoms) ** (1.0 / 3.0)
    atoms = box_atoms(rng, n_atoms, box)
    shells = []
    for center in atoms:
        n_sh = int(rng.integers(1, 4))
        for _ in range(n_sh):
            l = int(rng.integers(0, 3))
            K = int(rng.integers(1, 7))
            shells.append(random_shell(rng, l, K, center, "cartesian"))
    return shells


def density_matrix(n, seed=5):
    """Seeded symmetric positive-semidefinite D = X X^T / ||X X^T||, X in R^{n x n/4}."""
    rng = np.random.default_rng(seed)
    X = rng.normal(size=(n, max(1, n // 4)))
    D = X @ X.T
    return D / np.linalg.norm(D)
