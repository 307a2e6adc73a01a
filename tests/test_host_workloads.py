"""The seeded synthetic workloads have the shapes and value distributions they are specified
with (atoms, shells, primitives, functions, shell quartets, unique integrals, exponent and
coefficient ranges, geometry).  No device needed."""
import itertools

import numpy as np
import pytest

from gbasis_b200 import _engine
from gbasis_b200.flops import unique_eris
from gbasis_b200.synthetic import batch_molecule, density_matrix, make_workload


def _centres(shells):
    return np.unique(np.round(np.array([s.coord for s in shells]), 12), axis=0)


def _nbf(shells):
    return int(_engine.pack_basis(shells)["nout"].sum())


def _quartets(n_shells):
    npair = n_shells * (n_shells + 1) // 2
    return npair * (npair + 1) // 2


def _check_shell_distributions(shells):
    for s in shells:
        e = np.asarray(s.exps)
        assert 0.1 <= e[0] <= 0.5
        if len(e) > 1:
            r = e[1:] / e[:-1]
            assert np.allclose(r, r[0]) and 2.5 <= r[0] <= 3.5
        c = np.asarray(s.coeffs)
        assert c.shape == (len(e), 1) and np.all((c > 0.1) & (c < 1.0))


def _min_sep(c):
    return min(np.linalg.norm(a - b) for a, b in itertools.combinations(c, 2))


@pytest.mark.parametrize("name, atoms, shells, nbf, per_atom_prims, ctype", [
    ("tiny4", 4, 12, 20, [3, 1, 3], "cartesian"),
    ("medium8", 8, 48, 120, [6, 3, 1, 3, 1, 1], "cartesian"),
    ("chain20", 20, 140, 420, [5, 5, 5, 3, 3, 2, 1], "spherical"),
    ("large64", 64, 640, 1920, [8, 4, 2, 1, 3, 3, 3, 2, 2, 1], "spherical"),
])
def test_named_workload_shapes(name, atoms, shells, nbf, per_atom_prims, ctype):
    sh = make_workload(name)
    assert len(sh) == shells
    c = _centres(sh)
    assert len(c) == atoms
    assert _nbf(sh) == nbf
    assert all(s.coord_type == ctype for s in sh)
    per = len(per_atom_prims)
    assert [len(s.exps) for s in sh] == per_atom_prims * atoms
    assert all(sh[i].coord is not None and np.allclose(sh[i].coord, sh[per * (i // per)].coord)
               for i in range(len(sh)))
    _check_shell_distributions(sh)
    if name == "chain20":
        steps = np.linalg.norm(np.diff(np.array([sh[per * a].coord for a in range(atoms)]),
                                       axis=0), axis=1)
        assert np.all((steps >= 1.4) & (steps <= 2.0))
    else:
        box = {"tiny4": 6.0, "medium8": 10.0, "large64": 20.0}[name]
        assert np.all((c >= 0.0) & (c <= box)) and _min_sep(c) >= 1.2


def test_quartet_and_unique_counts():
    assert _quartets(len(make_workload("tiny4"))) == 3081
    assert _quartets(len(make_workload("medium8"))) == 692076
    assert unique_eris(20) == 22155
    assert unique_eris(120) == 26357430


def test_batch_molecules():
    mols = [batch_molecule(m) for m in range(512)]
    for m in mols:
        c = _centres(m)
        assert 2 <= len(c) <= 14
        assert _min_sep(c) >= 1.2
        assert all(s.angmom in (0, 1, 2) and 1 <= len(s.exps) <= 6 for s in m)
        assert all(s.coord_type == "cartesian" for s in m)
        per_atom = [sum(np.allclose(s.coord, x) for s in m) for x in c]
        assert all(1 <= k <= 3 for k in per_atom)
        _check_shell_distributions(m)
    sizes = [len(_centres(m)) for m in mols]
    assert min(sizes) == 2 and max(sizes) == 14


def test_density_matrix_is_symmetric_psd():
    d = density_matrix(64)
    assert np.allclose(d, d.T)
    assert np.linalg.eigvalsh(d).min() > -1e-12
    assert np.isclose(np.linalg.norm(d), 1.0)
