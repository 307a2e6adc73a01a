"""Mixed-precision form against the FP64 form (through the C ABI).

Bar: max absolute error <= 1e-10 on every element at the default thresholds (quartets whose
final-value Schwarz bound is below 1e-11 are zero, below the FP32 threshold their vertical and
transfer recursions run in FP32); max abs and rel errors are printed.
"""
import numpy as np
import pytest

from conftest import load_npz, shells_from_json
from gbasis_b200 import electron_repulsion as er
from gbasis_b200.synthetic import make_workload, random_shell, random_walk_atoms

pytestmark = pytest.mark.gpu


def chain_basis(n_atoms=4, seed=3):
    rng = np.random.default_rng(seed)
    atoms = random_walk_atoms(rng, n_atoms)
    shells = []
    for c in atoms:
        for l, K in [(0, 5), (0, 5), (1, 3), (2, 2), (3, 1)]:
            shells.append(random_shell(rng, l, K, c, "spherical"))
    return shells


@pytest.mark.parametrize("name", ["medium8_part", "chain_f", "mixed_fixture"])
def test_mixed_error_below_1e10(name):
    if name == "medium8_part":
        shells = make_workload("medium8")[:30]
    elif name == "chain_f":
        shells = chain_basis(6)
    else:
        shells = shells_from_json(load_npz("mixed.npz")["shells"])
    ref = er.electron_repulsion_integral(shells, notation="chemist")
    got = er.electron_repulsion_integral(shells, notation="chemist", precision="mixed")
    err = np.abs(got - ref)
    big = np.abs(ref) > 1e-8
    rel = (err[big] / np.abs(ref[big])).max() if big.any() else 0.0
    print(f"{name}: N={ref.shape[0]} max abs {err.max():.3e} max rel (|ref|>1e-8) {rel:.3e}")
    assert err.max() <= 1e-10
