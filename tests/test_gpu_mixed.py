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


def test_left_out_quartets_zeroed_in_a_dirty_store():
    """The mixed form writes zeros for its left-out quartets itself (no clearing of the whole
    compact store): with every store entry set to NaN before the call, the expanded tensor has
    no NaN, matches the FP64 tensor at the mixed bar, and the quartet counts add up."""
    import torch
    from gbasis_b200 import _engine
    from gbasis_b200.electron_repulsion import MIXED_FP32, MIXED_SKIP
    shells = make_workload("large64")[:40]  # 4 atoms of the 20-bohr box: many left out
    db = _engine.DeviceBasis(shells)
    n = db.nbf
    ref = torch.empty(n ** 4, dtype=torch.float64, device="cuda")
    db.full_device(ref.data_ptr())
    torch.cuda.synchronize()
    n64_ref, n32_ref, left_ref = db.mixed_counts()
    assert n32_ref == 0 and left_ref == 0 and n64_ref == db.stats()[0]
    got = torch.empty_like(ref)
    db.set_fp32_lists(1, 1 << 30)  # every block's FP32 quartets get their own launch here
    for _ in range(2):  # the second call reuses the zero list
        db.compact_view().fill_(float("nan"))
        got.fill_(float("nan"))
        db.full_device(got.data_ptr(), mixed=(MIXED_SKIP, MIXED_FP32))
        torch.cuda.synchronize()
        n64, n32, left = db.mixed_counts()
        print(f"N={n}: quartets FP64 {n64} FP32 {n32} left out {left}")
        assert left > 0 and n32 > 0
        assert n64 + n32 + left == db.stats()[0]
        assert not torch.isnan(got).any()
        assert float((got - ref).abs().max()) <= 1e-10
    db.close()
