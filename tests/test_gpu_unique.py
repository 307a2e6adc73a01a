"""Unique-integral form on the 20-atom chain (140 spherical s/p/d/f shells, N = 420):
sampled shell-quartet parity against the oracle through ``gbx_unique_values`` (all quartet
classes with an f shell represented), and the mixed form against the FP64 form over every
unique integral of the compact store (``gbx_compact_view``), bar 1e-10.
"""
import itertools

import numpy as np
import pytest

from gbasis_b200 import _engine
from gbasis_b200.electron_repulsion import MIXED_FP32, MIXED_SKIP
from gbasis_b200.synthetic import make_workload
from oracle import eri_oracle as orc

pytestmark = pytest.mark.gpu
ATOL = 1e-12


def _block_ref(shells, i, j, k, l):
    raw = orc.construct_array_contraction(shells[i], shells[j], shells[k], shells[l],
                                          reorder="exponent")
    s = raw.shape
    blk = raw.reshape(s[0] * s[1], s[2] * s[3], s[4] * s[5], s[6] * s[7])
    W = [orc._shell_matrix(shells[x], "spherical") for x in (i, j, k, l)]
    return np.einsum("pa,qb,rc,sd,abcd->pqrs", *W, blk)


def test_chain20_unique_sampled_parity_and_mixed_error():
    import torch
    shells = make_workload("chain20")
    db = _engine.DeviceBasis(shells)
    n = db.nbf
    assert n == 420
    db.unique()
    torch.cuda.synchronize()
    sizes = [2 * s.angmom + 1 for s in shells]
    off = np.concatenate([[0], np.cumsum(sizes)]).astype(int)
    rng = np.random.default_rng(7)
    by_l = {l: [i for i, s in enumerate(shells) if s.angmom == l] for l in range(4)}
    # every (l_i, l_j, l_k, l_l) pattern with an f shell once, plus random quartets
    quartets = []
    for ls in itertools.product(range(4), repeat=4):
        if 3 in ls and ls[0] >= ls[1] and ls[2] >= ls[3] and ls[:2] >= ls[2:]:
            quartets.append(tuple(int(rng.choice(by_l[x])) for x in ls))
    quartets += [tuple(int(v) for v in rng.integers(0, len(shells), 4)) for _ in range(12)]
    for (i, j, k, l) in quartets:
        ref = _block_ref(shells, i, j, k, l)
        ia, ib, ic, id_ = np.meshgrid(np.arange(off[i], off[i + 1]), np.arange(off[j], off[j + 1]),
                                      np.arange(off[k], off[k + 1]), np.arange(off[l], off[l + 1]),
                                      indexing="ij")
        idx = np.stack([ia.ravel(), ib.ravel(), ic.ravel(), id_.ravel()], axis=1)
        got = db.unique_values(idx).reshape(ref.shape)
        np.testing.assert_allclose(got, ref, rtol=0, atol=ATOL, err_msg=str((i, j, k, l)))

    ref_store = db.compact_view().clone()
    db.unique((MIXED_SKIP, MIXED_FP32))
    torch.cuda.synchronize()
    cur = db.compact_view()
    max_abs = 0.0
    for c0 in range(0, ref_store.numel(), 1 << 27):
        d = (cur[c0:c0 + (1 << 27)] - ref_store[c0:c0 + (1 << 27)]).abs()
        max_abs = max(max_abs, float(d.max()))
    print(f"chain20 mixed vs FP64 over {ref_store.numel()} stored integrals: max abs {max_abs:.3e}")
    assert max_abs <= 1e-10
    with pytest.raises(ValueError):
        db.unique_values([[0, 0, 0, n]])
    db.close()
