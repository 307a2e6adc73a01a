"""The 8-atom, 120-function workload (1.66 GB tensor) against the oracle at 1e-12 absolute.

* every one of the engine's class blocks (bra pair class x ket pair class, pairs oriented with
  the larger-exponent shell first as the engine stores them) is sampled: at least 20 shell
  quartets from each, all of them where a block has fewer;
* the whole tensor: every one of the 692,076 unique shell quartets through the oracle, split
  over spawned host processes, compared block by block with the engine's tensor.
"""
import os

import numpy as np
import pytest

from gbasis_b200 import electron_repulsion as er
from gbasis_b200 import _engine
from gbasis_b200.synthetic import make_workload
from oracle import parallel as opar

pytestmark = pytest.mark.gpu
ATOL = 1e-12
# pair classes (l of the larger-exponent shell, l of the other) in the engine's order
PAIR_CLASSES = [(0, 0), (0, 1), (1, 0), (1, 1), (0, 2), (2, 0), (1, 2), (2, 1),
                (0, 3), (3, 0), (2, 2), (1, 3), (3, 1), (2, 3), (3, 2), (3, 3)]


def _pair_class(shells, i, j):
    ei, ej = max(shells[i].exps), max(shells[j].exps)
    a, b = i, j
    if ej > ei or (ej == ei and shells[j].angmom > shells[i].angmom):
        a, b = j, i
    return PAIR_CLASSES.index((shells[a].angmom, shells[b].angmom))


def _quartet_blocks(shells, quartets):
    pairs = opar.unique_pairs(len(shells))
    pidx = {p: n for n, p in enumerate(pairs)}
    cls = np.array([_pair_class(shells, i, j) for i, j in pairs])
    q = np.asarray(quartets)
    cp = cls[[pidx[(i, j)] for i, j in q[:, :2]]]
    cq = cls[[pidx[(k, l)] for k, l in q[:, 2:]]]
    return np.maximum(cp, cq) * len(PAIR_CLASSES) + np.minimum(cp, cq)


def _engine_values(T, shells, quartets):
    """The engine tensor's blocks of ``quartets``, flattened and concatenated in order (the
    layout of ``oracle.parallel.oracle_blocks``)."""
    nf = np.array([len(s.angmom_components_cart) for s in shells])
    off = np.concatenate([[0], np.cumsum(nf)])
    n = T.shape[0]
    flat = T.reshape(-1)
    q = np.asarray(quartets)
    sizes = nf[q].prod(axis=1)
    start = np.concatenate([[0], np.cumsum(sizes)])
    out = np.empty(int(start[-1]))
    dims = nf[q]
    keys = dims @ np.array([1000, 100, 10, 1])
    for key in np.unique(keys):
        sel = np.nonzero(keys == key)[0]
        a, b, c, d = dims[sel[0]]
        o = off[q[sel]]
        ia = (o[:, 0, None] + np.arange(a))[:, :, None, None, None]
        ib = (o[:, 1, None] + np.arange(b))[:, None, :, None, None]
        ic = (o[:, 2, None] + np.arange(c))[:, None, None, :, None]
        id_ = (o[:, 3, None] + np.arange(d))[:, None, None, None, :]
        vals = flat[((ia * n + ib) * n + ic) * n + id_].reshape(len(sel), -1)
        dst = start[sel, None] + np.arange(a * b * c * d)
        out[dst] = vals
    return out


@pytest.fixture(scope="module")
def medium8():
    shells = make_workload("medium8")
    T = er.electron_repulsion_integral(shells, notation="chemist")
    assert T.shape == (120,) * 4
    return shells, T


def test_medium8_every_class_block_sampled(medium8):
    shells, T = medium8
    pairs = opar.unique_pairs(len(shells))
    nq = opar.quartet_count(len(shells))
    allq = opar.quartet_at(pairs, np.arange(nq))
    blk = _quartet_blocks(shells, allq)
    db = _engine.DeviceBasis(shells)
    n_engine_blocks = len(db.blocks())
    db.close()
    assert len(np.unique(blk)) == n_engine_blocks == 45
    rng = np.random.default_rng(8)
    pick = []
    for b in np.unique(blk):
        members = np.nonzero(blk == b)[0]
        pick.extend(rng.choice(members, size=min(20, len(members)), replace=False))
    q = allq[np.sort(np.array(pick))]
    ref = opar.oracle_blocks("medium8", q, processes=min(os.cpu_count() or 1, 16), chunk=16)
    got = _engine_values(T, shells, q)
    err = np.abs(got - ref)
    assert err.max() <= ATOL, float(err.max())


def test_medium8_whole_tensor_against_oracle(medium8):
    shells, T = medium8
    pairs = opar.unique_pairs(len(shells))
    allq = opar.quartet_at(pairs, np.arange(opar.quartet_count(len(shells))))
    assert len(allq) == 692076
    ref = opar.oracle_blocks("medium8", allq, chunk=512)
    got = _engine_values(T, shells, allq)
    assert got.shape == ref.shape
    err = np.abs(got - ref)
    assert err.max() <= ATOL, float(err.max())
