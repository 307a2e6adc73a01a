"""Process-parallel CPU oracle over the unique shell quartets of a basis — TEST INFRASTRUCTURE ONLY.

The checker, not the product: only ``tests/`` and the CPU legs of ``bench.py`` use it.  It runs
``eri_oracle.construct_array_contraction`` (the NumPy restatement of gbasis's per-quartet
integrals, ``gbasis/integrals/electron_repulsion.py:86-211``) on unique shell quartets
(i <= j, k <= l, pair (i, j) <= pair (k, l): the loop of ``gbasis/base_four_symm.py:189-191``)
of a synthetic workload, split over spawned worker processes, and returns each quartet's
block of output functions: scaled by ``norm_cont`` (``base_four_symm.py:195-205``) and, for
spherical shells, transformed (``base_four_symm.py:280-349``).

Workers rebuild the basis from the workload name (the workloads are seeded), so only quartet
indices and finished blocks cross the process boundary.  The pool is always started with the
``spawn`` method, so it is safe after CUDA has been initialised in the parent.
"""
from __future__ import annotations

import itertools
import os
import time

import numpy as np

__all__ = ["unique_pairs", "quartet_count", "quartet_at", "unique_eri_count", "oracle_blocks",
           "SlicePool", "slice_quartets"]

_W = {}


def unique_pairs(n_shells):
    return list(itertools.combinations_with_replacement(range(n_shells), 2))


def quartet_count(n_shells):
    p = n_shells * (n_shells + 1) // 2
    return p * (p + 1) // 2


def quartet_at(pairs, idx):
    """Shell indices (i, j, k, l) of unique quartets given by their position in the
    reference's loop order (pair p, then every pair q >= p)."""
    npair = len(pairs)
    idx = np.asarray(idx, dtype=np.int64)
    r = np.arange(npair, dtype=np.int64)
    start = r * npair - r * (r - 1) // 2  # position of (p, p)
    p = np.searchsorted(start, idx, side="right") - 1
    q = p + (idx - start[p])
    pa = np.asarray(pairs, dtype=np.int64)
    return np.stack([pa[p, 0], pa[p, 1], pa[q, 0], pa[q, 1]], axis=1)


def _nfunc(shell):
    m = np.asarray(shell.coeffs).reshape(len(shell.exps), -1).shape[1]
    return len(shell.angmom_components_cart) * m


def unique_eri_count(shells, quartets):
    """Unique Cartesian function quadruples (8-fold symmetry) in the given shell quartets; over
    every unique quartet this is P(P+1)/2 with P = N(N+1)/2."""
    nf = np.array([_nfunc(s) for s in shells], dtype=np.int64)
    q = np.asarray(quartets, dtype=np.int64).reshape(-1, 4)
    i, j, k, l = q.T
    pij = np.where(i == j, nf[i] * (nf[i] + 1) // 2, nf[i] * nf[j])
    pkl = np.where(k == l, nf[k] * (nf[k] + 1) // 2, nf[k] * nf[l])
    same = (i == k) & (j == l)
    return int(np.sum(np.where(same, pij * (pij + 1) // 2, pij * pkl)))


def workload_shells(workload):
    """The shells of a named synthetic workload; ``"name:n"`` takes its first n shells and
    ``"batch512@m"`` is molecule m of the batch."""
    from gbasis_b200.synthetic import batch_molecule, make_workload
    if workload.startswith("batch512@"):
        return batch_molecule(int(workload.split("@", 1)[1]))
    name, _, n = workload.partition(":")
    shells = make_workload(name)
    return shells[: int(n)] if n else shells


def _init(workload, reorder):
    os.environ.setdefault("OMP_NUM_THREADS", "1")
    from oracle import eri_oracle as orc
    _W["shells"] = workload_shells(workload)
    _W["reorder"] = reorder
    _W["W"] = [orc._shell_matrix(s, t) for s, t in zip(_W["shells"], orc._coord_types(_W["shells"]))]


def _blocks(quartets):
    from oracle import eri_oracle as orc
    sh, reorder, W = _W["shells"], _W["reorder"], _W["W"]
    out = []
    for i, j, k, l in quartets:
        if reorder == "by_primitive":
            raw = orc.construct_array_contraction_by_primitive(sh[i], sh[j], sh[k], sh[l])
        else:
            raw = orc.construct_array_contraction(sh[i], sh[j], sh[k], sh[l], reorder=reorder)
        s = raw.shape
        blk = raw.reshape(s[0] * s[1], s[2] * s[3], s[4] * s[5], s[6] * s[7])
        out.append(np.einsum("pa,qb,rc,sd,abcd->pqrs", W[i], W[j], W[k], W[l], blk).ravel())
    return np.concatenate(out) if out else np.zeros(0)


def _timed(quartets):
    """Time of the per-quartet work of gbasis's Cartesian assembly loop: the contraction, then
    the four norm_cont scalings (``base_four_symm.py:189-205``)."""
    from oracle import eri_oracle as orc
    sh, reorder = _W["shells"], _W["reorder"]
    t = time.perf_counter()
    for q in quartets:
        blk = orc.construct_array_contraction(*(sh[x] for x in q), reorder=reorder)
        for ax, x in enumerate(q):
            nc = np.asarray(sh[x].norm_cont)
            shape = [1] * 8
            shape[2 * ax:2 * ax + 2] = nc.shape
            blk = blk * nc.reshape(shape)
    return time.perf_counter() - t


def _chunks(quartets, n):
    q = np.asarray(quartets)
    return [q[c:c + n] for c in range(0, len(q), n)]


def oracle_blocks(workload, quartets, processes=None, chunk=256, reorder="exponent"):
    """Flattened output-function blocks ([a][b][c][d] order) of ``quartets`` (rows of shell
    indices of the workload ``workload``), concatenated in the given order.  ``reorder``:
    ``"exponent"`` (the engine's recursion order), ``False`` (the reference's own order) or
    ``"by_primitive"`` (``construct_array_contraction_by_primitive``: each primitive quartet in
    its own order, the accurate checker for heavily contracted shells)."""
    import multiprocessing as mp
    processes = processes or os.cpu_count() or 1
    with mp.get_context("spawn").Pool(processes, initializer=_init,
                                      initargs=(workload, reorder)) as pool:
        parts = pool.map(_blocks, _chunks(quartets, chunk), chunksize=1)
    return np.concatenate(parts) if parts else np.zeros(0)


def slice_quartets(pairs, n_quartets, s, n_slices):
    """Slice ``s`` of ``n_slices``: the quartets whose loop position is congruent to s, so
    that every slice carries the workload's mix of classes."""
    return quartet_at(pairs, np.arange(s % n_slices, n_quartets, n_slices, dtype=np.int64))


class SlicePool:
    """Spawned workers that each hold the workload's basis and time the oracle on the quartets
    they are given (the CPU reference leg of ``bench.py``)."""

    def __init__(self, workload, processes=None, reorder=False):
        import multiprocessing as mp
        self.processes = processes or os.cpu_count() or 1
        self._pool = mp.get_context("spawn").Pool(self.processes, initializer=_init,
                                                  initargs=(workload, reorder))

    def run(self, quartets, chunk=32):
        """Wall time (s) of the oracle over all of ``quartets`` on the pool."""
        t = time.perf_counter()
        self._pool.map(_timed, _chunks(quartets, chunk), chunksize=1)
        return time.perf_counter() - t

    def close(self):
        self._pool.close()
        self._pool.join()
