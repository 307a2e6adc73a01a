"""Autotuner of the work decomposition: lanes per quartet ("team") per class block.

A class block holds every quartet of one (bra pair class, ket pair class); its register
kernel splits each quartet's primitive loop over `team` lanes (1..32) and sums the partial
[e0|f0] with warp shuffles.  Few primitives favour small teams (no reduction, more
quartets in flight); heavily contracted quartets favour large ones (parallel primitive
loop, balanced warps).  The tuner times every register-kernel block for each candidate on
the device (CUDA events on the launching stream, one unique-integral call per candidate, the
blocks run one after another) and keeps the fastest; ``EriBatch.autotune`` does the same for
the block types of a batch.

Choices are stored in a JSON cache keyed by class and log2 of the block's mean primitive
quartets per shell quartet, so a new basis or batch of similar shape starts tuned
(``DeviceBasis`` and ``EriBatch`` apply the cache on creation).
"""
from __future__ import annotations

import json
import math
import os

import numpy as np

from . import _engine

__all__ = ["autotune", "apply_cache", "cache_path", "TEAMS"]

TEAMS = (1, 2, 4, 8, 16, 32)


def light_class(cls4):
    """Classes run by the register kernel (the only ones whose team matters): the [e0|f0]
    accumulators and the (ab|cd) block of one quartet fit one thread (170 doubles, the limit
    the kernel generator uses)."""
    def nc(l):
        return (l + 1) * (l + 2) // 2
    la, lb, lc, ld = cls4
    ne = sum(nc(e) for e in range(la, la + lb + 1))
    nf = sum(nc(f) for f in range(lc, lc + ld + 1))
    return ne * nf + nc(la) * nc(lb) * nc(lc) * nc(ld) <= 170


def cache_path():
    return os.environ.get("GBX_TUNE_CACHE",
                          os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning.json"))


def _key(cls4, avg_prims):
    return "%d%d%d%d:%d" % (*cls4, int(round(math.log2(max(avg_prims, 1.0)))))


_loaded = {}  # path -> (modification time, table): read once per change of the file


def _load():
    path = cache_path()
    try:
        mtime = os.stat(path).st_mtime_ns
        hit = _loaded.get(path)
        if hit and hit[0] == mtime:
            return dict(hit[1])
        with open(path) as f:
            table = json.load(f)
        _loaded[path] = (mtime, table)
        return dict(table)
    except (OSError, ValueError):
        return {}


def apply_cache(db, table=None):
    """Set the team of every block whose (class, primitive bucket) the cache knows."""
    table = _load() if table is None else table
    n = 0
    for k, (cls4, team, avg, _) in enumerate(db.blocks()):
        t = table.get(_key(cls4, avg))
        if t and t != team:
            db.set_team(k, int(t))
            n += 1
    return n


def autotune(shells, coord_types=None, reps=3, teams=TEAMS, save=True, device=None):
    """Tune the teams of ``shells``'s class blocks; returns {key: team} and the timings."""
    # the unique-integral call runs the same class kernels without the N^4 tensor
    db = _engine.DeviceBasis(shells, coord_types, device=device)
    db.set_profiling(2)
    blocks = db.blocks()
    light = [k for k, (cls4, _, _, _) in enumerate(blocks) if light_class(cls4)]
    times = np.full((len(teams), len(blocks)), np.inf)
    db.unique()
    for ti, t in enumerate(teams):
        for k in light:
            db.set_team(k, t)
        for _ in range(reps):
            db.unique()
            times[ti] = np.minimum(times[ti], db.block_times())
    table = _load()
    chosen = {}
    for k in light:
        cls4, _, avg, _ = blocks[k]
        best = teams[int(np.argmin(times[:, k]))]
        db.set_team(k, best)
        chosen[_key(cls4, avg)] = best
    table.update(chosen)
    if save:
        with open(cache_path(), "w") as f:
            json.dump(table, f, indent=1, sort_keys=True)
    db.close()
    return chosen, times
