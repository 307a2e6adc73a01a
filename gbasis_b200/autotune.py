"""Autotuner of the work decomposition: lanes per quartet ("team") per class block.

A class block holds every quartet of one (bra pair class, ket pair class); its register
kernel splits each quartet's primitive loop over `team` lanes (1..32) and sums the partial
[e0|f0] with warp shuffles.  Few primitives favour small teams (no reduction, more
quartets in flight); heavily contracted quartets favour large ones (parallel primitive
loop, balanced warps).  The tuner times every block for each candidate on the device (CUDA
events on the launching stream, one full call per candidate) and keeps the fastest.

Choices are stored in a JSON cache keyed by class and log2 of the block's mean primitive
quartets per shell quartet, so a new basis of similar shape starts tuned
(``DeviceBasis`` applies the cache on creation).
"""
from __future__ import annotations

import json
import math
import os

import numpy as np

from . import _engine

__all__ = ["autotune", "apply_cache", "cache_path", "TEAMS"]

TEAMS = (1, 2, 4, 8, 16, 32)


def cache_path():
    return os.environ.get("GBX_TUNE_CACHE",
                          os.path.join(os.path.dirname(os.path.abspath(__file__)), "tuning.json"))


def _key(cls4, avg_prims):
    return "%d%d%d%d:%d" % (*cls4, int(round(math.log2(max(avg_prims, 1.0)))))


def _load():
    try:
        with open(cache_path()) as f:
            return json.load(f)
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
    import torch
    db = _engine.DeviceBasis(shells, coord_types, device=device)
    n = db.nbf
    out = torch.empty(n ** 4, dtype=torch.float64, device=torch.device("cuda", db.device))
    db.set_profiling(2)
    blocks = db.blocks()
    times = np.full((len(teams), len(blocks)), np.inf)
    db.full_device(out.data_ptr())
    for ti, t in enumerate(teams):
        for k in range(len(blocks)):
            db.set_team(k, t)
        for _ in range(reps):
            db.full_device(out.data_ptr())
            times[ti] = np.minimum(times[ti], db.block_times())
    table = _load()
    chosen = {}
    for k, (cls4, _, avg, _) in enumerate(blocks):
        best = teams[int(np.argmin(times[:, k]))]
        db.set_team(k, best)
        chosen[_key(cls4, avg)] = best
    table.update(chosen)
    if save:
        with open(cache_path(), "w") as f:
            json.dump(table, f, indent=1, sort_keys=True)
    db.close()
    return chosen, times
