"""Autotuner of the work decomposition of the class kernels.

Knobs, each chosen by timing on the device (CUDA events on the launching stream):

* ``team`` — lanes per quartet of the register kernel (light classes): each quartet's
  primitive loop is split over `team` lanes (1..32) and the partial [e0|f0] summed with warp
  shuffles.  Few primitives favour small teams, heavily contracted quartets large ones.
* ``variant`` — heavy classes that have both kernels: the split register kernel (0) or the
  line-factorised kernel (1).
* ``ctas_per_sm`` — the register kernel's grid cap, in resident CTAs per SM (2..16): more
  CTAs shorten the tail of a block, fewer stage the Boys table fewer times.
* ``streams`` — how many concurrent streams the class blocks of a call are spread over
  (class-block grouping: blocks go round robin, largest first, to that many streams).

Per-block knobs are timed with the blocks run one after another (``set_profiling(2)``); the
stream count is timed on whole unique-integral calls.  ``EriBatch.autotune`` does the same for
the block types of a batch.  Choices are stored in a JSON cache keyed by class and log2 of
the block's mean primitive quartets per shell quartet (team: ``"abcd:k"``, variant:
``"v:abcd:k"``, grid cap: ``"c:abcd:k"``; stream count: ``"streams"``), so a new basis or
batch of similar shape starts tuned (``DeviceBasis`` and ``EriBatch`` apply the cache on
creation).  gbasis has no counterpart: it evaluates one quartet at a time in NumPy.
"""
from __future__ import annotations

import json
import math
import os

import numpy as np

from . import _engine

__all__ = ["autotune", "apply_cache", "cache_path", "TEAMS", "CTAS", "STREAMS"]

TEAMS = (1, 2, 4, 8, 16, 32)
CTAS = (2, 4, 8, 16)
STREAMS = (1, 2, 4, 6, 8, 12, 16)


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
    """Set the knobs of every block whose (class, primitive bucket) the cache knows, and the
    stream count; returns how many blocks changed."""
    table = _load() if table is None else table
    n = 0
    for k, (cls4, team, avg, _) in enumerate(db.blocks()):
        key = _key(cls4, avg)
        t = table.get(key)
        if t and t != team:
            db.set_team(k, int(t))
            n += 1
        v, c = table.get("v:" + key), table.get("c:" + key)
        if v is not None or c is not None:
            db.set_block_config(k, int(v or 0), int(c or 8))
            n += 1
    if table.get("streams"):
        db.set_streams(int(table["streams"]))
    return n


def _call_ms(db, reps):
    import torch
    st = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = float("inf")
    for _ in range(reps):
        e0.record(st)
        db.unique(stream=__import__("ctypes").c_void_p(st.cuda_stream))
        e1.record(st)
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    return best


def _sweep(db, blocks, ks, values, setter, reps):
    """Per-block times (values x blocks) of each value of one knob, blocks run in order."""
    times = np.full((len(values), len(blocks)), np.inf)
    for vi, v in enumerate(values):
        for k in ks:
            setter(k, v)
        for _ in range(reps):
            db.unique()
            times[vi] = np.minimum(times[vi], db.block_times())
    return times


def autotune(shells, coord_types=None, reps=3, teams=TEAMS, ctas=CTAS, streams=STREAMS,
             save=True, device=None):
    """Tune the knobs of ``shells``'s class blocks (team, variant, grid cap) and the stream
    count, one knob after another with the earlier choices in place; returns the chosen
    {key: value} and the per-knob timings."""
    # the unique-integral call runs the same class kernels without the N^4 tensor
    db = _engine.DeviceBasis(shells, coord_types, device=device, tuned=False)
    db.set_profiling(2)
    blocks = db.blocks()
    keys = [_key(c4, avg) for c4, _, avg, _ in blocks]
    light = [k for k, (cls4, _, _, _) in enumerate(blocks) if light_class(cls4)]
    heavy = [k for k in range(len(blocks)) if k not in light]
    db.unique()
    chosen, timings = {}, {}
    # lanes per quartet (light classes)
    t_team = _sweep(db, blocks, light, teams, db.set_team, reps)
    for k in light:
        best = teams[int(np.argmin(t_team[:, k]))]
        db.set_team(k, best)
        chosen[keys[k]] = best
    timings["team"] = t_team
    # kernel variant (heavy classes) and grid cap (light classes), keeping the other default
    var = {k: 0 for k in range(len(blocks))}
    cap = {k: 8 for k in range(len(blocks))}

    def set_var(k, v):
        var[k] = v
        db.set_block_config(k, v, cap[k])

    def set_cap(k, c):
        cap[k] = c
        db.set_block_config(k, var[k], c)
    t_var = _sweep(db, blocks, heavy, (0, 1), set_var, reps)
    for k in heavy:
        set_var(k, int(np.argmin(t_var[:, k])))
        chosen["v:" + keys[k]] = var[k]
    timings["variant"] = t_var
    t_cap = _sweep(db, blocks, light, ctas, set_cap, reps)
    for k in light:
        set_cap(k, ctas[int(np.argmin(t_cap[:, k]))])
        chosen["c:" + keys[k]] = cap[k]
    timings["ctas_per_sm"] = t_cap
    # stream count, on whole calls with the blocks concurrent
    db.set_profiling(0)
    t_st = []
    for n in streams:
        db.set_streams(n)
        db.unique()
        t_st.append(_call_ms(db, reps))
    chosen["streams"] = streams[int(np.argmin(t_st))]
    db.set_streams(chosen["streams"])
    timings["streams"] = np.array(t_st)
    if save:
        table = _load()
        table.update(chosen)
        with open(cache_path(), "w") as f:
            json.dump(table, f, indent=1, sort_keys=True)
    db.close()
    return chosen, timings


def main(argv):
    """``python -m gbasis_b200.autotune medium8 chain20 batch512``: tune the named synthetic
    workloads in order (the stream count of the last single-basis workload wins; the batch keeps
    the single-basis stream count) and store the choices in the cache."""
    import torch
    from .synthetic import make_workload
    for name in argv:
        if name == "batch512":
            from .batch import EriBatch
            b = EriBatch(make_workload("batch512"))
            outs = [torch.empty((n,) * 4, dtype=torch.float64, device="cuda") for n in b.nbf]
            chosen, _ = b.autotune(outs)
            b.close()
        else:
            keep = _load().get("streams")
            chosen, _ = autotune(make_workload(name))
            if keep is not None and name != argv[0]:
                # the first single-basis workload sets the stream count
                table = _load()
                table["streams"] = keep
                with open(cache_path(), "w") as f:
                    json.dump(table, f, indent=1, sort_keys=True)
        print(name, json.dumps(chosen, sort_keys=True), flush=True)


if __name__ == "__main__":
    import sys
    main(sys.argv[1:])
