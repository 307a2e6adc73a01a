"""Full ERI tensors of many molecules in one device pass (``gbx_batch_*``).

gbasis computes one basis per ``electron_repulsion_integral`` call
(``gbasis/integrals/electron_repulsion.py:214-281``); a batch of molecules is a Python loop of
such calls.  :class:`EriBatch` packs all molecules once, and every :meth:`EriBatch.run`
replays one CUDA graph: one class kernel per block type for the whole batch, then one batched
expansion that writes each molecule's tensor (same values, layout and notation as
``electron_repulsion_integral`` of that molecule alone).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _engine

__all__ = ["EriBatch", "electron_repulsion_integral_batch"]


class EriBatch:
    """Molecules (lists of shells) resident on one CUDA device."""

    def __init__(self, molecules, device=None, graph=True):
        L = _engine.lib()
        if device is None:
            device = _engine._current_device()
        packs = [_engine.pack_basis(list(m)) for m in molecules]
        if not packs:
            raise ValueError("At least one molecule must be given.")
        cat = {k: np.ascontiguousarray(np.concatenate([p[k] for p in packs]))
               for k in ("angmom", "nprim", "center", "exps", "coefs", "nout", "sph", "pos", "scl")}
        nsh = np.array([len(p["angmom"]) for p in packs], dtype=np.int32)
        h = ctypes.c_void_p()
        P = _engine._ptr
        _engine.check(L.gbx_batch_create(
            ctypes.byref(h), len(packs), P(nsh), P(cat["angmom"]), P(cat["nprim"]),
            P(cat["center"]), P(cat["exps"]), P(cat["coefs"]), P(cat["nout"]), P(cat["sph"]),
            P(cat["pos"]), P(cat["scl"]), int(device)), "gbx_batch_create")
        self.handle, self.device, self.n_mol = h, int(device), len(packs)
        nbf = np.zeros(self.n_mol, dtype=np.int64)
        q, cb = ctypes.c_int64(), ctypes.c_int64()
        _engine.check(L.gbx_batch_info(h, P(nbf), ctypes.byref(q), ctypes.byref(cb)))
        self.nbf = [int(v) for v in nbf]
        self.n_quartets, self.compact_bytes = int(q.value), int(cb.value)
        if not graph:
            _engine.check(L.gbx_batch_set_graph(h, 0))
        self.apply_tuning()

    # ------------------------------------------------------------------ autotuner
    def types(self):
        """[(class (la, lb, lc, ld), team, mean primitive quartets, quartets)] per block type."""
        L = _engine.lib()
        n = ctypes.c_int()
        _engine.check(L.gbx_batch_num_types(self.handle, ctypes.byref(n)))
        out = []
        for k in range(n.value):
            c4 = np.zeros(4, dtype=np.int32)
            t, ap, nq = ctypes.c_int(), ctypes.c_double(), ctypes.c_int64()
            _engine.check(L.gbx_batch_type_info(self.handle, k, _engine._ptr(c4), ctypes.byref(t),
                                                ctypes.byref(ap), ctypes.byref(nq)))
            out.append((tuple(int(v) for v in c4), t.value, ap.value, nq.value))
        return out

    def set_team(self, k, team):
        _engine.check(_engine.lib().gbx_batch_set_team(self.handle, int(k), int(team)),
                      "gbx_batch_set_team")

    def set_queue(self, on=True):
        """True: FP64 runs evaluate every block type in ONE persistent launch that drains a
        single multi-class work queue (``gbx_batch_set_queue``); False: one class kernel per
        block type (the default)."""
        _engine.check(_engine.lib().gbx_batch_set_queue(self.handle, 1 if on else 0),
                      "gbx_batch_set_queue")

    def apply_tuning(self, table=None):
        """Teams from the tuning cache (keyed by class and primitive bucket, shared with the
        single-basis tuner); returns how many types changed."""
        from .autotune import _key, _load
        table = _load() if table is None else table
        n = 0
        for k, (cls4, team, avg, _) in enumerate(self.types()):
            key = _key(cls4, avg)
            t = table.get(key)
            if t and t != team:
                self.set_team(k, int(t))
                n += 1
            v, c = table.get("v:" + key), table.get("c:" + key)
            if v is not None or c is not None:
                self.set_type_config(k, int(v or 0), int(c or 8))
                n += 1
        return n

    def set_type_config(self, k, variant=0, ctas_per_sm=8):
        _engine.check(_engine.lib().gbx_batch_set_type_config(self.handle, int(k), int(variant),
                                                              int(ctas_per_sm)),
                      "gbx_batch_set_type_config")

    def autotune(self, outs, teams=None, reps=2, save=True, stream=None):
        """Time every block type with each value of its knobs (types run one after another,
        CUDA events per type): the team of the register-kernel types, then the kernel variant
        of the heavy types, then the grid cap of the register-kernel types; keep the fastest
        and store the choices in the tuning cache."""
        import json
        from .autotune import CTAS, TEAMS, _key, _load, cache_path, light_class
        teams = TEAMS if teams is None else teams
        L = _engine.lib()
        types = self.types()
        keys = [_key(c4, avg) for c4, _, avg, _ in types]
        light = [k for k, (c4, _, _, _) in enumerate(types) if light_class(c4)]
        heavy = [k for k in range(len(types)) if k not in light]
        var = {k: 0 for k in range(len(types))}
        cap = {k: 8 for k in range(len(types))}

        def sweep(ks, values, setter):
            times = np.full((len(values), len(types)), np.inf)
            for vi, v in enumerate(values):
                for k in ks:
                    setter(k, v)
                for _ in range(reps):
                    self.run(outs, stream=stream)
                    ms = np.zeros(len(types))
                    _engine.check(L.gbx_batch_type_times(self.handle, _engine._ptr(ms), len(ms)))
                    times[vi] = np.minimum(times[vi], ms)
            return times

        def set_var(k, v):
            var[k] = v
            self.set_type_config(k, v, cap[k])

        def set_cap(k, c):
            cap[k] = c
            self.set_type_config(k, var[k], c)
        chosen = {}
        _engine.check(L.gbx_batch_set_profiling(self.handle, 1))
        try:
            times = sweep(light, teams, self.set_team)
            for k in light:
                best = teams[int(np.argmin(times[:, k]))]
                self.set_team(k, best)
                chosen[keys[k]] = best
            t_var = sweep(heavy, (0, 1), set_var)
            for k in heavy:
                set_var(k, int(np.argmin(t_var[:, k])))
                chosen["v:" + keys[k]] = var[k]
            t_cap = sweep(light, CTAS, set_cap)
            for k in light:
                set_cap(k, CTAS[int(np.argmin(t_cap[:, k]))])
                chosen["c:" + keys[k]] = cap[k]
        finally:
            _engine.check(L.gbx_batch_set_profiling(self.handle, 0))
        times = {"team": times, "variant": t_var, "ctas_per_sm": t_cap}
        if save:
            table = _load()
            table.update(chosen)
            with open(cache_path(), "w") as f:
                json.dump(table, f, indent=1, sort_keys=True)
        return chosen, times

    def run(self, outs, notation="chemist", stream=None, mixed=None):
        """Write molecule m's (N_m,)*4 float64 tensor to device buffer ``outs[m]`` (torch
        tensors or raw device pointers).  Asynchronous on ``stream``.

        ``mixed=(skip, fp32)`` runs the mixed-precision form: quartets whose final-value bound
        is below ``skip`` are zero, those below ``fp32`` (light classes) run their recursions
        in FP32.  Its first run computes the batch's bounds (synchronously)."""
        if notation not in ("physicist", "chemist"):
            raise ValueError("`notation` must be one of 'physicist' or 'chemist'")
        if len(outs) != self.n_mol:
            raise ValueError(f"expected {self.n_mol} outputs")
        ptrs = (ctypes.c_void_p * self.n_mol)()
        for m, o in enumerate(outs):
            if hasattr(o, "data_ptr"):
                if o.numel() != self.nbf[m] ** 4 or not o.is_contiguous():
                    raise ValueError(f"output {m} must be a contiguous tensor of "
                                     f"{self.nbf[m] ** 4} float64 values")
                ptrs[m] = o.data_ptr()
            else:
                ptrs[m] = int(o)
        code = _engine.GBX_PHYSICIST if notation == "physicist" else _engine.GBX_CHEMIST
        if mixed is None:
            _engine.check(_engine.lib().gbx_batch_run(self.handle, code, ptrs, stream),
                          "gbx_batch_run")
        else:
            _engine.check(_engine.lib().gbx_batch_run_mixed(
                self.handle, code, float(mixed[0]), float(mixed[1]), ptrs, stream),
                "gbx_batch_run_mixed")

    def mixed_counts(self):
        """(FP64, FP32, left-out) quartets of the last mixed-form lists."""
        v = [ctypes.c_int64() for _ in range(3)]
        _engine.check(_engine.lib().gbx_batch_mixed_counts(self.handle, *map(ctypes.byref, v)),
                      "gbx_batch_mixed_counts")
        return tuple(int(x.value) for x in v)

    def close(self):
        if getattr(self, "handle", None):
            _engine.lib().gbx_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def electron_repulsion_integral_batch(molecules, notation="physicist", device=None,
                                      precision="fp64", mixed_skip=None, mixed_fp32=None):
    """ERI tensors of every molecule as device-resident torch tensors of shape (N_m,)*4;
    ``notation`` as in ``electron_repulsion_integral`` (physicist is the
    ``permute(0, 2, 1, 3)`` view of the chemist tensor).  ``precision="mixed"`` selects the
    mixed form with the thresholds of ``electron_repulsion_integral``."""
    import torch
    from .electron_repulsion import MIXED_FP32, MIXED_SKIP
    if notation not in ["physicist", "chemist"]:
        raise ValueError("`notation` must be one of 'physicist' or 'chemist'")
    if precision not in ("fp64", "mixed"):
        raise ValueError("`precision` must be 'fp64' or 'mixed'")
    mixed = None
    if precision == "mixed":
        mixed = (MIXED_SKIP if mixed_skip is None else float(mixed_skip),
                 MIXED_FP32 if mixed_fp32 is None else float(mixed_fp32))
    b = EriBatch(molecules, device=device)
    dev = torch.device("cuda", b.device)
    outs = [torch.empty((n,) * 4, dtype=torch.float64, device=dev) for n in b.nbf]
    b.run(outs, "chemist", stream=ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream),
          mixed=mixed)
    torch.cuda.current_stream(dev).synchronize()
    b.close()
    if notation == "physicist":
        outs = [o.permute(0, 2, 1, 3) for o in outs]
    return outs
