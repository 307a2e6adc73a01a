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

    def run(self, outs, notation="chemist", stream=None):
        """Write molecule m's (N_m,)*4 float64 tensor to device buffer ``outs[m]`` (torch
        tensors or raw device pointers).  Asynchronous on ``stream``."""
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
        _engine.check(_engine.lib().gbx_batch_run(self.handle, code, ptrs, stream),
                      "gbx_batch_run")

    def close(self):
        if getattr(self, "handle", None):
            _engine.lib().gbx_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def electron_repulsion_integral_batch(molecules, notation="physicist", device=None):
    """ERI tensors of every molecule as device-resident torch tensors of shape (N_m,)*4;
    ``notation`` as in ``electron_repulsion_integral`` (physicist is the
    ``permute(0, 2, 1, 3)`` view of the chemist tensor)."""
    import torch
    if notation not in ["physicist", "chemist"]:
        raise ValueError("`notation` must be one of 'physicist' or 'chemist'")
    b = EriBatch(molecules, device=device)
    dev = torch.device("cuda", b.device)
    outs = [torch.empty((n,) * 4, dtype=torch.float64, device=dev) for n in b.nbf]
    b.run(outs, "chemist", stream=ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream))
    torch.cuda.current_stream(dev).synchronize()
    b.close()
    if notation == "physicist":
        outs = [o.permute(0, 2, 1, 3) for o in outs]
    return outs
