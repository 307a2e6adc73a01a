"""Coulomb and exchange matrices on the GPU.

``coulomb_matrix``: direct J_ab = sum_cd (ab|cd) D_cd.
The ERI tensor is never stored: screened unique shell quartets (Schwarz bound
Q_ab Q_cd >= ``schwarz_threshold``, bounds on blocks without ``norm_cont`` as gbasis's
``SchwarzScreener`` uses, ``gbasis/integrals/_schwarz_screening.py:14-191``) are evaluated
in chunks and contracted with D as they are produced (``gbx_eri_coulomb_j``).  gbasis has no
direct counterpart; it is the contraction users apply to ``electron_repulsion_integral``'s
chemist tensor, ``einsum("abcd,cd->ab", eri, D)``.

``coulomb_exchange``: J and K_ac = sum_bd (ab|cd) D_bd (``einsum("abcd,bd->ac", eri, D)``) of
any square density, from the unique integrals of the screened quartets (``gbx_eri_jk``): each
row of the unique-integral matrix yields one J element pair and 2N exchange terms, so the N^4
tensor is never formed (the N^4/8 unique values are).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _engine

__all__ = ["coulomb_matrix", "coulomb_exchange"]


def coulomb_matrix(basis, density, schwarz_threshold=1e-12, coord_type=None, device=None,
                   precision="fp64", mixed_thresholds=None):
    """J (K, K) float64 for the symmetric density ``density`` (K, K) in the basis's
    functions (coordinate types from the shells unless ``coord_type`` overrides them).

    ``precision="mixed"``: quartets are classified by the bound of their final values
    instead of ``schwarz_threshold``: below ``skip`` left out, below ``fp32`` FP32 recursions
    (light classes), else FP64; ``mixed_thresholds=(skip, fp32)`` defaults to the mixed
    full-tensor form's thresholds."""
    import torch
    if precision not in ("fp64", "mixed"):
        raise ValueError("`precision` must be 'fp64' or 'mixed'")
    types = None
    if coord_type is not None:
        types = [coord_type] * len(basis) if isinstance(coord_type, str) else list(coord_type)
    db = _engine.DeviceBasis(list(basis), types, device=device)
    try:
        n = db.nbf
        D = np.ascontiguousarray(density, dtype=np.float64)
        if D.shape != (n, n):
            raise ValueError(f"`density` must have shape ({n}, {n})")
        dev = torch.device("cuda", db.device)
        d_D = torch.from_numpy(D).to(dev)
        d_J = torch.empty((n, n), dtype=torch.float64, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        if precision == "mixed":
            from .electron_repulsion import MIXED_FP32, MIXED_SKIP
            skip, fp32 = mixed_thresholds or (MIXED_SKIP, MIXED_FP32)
            _engine.check(_engine.lib().gbx_eri_coulomb_j_mixed(
                db.handle, ctypes.c_void_p(d_D.data_ptr()), float(skip), float(fp32),
                ctypes.c_void_p(d_J.data_ptr()), ctypes.c_void_p(stream)),
                "gbx_eri_coulomb_j_mixed")
        else:
            _engine.check(_engine.lib().gbx_eri_coulomb_j(
                db.handle, ctypes.c_void_p(d_D.data_ptr()), float(schwarz_threshold),
                ctypes.c_void_p(d_J.data_ptr()), ctypes.c_void_p(stream)), "gbx_eri_coulomb_j")
        return d_J.cpu().numpy()
    finally:
        db.close()


def coulomb_exchange(basis, density, schwarz_threshold=0.0, coord_type=None, device=None):
    """(J, K), each (K, K) float64, for the density ``density`` (K, K; need not be symmetric)
    in the basis's functions: J_ab = sum_cd (ab|cd) D_cd and K_ac = sum_bd (ab|cd) D_bd."""
    import torch
    types = None
    if coord_type is not None:
        types = [coord_type] * len(basis) if isinstance(coord_type, str) else list(coord_type)
    db = _engine.DeviceBasis(list(basis), types, device=device)
    try:
        n = db.nbf
        D = np.ascontiguousarray(density, dtype=np.float64)
        if D.shape != (n, n):
            raise ValueError(f"`density` must have shape ({n}, {n})")
        dev = torch.device("cuda", db.device)
        d_D = torch.from_numpy(D).to(dev)
        d_J = torch.empty((n, n), dtype=torch.float64, device=dev)
        d_K = torch.empty((n, n), dtype=torch.float64, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        _engine.check(_engine.lib().gbx_eri_jk(
            db.handle, ctypes.c_void_p(d_D.data_ptr()), float(schwarz_threshold),
            ctypes.c_void_p(d_J.data_ptr()), ctypes.c_void_p(d_K.data_ptr()),
            ctypes.c_void_p(stream)), "gbx_eri_jk")
        return d_J.cpu().numpy(), d_K.cpu().numpy()
    finally:
        db.close()
