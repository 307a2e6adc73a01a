"""Drop-in for ``gbasis.integrals.point_charge`` and ``nuclear_electron_attraction`` on the GPU.

* :func:`point_charge_integral` (``gbasis/integrals/point_charge.py:271-325``): (K, K, N) array
  of -q_c (a| 1/|r - R_c| |b) for the N point charges;
* :func:`nuclear_electron_attraction_integral`
  (``gbasis/integrals/nuclear_electron_attraction.py:8-42``): its sum over the points, (K, K).

Same arguments, layouts and errors as the reference (``point_charge.py:165-218`` checks); each
shell's ``coord_type`` (or the keyword-only ``coord_type``) selects Cartesian or spherical
functions, ``transform`` gives the linear-combination form.  Computed by
``gbx_point_charge`` (one thread per shell pair and point charge); there is no CPU path.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _engine
from .base import check_shell_list

__all__ = ["point_charge_integral", "nuclear_electron_attraction_integral"]


def _check_points(points_coords, points_charge):
    # gbasis/integrals/point_charge.py:180-218
    if not (isinstance(points_coords, np.ndarray) and points_coords.ndim == 2
            and points_coords.shape[1] == 3 and points_coords.dtype in [int, float]):
        raise TypeError("`points_coords` must be a two-dimensional `numpy` array of `dtype` "
                        "int/float with three columns.")
    if not (isinstance(points_charge, np.ndarray) and points_charge.ndim == 1
            and points_charge.dtype in [int, float]):
        raise TypeError("`points_charge` must be a one-dimensional `numpy` array of integers or "
                        "floats.")
    if points_coords.shape[0] != points_charge.size:
        raise ValueError("`points_coords` must have the same number of rows as there are elements "
                         "in `points_charge`.")


def _run(basis, points_coords, points_charge, sum_points, coord_type, device):
    import torch
    check_shell_list(basis)
    _check_points(points_coords, points_charge)
    types = None
    if coord_type is not None:
        types = [coord_type] * len(basis) if isinstance(coord_type, str) else list(coord_type)
    db = _engine.DeviceBasis(list(basis), types, device=device)
    try:
        n, npt = db.nbf, int(points_charge.size)
        coords = np.ascontiguousarray(points_coords, dtype=np.float64)
        charges = np.ascontiguousarray(points_charge, dtype=np.float64)
        dev = torch.device("cuda", db.device)
        shape = (n, n) if sum_points else (n, n, npt)
        out = torch.empty(shape, dtype=torch.float64, device=dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        _engine.check(_engine.lib().gbx_point_charge(
            db.handle, npt, _engine._ptr(coords), _engine._ptr(charges), 1 if sum_points else 0,
            ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream)), "gbx_point_charge")
        return out.cpu().numpy()
    finally:
        db.close()


def point_charge_integral(basis, points_coords, points_charge, transform=None, *,
                          coord_type=None, device=None):
    """(K, K, N) point-charge interaction integrals; with ``transform`` (K', K) the
    linear-combination form T V T^T per point (``base_two_symm.py`` construct_array_lincomb)."""
    arr = _run(basis, points_coords, points_charge, False, coord_type, device)
    if transform is not None:
        t = np.asarray(transform)
        arr = np.einsum("ia,jb,abn->ijn", t, t, arr)
    return arr


def nuclear_electron_attraction_integral(basis, nuclear_coords, nuclear_charges, transform=None,
                                         *, coord_type=None, device=None):
    """(K, K) sum over the nuclei of the point-charge integrals."""
    arr = _run(basis, nuclear_coords, nuclear_charges, True, coord_type, device)
    if transform is not None:
        t = np.asarray(transform)
        arr = t @ arr @ t.T
    return arr
