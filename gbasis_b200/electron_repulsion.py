"""Drop-in for ``gbasis.integrals.electron_repulsion`` backed by the B200 engine.

Same entry points, arguments, array layouts and errors as the reference:

* :func:`electron_repulsion_integral` (``gbasis/integrals/electron_repulsion.py:214-281``);
* :class:`ElectronRepulsionIntegral` with ``construct_array_contraction`` (classmethod,
  ``:86-211``) and ``construct_array_{cartesian,spherical,mix,lincomb}``
  (``gbasis/base_four_symm.py:160-616``);
* :func:`electron_repulsion_integral_improved` with ``schwarz_threshold``
  (``electron_repulsion.py:415-504``).

Every array is computed on the GPU by ``libgbx_eri.so`` through its C ABI; there is no CPU
path (a missing library or device raises).  The chemist-order tensor is produced
contiguously and the physicist result is the reference's ``transpose(0, 2, 1, 3)`` view.
Extras are keyword-only: ``coord_type`` (overrides every shell's ``coord_type``),
``device`` and ``out`` (a preallocated C-contiguous float64 array, e.g. page-locked).
"""
from __future__ import annotations

import numpy as np

from . import _engine
from .base_four_symm import BaseFourIndexSymmetric, register_with_gbasis
from .contractions import is_shell

__all__ = ["ElectronRepulsionIntegral", "ElectronRepulsionIntegralImproved",
           "electron_repulsion_integral", "electron_repulsion_integral_improved"]


def _boys_host(orders, weighted_dist, rho=None):
    """F_m(T) = 1F1(m+1/2; m+3/2; -T)/(2m+1) on the host.  Kept as the ``boys_func`` class
    attribute for API compatibility (``electron_repulsion.py:84``); the device engine uses its
    own tabulated Boys function and does not call this."""
    from scipy.special import hyp1f1
    orders = np.asarray(orders)
    return hyp1f1(orders + 0.5, orders + 1.5, -np.asarray(weighted_dist)) / (2 * orders + 1)


def _norm_types(coord_types, n):
    if not isinstance(coord_types, (list, tuple)):
        raise TypeError("`coord_types` must be a list or a tuple.")
    if not all(i in ["cartesian", "spherical"] for i in coord_types):
        raise ValueError("Each entry of `coord_types` must be one of 'cartesian' or 'spherical'.")
    if len(coord_types) != n:
        raise ValueError("`coord_types` must have the same number of entries as the number of "
                         "`GeneralizedContractionShell` in the instance.")
    return list(coord_types)


class ElectronRepulsionIntegral(BaseFourIndexSymmetric):
    """Electron-repulsion integrals of a basis, chemist notation (``(ab|cd)``); a
    ``BaseFourIndexSymmetric`` as in gbasis (``gbasis/integrals/electron_repulsion.py:20``)."""

    boys_func = staticmethod(_boys_host)
    _screen = 0.0
    _mixed = None  # (skip, fp32) thresholds of the mixed-precision form
    _potential = (0, 0.0)  # two-electron operator (code, omega), see potential_code

    def __init__(self, contractions):
        # argument checks and messages of gbasis/base.py:32-65
        super().__init__(contractions)

    # ------------------------------------------------------------------ per quartet
    @classmethod
    def construct_array_contraction(cls, cont_one, cont_two, cont_three, cont_four):
        """(M1, L1, M2, L2, M3, L3, M4, L4) block of four shells, Cartesian, primitive and
        component norms applied, ``norm_cont`` not applied (``electron_repulsion.py:86-211``).
        Computed on the device as a batch of one."""
        for name, c in (("cont_one", cont_one), ("cont_two", cont_two),
                        ("cont_three", cont_three), ("cont_four", cont_four)):
            if not is_shell(c):
                raise TypeError(f"`{name}` must be a `GeneralizedContractionShell` instance.")
        shells = [cont_one, cont_two, cont_three, cont_four]
        db = _engine.DeviceBasis(shells, raw=True)
        full = db.full_host("chemist")
        db.close()
        dims = []
        for s in shells:
            c = np.asarray(s.coeffs)
            dims.append((c.shape[1] if c.ndim == 2 else 1, len(s.angmom_components_cart)))
        off = np.cumsum([0] + [m * l for m, l in dims])
        blk = full[off[0]:off[1], off[1]:off[2], off[2]:off[3], off[3]:off[4]]
        return np.ascontiguousarray(blk).reshape(
            dims[0][0], dims[0][1], dims[1][0], dims[1][1], dims[2][0], dims[2][1],
            dims[3][0], dims[3][1])

    # ---------------------------------------------------------------- whole basis
    def _full(self, coord_types, out=None, device=None):
        db = _engine.DeviceBasis(list(self.contractions), coord_types, device=device)
        try:
            if self._potential[0]:
                db.set_potential(*self._potential)
            if self._mixed is None:
                return db.full_host("chemist", self._screen, out=out)
            import ctypes
            import torch
            n = db.nbf
            dev = torch.device("cuda", db.device)
            buf = torch.empty(n ** 4, dtype=torch.float64, device=dev)
            stream = torch.cuda.current_stream(dev).cuda_stream
            db.full_device(buf.data_ptr(), "chemist", stream=ctypes.c_void_p(stream),
                           mixed=self._mixed)
            if out is None:
                return buf.cpu().numpy().reshape(n, n, n, n)
            torch.from_numpy(out.reshape(-1)).copy_(buf)
            return out
        finally:
            db.close()

    def construct_array_cartesian(self, out=None, device=None):
        return self._full(["cartesian"] * len(self.contractions), out, device)

    def construct_array_spherical(self, out=None, device=None):
        return self._full(["spherical"] * len(self.contractions), out, device)

    def construct_array_mix(self, coord_types, out=None, device=None):
        return self._full(_norm_types(coord_types, len(self.contractions)), out, device)

    def construct_array_lincomb(self, transform, coord_type, device=None):
        """``base_four_symm.py:559-616``: ERI tensor in the given coordinate types, then the
        four-index transform on the device (cuBLAS DGEMM chain)."""
        if all(ct == "cartesian" for ct in coord_type):
            types = ["cartesian"] * len(self.contractions)
        elif all(ct == "spherical" for ct in coord_type):
            types = ["spherical"] * len(self.contractions)
        elif isinstance(coord_type, (list, tuple)):
            types = _norm_types(coord_type, len(self.contractions))
        else:
            raise TypeError("`coord_type` must be a list/tuple of the strings 'cartesian' or "
                            "'spherical'")
        return _lincomb_device(list(self.contractions), types, np.asarray(transform, dtype=float),
                               self._screen, device, self._potential)


class ElectronRepulsionIntegralImproved(ElectronRepulsionIntegral):
    """Same integrals; ``schwarz_threshold`` zeroes quartets with Q_ij Q_kl below it."""

    def __init__(self, contractions, schwarz_threshold=0.0):
        super().__init__(contractions)
        self._screen = float(schwarz_threshold)

    @classmethod
    def construct_array_contraction(cls, cont_one, cont_two, cont_three, cont_four, **kwargs):
        """As :meth:`ElectronRepulsionIntegral.construct_array_contraction`, with the screening
        hook of ``electron_repulsion.py:306-360``: given ``screener`` (an object with
        ``is_significant(i, j, k, l)``, such as :class:`~gbasis_b200.schwarz_screening.
        SchwarzScreener`) and ``contraction_index_map`` (``{id(shell): shell index}``), a
        quartet the screener rejects is returned as zeros without a device call."""
        shells = (cont_one, cont_two, cont_three, cont_four)
        for name, c in zip(("cont_one", "cont_two", "cont_three", "cont_four"), shells):
            if not is_shell(c):
                raise TypeError(f"`{name}` must be a `GeneralizedContractionShell` instance.")
        screener = kwargs.get("screener")
        index_map = kwargs.get("contraction_index_map")
        if screener is not None and index_map is not None:
            idx = [index_map.get(id(c)) for c in shells]
            if None not in idx and not screener.is_significant(*idx):
                shape = []
                for c in shells:
                    cf = np.asarray(c.coeffs)
                    shape += [cf.shape[1] if cf.ndim == 2 else 1, len(c.angmom_components_cart)]
                return np.zeros(shape)
        return super().construct_array_contraction(*shells)

    def _screen_from(self, kwargs):
        """Threshold of a whole-array call given the reference's screener hook.

        gbasis's whole-array methods pass ``screener`` and ``contraction_index_map`` to every
        ``construct_array_contraction`` call of their loop over unique shell quartets
        ((i, j) <= (k, l) over pairs i <= j, ``base_four_symm.py:189-191``).  Here the device
        zeroes the quartets with Q_ij Q_kl below ``screener.threshold`` in one pass, and the
        screener's counters grow as that loop would make them grow."""
        screener = kwargs.pop("screener", None)
        index_map = kwargs.pop("contraction_index_map", None)
        if kwargs:
            raise TypeError(f"unexpected keyword arguments: {', '.join(sorted(kwargs))}")
        if screener is None or index_map is None:
            return self._screen
        n = len(self.contractions)
        if [index_map.get(id(c)) for c in self.contractions] != list(range(n)):
            raise NotImplementedError("`contraction_index_map` must number the instance's "
                                      "shells 0..n-1 in order")
        t = float(screener.threshold)
        qp = np.sort(np.asarray(screener.bounds, dtype=float)[np.triu_indices(n)])
        npair = len(qp)
        total = npair * (npair + 1) // 2
        if t <= 0.0:
            computed = total
        else:
            # ordered pairs (a, b) with q_a q_b >= t, then unordered with a == b allowed
            pos = qp[qp > 0.0]
            need = t / pos
            ordered = int(np.sum(len(qp) - np.searchsorted(qp, need, side="left")))
            diag = int(np.count_nonzero(qp * qp >= t))
            computed = (ordered + diag) // 2
        screener.n_computed += computed
        screener.n_screened += total - computed
        return max(self._screen, t)

    def _screened(self, kwargs, call):
        saved = self._screen
        self._screen = self._screen_from(dict(kwargs))
        try:
            return call()
        finally:
            self._screen = saved

    def construct_array_cartesian(self, out=None, device=None, **kwargs):
        return self._screened(kwargs, lambda: super(ElectronRepulsionIntegralImproved, self)
                              .construct_array_cartesian(out, device))

    def construct_array_spherical(self, out=None, device=None, **kwargs):
        return self._screened(kwargs, lambda: super(ElectronRepulsionIntegralImproved, self)
                              .construct_array_spherical(out, device))

    def construct_array_mix(self, coord_types, out=None, device=None, **kwargs):
        return self._screened(kwargs, lambda: super(ElectronRepulsionIntegralImproved, self)
                              .construct_array_mix(coord_types, out, device))

    def construct_array_lincomb(self, transform, coord_type, device=None, **kwargs):
        return self._screened(kwargs, lambda: super(ElectronRepulsionIntegralImproved, self)
                              .construct_array_lincomb(transform, coord_type, device))


# isinstance checks against gbasis's own base classes accept these (when gbasis is importable)
register_with_gbasis(ElectronRepulsionIntegral, ElectronRepulsionIntegralImproved)


def _lincomb_device(shells, types, transform, screen, device, potential=(0, 0.0)):
    import ctypes
    import torch
    db = _engine.DeviceBasis(shells, types, device=device)
    try:
        if potential[0]:
            db.set_potential(*potential)
        n = db.nbf
        if transform.ndim != 2 or transform.shape[1] != n:
            raise ValueError(f"`transform` must have shape (K, {n})")
        k = transform.shape[0]
        dev = torch.device("cuda", db.device)
        m = max(n, k)
        eri = torch.empty(n ** 4, dtype=torch.float64, device=dev)
        work = torch.empty(2 * m ** 4, dtype=torch.float64, device=dev)
        out = torch.empty(k ** 4, dtype=torch.float64, device=dev)
        T = torch.from_numpy(np.ascontiguousarray(transform)).to(dev)
        stream = torch.cuda.current_stream(dev).cuda_stream
        db.full_device(eri.data_ptr(), "chemist", screen, stream=ctypes.c_void_p(stream))
        _engine.check(_engine.lib().gbx_lincomb(
            ctypes.c_void_p(eri.data_ptr()), n, ctypes.c_void_p(T.data_ptr()), k,
            ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(work.data_ptr()),
            ctypes.c_void_p(stream)), "gbx_lincomb")
        return out.cpu().numpy().reshape(k, k, k, k)
    finally:
        db.close()


def _dispatch(cls_obj, basis, transform, coord_type, out, device):
    types = [{"c": "cartesian", "p": "spherical"}.get(s.coord_type, s.coord_type) for s in basis]
    if coord_type is not None:
        types = [coord_type] * len(basis) if isinstance(coord_type, str) else list(coord_type)
    if transform is not None:
        return cls_obj.construct_array_lincomb(transform, types, device=device)
    if all(ct == "cartesian" for ct in types):
        return cls_obj.construct_array_cartesian(out=out, device=device)
    if all(ct == "spherical" for ct in types):
        return cls_obj.construct_array_spherical(out=out, device=device)
    return cls_obj.construct_array_mix(types, out=out, device=device)


def potential_code(potential="coulomb", omega=None):
    """Operator code of the engine for the names of gbasis's ``get_boys_function``
    (``gbasis/integrals/boys_functions.py:283-350``): 1/r, erf(omega r)/r or erfc(omega r)/r."""
    p = str(potential).lower()
    if p in ["coulomb", "standard", "1/r"]:
        return (0, 0.0)
    if p in ["erf", "erf_coulomb", "erfc", "erfc_coulomb"]:
        kind = "erf" if p.startswith("erf_") or p == "erf" else "erfc"
        if omega is None:
            raise ValueError(f"omega parameter is required for {kind}-attenuated potential")
        return (1 if kind == "erf" else 2, float(omega))
    raise ValueError(f"Unknown potential type: {potential}. Valid options: coulomb, erf, erfc")


# Mixed form thresholds on B_pq = Q_p Q_q, Q_p = sqrt(max |(ab|ab)|) over the pair's output
# functions (a rigorous bound on |(ab|cd)|).  Skipped quartets contribute at most MIXED_SKIP;
# an FP32 quartet's error is a fraction of its B_pq that depends on the molecule: about 1e-4
# on the 20-atom s/p/d/f chain (max error 1.2e-11 at an FP32 bound of 2e-7, 1.3e-10 at 1e-6),
# 1.6e-3 on the synthetic 2-14-atom s/p/d molecules with up to 6 primitives (3.2e-10 at 2e-7).
# The FP32 bound of 1e-8 keeps both below 1e-10 with margin; lowering it only moves quartets
# to FP64, so the error can only shrink.
MIXED_SKIP = 1e-11
MIXED_FP32 = 1e-8


def electron_repulsion_integral(basis, transform=None, notation="physicist", *, coord_type=None,
                                device=None, out=None, precision="fp64", mixed_skip=MIXED_SKIP,
                                mixed_fp32=MIXED_FP32, potential="coulomb", omega=None):
    """ERIs of ``basis`` (``electron_repulsion.py:214-281``): (K, K, K, K) float64, physicist
    notation by default (a ``transpose(0, 2, 1, 3)`` view of the chemist array).

    ``precision="mixed"`` selects the mixed form: quartets whose final-value Schwarz bound is
    below ``mixed_skip`` are zero, those below ``mixed_fp32`` run their vertical and transfer
    recursions in FP32.  ``potential`` ("coulomb", "erf" or "erfc", with ``omega``) selects the
    operator, as ``get_boys_function`` does for the reference's integral classes."""
    if notation not in ["physicist", "chemist"]:
        raise ValueError("`notation` must be one of 'physicist' or 'chemist'")
    if precision not in ("fp64", "mixed"):
        raise ValueError("`precision` must be 'fp64' or 'mixed'")
    obj = ElectronRepulsionIntegral(basis)
    obj._potential = potential_code(potential, omega)
    if precision == "mixed" and obj._potential[0]:
        raise NotImplementedError("the mixed-precision form computes 1/r integrals only")
    if precision == "mixed":
        obj._mixed = (float(mixed_skip), float(mixed_fp32))
    array = _dispatch(obj, basis, transform, coord_type, out, device)
    if notation == "physicist":
        array = np.transpose(array, (0, 2, 1, 3))
    return array


def electron_repulsion_integral_improved(basis, transform=None, notation="physicist",
                                         schwarz_threshold=0.0, *, coord_type=None, device=None,
                                         out=None, potential="coulomb", omega=None):
    """``electron_repulsion.py:415-504``: as :func:`electron_repulsion_integral`, with shell
    quartets whose Schwarz bound Q_ij Q_kl (blocks without ``norm_cont``) is below
    ``schwarz_threshold`` set to zero (Coulomb bounds, also for the erf/erfc operators)."""
    if notation not in ["physicist", "chemist"]:
        raise ValueError("`notation` must be one of 'physicist' or 'chemist'")
    obj = ElectronRepulsionIntegralImproved(basis, schwarz_threshold)
    obj._potential = potential_code(potential, omega)
    array = _dispatch(obj, basis, transform, coord_type, out, device)
    if notation == "physicist":
        array = np.transpose(array, (0, 2, 1, 3))
    return array
