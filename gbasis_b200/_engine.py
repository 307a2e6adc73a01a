"""ctypes binding of ``libgbx_eri.so`` (the C ABI declared in ``include/gbx_eri.h``).

The library is built in-tree by ``python -m gbasis_b200.build``.  Loading fails loudly when
it is missing or when no CUDA device is present: the engine has no CPU path.
"""
from __future__ import annotations

import ctypes
import os
import threading

import numpy as np

from .contractions import is_shell

__all__ = ["lib", "EngineError", "check", "pack_basis", "DeviceBasis", "EXPORTED_SYMBOLS",
           "library_path", "fp64_peak", "release_cached_memory"]

LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib")
# GBX_DEBUG_BOUNDS=1 selects the bounds-checking build (python -m gbasis_b200.build
# --debug-bounds): every store of the kernels is index-checked and a call that went out of
# range returns an error instead of writing there
LIB_PATH = os.path.join(LIB_DIR, "libgbx_eri_debug.so" if os.environ.get("GBX_DEBUG_BOUNDS") == "1"
                        else "libgbx_eri.so")

GBX_OK, GBX_ERR_INVALID, GBX_ERR_UNSUPPORTED, GBX_ERR_OOM, GBX_ERR_CUDA, GBX_ERR_TIMEOUT = range(6)
GBX_CHEMIST, GBX_PHYSICIST = 0, 1
MAX_CART = 10

EXPORTED_SYMBOLS = (
    "gbx_basis_create", "gbx_basis_destroy", "gbx_basis_nbf", "gbx_basis_stats",
    "gbx_basis_set_groups", "gbx_eri_full", "gbx_eri_full_host", "gbx_schwarz_bounds",
    "gbx_lincomb", "gbx_eri_coulomb_j", "gbx_last_counts", "gbx_last_error", "gbx_fp64_peak",
    "gbx_set_profiling", "gbx_phase_times", "gbx_eri_full_noalloc",
    "gbx_num_blocks", "gbx_block_info", "gbx_set_team", "gbx_block_times",
    "gbx_eri_full_mixed", "gbx_eri_unique",
    "gbx_batch_create", "gbx_batch_destroy", "gbx_batch_info", "gbx_batch_run",
    "gbx_batch_set_graph", "gbx_unique_values", "gbx_compact_view",
    "gbx_batch_num_types", "gbx_batch_type_info", "gbx_batch_set_team", "gbx_batch_set_profiling",
    "gbx_batch_type_times", "gbx_release_cached_memory", "gbx_eri_jk", "gbx_point_charge",
    "gbx_basis_set_potential", "gbx_batch_run_mixed", "gbx_batch_mixed_counts", "gbx_boys_eval",
    "gbx_pipe_peak", "gbx_eri_coulomb_j_mixed", "gbx_set_block_config", "gbx_basis_set_streams",
    "gbx_batch_set_type_config", "gbx_mixed_counts", "gbx_batch_set_queue", "gbx_debug_bounds",
    "gbx_basis_set_fp32_lists",
)


class EngineError(RuntimeError):
    """A CUDA-side failure of the engine (launch error, device fault, timeout)."""


_lib = None
_lock = threading.Lock()

_P = ctypes.c_void_p
_I = ctypes.c_int
_D = ctypes.c_double
_I64 = ctypes.c_int64


def library_path():
    return LIB_PATH


def lib():
    """Load the engine library (once)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} is not built; run `python -m gbasis_b200.build` (needs nvcc)")
        L = ctypes.CDLL(LIB_PATH)
        sig = {
            "gbx_basis_create": [ctypes.POINTER(_P), _I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I],
            "gbx_basis_destroy": [_P],
            "gbx_basis_nbf": [_P, ctypes.POINTER(_I64)],
            "gbx_basis_stats": [_P, ctypes.POINTER(_I64), ctypes.POINTER(_I64)],
            "gbx_basis_set_groups": [_P, _P],
            "gbx_eri_full": [_P, _I, _D, _P, _P],
            "gbx_eri_full_host": [_P, _I, _D, _P, _P],
            "gbx_schwarz_bounds": [_P, _P],
            "gbx_lincomb": [_P, _I64, _P, _I64, _P, _P, _P],
            "gbx_eri_coulomb_j": [_P, _P, _D, _P, _P],
            "gbx_last_counts": [_P, ctypes.POINTER(_I64), ctypes.POINTER(_I64)],
            "gbx_mixed_counts": [_P, ctypes.POINTER(_I64), ctypes.POINTER(_I64),
                                 ctypes.POINTER(_I64)],
            "gbx_last_error": [ctypes.c_char_p, ctypes.c_size_t],
            "gbx_fp64_peak": [_I, ctypes.POINTER(_D)],
            "gbx_boys_eval": [_I, _I64, _P, _P],
            "gbx_pipe_peak": [_I, _I, ctypes.POINTER(_D)],
            "gbx_eri_coulomb_j_mixed": [_P, _P, _D, _D, _P, _P],
            "gbx_set_block_config": [_P, _I, _I, _I],
            "gbx_basis_set_streams": [_P, _I],
            "gbx_batch_set_type_config": [_P, _I, _I, _I],
            "gbx_set_profiling": [_P, _I],
            "gbx_phase_times": [_P, _P],
            "gbx_eri_full_noalloc": [_I, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I, _P, _P],
            "gbx_num_blocks": [_P, ctypes.POINTER(_I)],
            "gbx_block_info": [_P, _I, _P, ctypes.POINTER(_I), ctypes.POINTER(_D),
                               ctypes.POINTER(_I64)],
            "gbx_set_team": [_P, _I, _I],
            "gbx_block_times": [_P, _P, _I],
            "gbx_eri_full_mixed": [_P, _I, _D, _D, _P, _P],
            "gbx_eri_unique": [_P, _D, _D, _P],
            "gbx_batch_create": [ctypes.POINTER(_P), _I, _P, _P, _P, _P, _P, _P, _P, _P, _P,
                                 _P, _I],
            "gbx_batch_destroy": [_P],
            "gbx_batch_info": [_P, _P, ctypes.POINTER(_I64), ctypes.POINTER(_I64)],
            "gbx_batch_run": [_P, _I, _P, _P],
            "gbx_batch_set_graph": [_P, _I],
            "gbx_batch_set_queue": [_P, _I],
            "gbx_debug_bounds": [ctypes.POINTER(_I)],
            "gbx_basis_set_fp32_lists": [_P, _I64, _I64],
            "gbx_unique_values": [_P, _I64, _P, _P, _P],
            "gbx_compact_view": [_P, ctypes.POINTER(_P), ctypes.POINTER(_I64)],
            "gbx_batch_num_types": [_P, ctypes.POINTER(_I)],
            "gbx_batch_type_info": [_P, _I, _P, ctypes.POINTER(_I), ctypes.POINTER(_D),
                                    ctypes.POINTER(_I64)],
            "gbx_batch_set_team": [_P, _I, _I],
            "gbx_batch_set_profiling": [_P, _I],
            "gbx_batch_type_times": [_P, _P, _I],
            "gbx_release_cached_memory": [],
            "gbx_eri_jk": [_P, _P, _D, _P, _P, _P],
            "gbx_point_charge": [_P, _I, _P, _P, _I, _P, _P],
            "gbx_basis_set_potential": [_P, _I, _D],
            "gbx_batch_run_mixed": [_P, _I, _D, _D, _P, _P],
            "gbx_batch_mixed_counts": [_P, ctypes.POINTER(_I64), ctypes.POINTER(_I64),
                                       ctypes.POINTER(_I64)],
        }
        for name, args in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = _I
        _lib = L
        return L


def last_error():
    buf = ctypes.create_string_buffer(2048)
    lib().gbx_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(code, what=""):
    """Map a C-ABI status code to a Python exception."""
    if code == GBX_OK:
        return
    msg = f"{what}: {last_error()}" if what else last_error()
    if code == GBX_ERR_INVALID:
        raise ValueError(msg)
    if code == GBX_ERR_UNSUPPORTED:
        raise NotImplementedError(msg)
    if code == GBX_ERR_OOM:
        raise MemoryError(msg)
    if code == GBX_ERR_TIMEOUT:
        raise TimeoutError(msg)
    raise EngineError(msg)


# ---------------------------------------------------------------------------- packing
def _dfact(n):
    r = 1
    while n > 1:
        r *= n
        n -= 2
    return r


def _canon_cart(l):
    return [(x, y, l - x - y) for x in range(l, -1, -1) for y in range(l - x, -1, -1)]


def _canon_sph_labels(l):
    return [f"s{m}" for m in range(l, 0, -1)] + [f"c{m}" for m in range(l + 1)]


# real solid harmonics of l <= 1 as Cartesian components: s -> 1; p: c1=x, s1=y, c0=z
_P_LABEL = {(1, 0, 0): "c1", (0, 1, 0): "s1", (0, 0, 1): "c0"}


def _norm_cont(shell):
    coeffs = np.asarray(shell.coeffs)
    M = coeffs.shape[1] if coeffs.ndim == 2 else 1
    L = len(shell.angmom_components_cart)
    return np.asarray(shell.norm_cont, dtype=float).reshape(M, L)


def _coord_type(shell, override=None):
    ct = override if override is not None else shell.coord_type
    ct = {"c": "cartesian", "p": "spherical"}.get(ct, ct)
    if ct not in ("cartesian", "spherical"):
        raise ValueError("Each entry of `coord_types` must be one of 'cartesian' or 'spherical'.")
    return ct


def pack_basis(shells, coord_types=None, raw=False):
    """Flatten shells into the per-segmented-contraction arrays of ``gbx_basis_create``.

    ``raw=True`` packs the layout of ``construct_array_contraction``: Cartesian components in
    each shell's order with the component norm, without ``norm_cont``.
    Returns a dict of numpy arrays plus the segment -> (shell, m) map.
    """
    ang, npr, cen, exps, coefs, nout, sph, pos, scl, group = ([] for _ in range(10))
    for si, sh in enumerate(shells):
        if not is_shell(sh):
            raise TypeError("Given contractions must be instances of the "
                            "`GeneralizedContractionShell` class.")
        l = int(sh.angmom)
        e = np.asarray(sh.exps, dtype=float).ravel()
        c = np.asarray(sh.coeffs, dtype=float)
        c = c[:, None] if c.ndim == 1 else c
        ct = "cartesian" if raw else _coord_type(sh, None if coord_types is None else coord_types[si])
        cart = [tuple(int(v) for v in r) for r in np.asarray(sh.angmom_components_cart)]
        if sorted(cart) != sorted(_canon_cart(l)):
            raise ValueError(f"shell {si}: angmom_components_cart is not a permutation of the "
                             f"{len(_canon_cart(l))} components of l={l}")
        nc = np.ones((c.shape[1], len(cart))) if raw else _norm_cont(sh)
        for m in range(c.shape[1]):
            p = np.full(MAX_CART, -1, dtype=np.int8)
            s = np.zeros(MAX_CART)
            if ct == "cartesian":
                for k, comp in enumerate(_canon_cart(l)):
                    j = cart.index(comp)
                    p[k] = j
                    s[k] = nc[m, j] / np.sqrt(_dfact(2 * comp[0] - 1) * _dfact(2 * comp[1] - 1)
                                               * _dfact(2 * comp[2] - 1))
                n_o = len(cart)
            else:
                if not np.allclose(nc[m], nc[m][0], rtol=1e-14, atol=0):
                    raise NotImplementedError(
                        f"shell {si}: spherical transform with component-dependent norm_cont")
                labels = list(sh.angmom_components_sph)
                bare = [lab.lstrip("-") for lab in labels]
                if l >= 2:
                    internal = _canon_sph_labels(l)
                    coef = [1.0] * len(internal)
                else:
                    internal = ["c0"] if l == 0 else [_P_LABEL[cc] for cc in _canon_cart(1)]
                    coef = [1.0] * len(internal)
                for k, lab in enumerate(internal):
                    j = bare.index(lab)
                    p[k] = j
                    s[k] = nc[m][0] * coef[k] * (-1.0 if labels[j].startswith("-") else 1.0)
                n_o = 2 * l + 1
            ang.append(l)
            npr.append(len(e))
            cen.extend(np.asarray(sh.coord, dtype=float).ravel().tolist())
            exps.extend(e.tolist())
            coefs.extend(c[:, m].tolist())
            nout.append(n_o)
            sph.append(1 if ct == "spherical" else 0)
            pos.append(p)
            scl.append(s)
            group.append(si)
    return {
        "angmom": np.array(ang, dtype=np.int32), "nprim": np.array(npr, dtype=np.int32),
        "center": np.array(cen, dtype=np.float64), "exps": np.array(exps, dtype=np.float64),
        "coefs": np.array(coefs, dtype=np.float64), "nout": np.array(nout, dtype=np.int32),
        "sph": np.array(sph, dtype=np.int32), "pos": np.array(pos, dtype=np.int8).ravel(),
        "scl": np.array(scl, dtype=np.float64).ravel(), "group": np.array(group, dtype=np.int32),
    }


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class DeviceBasis:
    """A basis resident on one CUDA device (owns a ``gbx_basis`` handle)."""

    def __init__(self, shells, coord_types=None, raw=False, device=None, tuned=True):
        L = lib()
        if device is None:
            device = _current_device()
        self.packed = pk = pack_basis(shells, coord_types, raw)
        h = ctypes.c_void_p()
        check(L.gbx_basis_create(ctypes.byref(h), len(pk["angmom"]), _ptr(pk["angmom"]),
                                 _ptr(pk["nprim"]), _ptr(pk["center"]), _ptr(pk["exps"]),
                                 _ptr(pk["coefs"]), _ptr(pk["nout"]), _ptr(pk["sph"]),
                                 _ptr(pk["pos"]), _ptr(pk["scl"]), int(device)),
              "gbx_basis_create")
        self.handle = h
        self.device = int(device)
        check(L.gbx_basis_set_groups(h, _ptr(pk["group"])), "gbx_basis_set_groups")
        n = ctypes.c_int64()
        check(L.gbx_basis_nbf(h, ctypes.byref(n)))
        self.nbf = int(n.value)
        if tuned:
            from .autotune import apply_cache
            apply_cache(self)

    def stats(self):
        q, b = ctypes.c_int64(), ctypes.c_int64()
        check(lib().gbx_basis_stats(self.handle, ctypes.byref(q), ctypes.byref(b)))
        return int(q.value), int(b.value)

    def full_host(self, notation="chemist", schwarz_threshold=0.0, out=None, stream=None):
        n = self.nbf
        if out is None:
            out = np.empty((n, n, n, n), dtype=np.float64)
        assert out.dtype == np.float64 and out.flags.c_contiguous and out.size == n ** 4
        code = GBX_PHYSICIST if notation == "physicist" else GBX_CHEMIST
        check(lib().gbx_eri_full_host(self.handle, code, float(schwarz_threshold), _ptr(out),
                                      stream), "gbx_eri_full_host")
        return out

    def full_device(self, out_ptr, notation="chemist", schwarz_threshold=0.0, stream=None,
                    mixed=None):
        """Full tensor into device memory.  ``mixed=(skip, fp32)`` selects the mixed form."""
        code = GBX_PHYSICIST if notation == "physicist" else GBX_CHEMIST
        if mixed is not None:
            check(lib().gbx_eri_full_mixed(self.handle, code, float(mixed[0]), float(mixed[1]),
                                           ctypes.c_void_p(out_ptr), stream), "gbx_eri_full_mixed")
            return
        check(lib().gbx_eri_full(self.handle, code, float(schwarz_threshold),
                                 ctypes.c_void_p(out_ptr), stream), "gbx_eri_full")

    def unique(self, mixed=(0.0, 0.0), stream=None):
        """Unique quartets into the engine's compact store (no expansion)."""
        check(lib().gbx_eri_unique(self.handle, float(mixed[0]), float(mixed[1]), stream),
              "gbx_eri_unique")

    def unique_values(self, idx4, stream=None):
        """(ab|cd) for rows (a, b, c, d) of ``idx4`` from the last call's compact store."""
        q = np.ascontiguousarray(np.asarray(idx4, dtype=np.int64).reshape(-1, 4))
        out = np.empty(len(q))
        check(lib().gbx_unique_values(self.handle, len(q), _ptr(q), _ptr(out), stream),
              "gbx_unique_values")
        return out

    def compact_view(self):
        """The compact store of the last call as a read-only 1-D float64 CUDA tensor (a view
        of engine memory, valid until the next call on this basis), or None."""
        import torch
        p, n = ctypes.c_void_p(), ctypes.c_int64()
        check(lib().gbx_compact_view(self.handle, ctypes.byref(p), ctypes.byref(n)))
        if not p.value or n.value == 0:
            return None

        class _View:
            __cuda_array_interface__ = {"shape": (int(n.value),), "typestr": "<f8",
                                        "data": (int(p.value), False), "version": 3}
        return torch.as_tensor(_View(), device=torch.device("cuda", self.device))

    def schwarz_bounds(self):
        ns = len(self.packed["angmom"])
        q = np.empty((ns, ns))
        check(lib().gbx_schwarz_bounds(self.handle, _ptr(q)), "gbx_schwarz_bounds")
        return q

    def set_profiling(self, level=1):
        """0 off; 1 phase events; 2 phase and per-block events (blocks run one at a time)."""
        check(lib().gbx_set_profiling(self.handle, int(level)), "gbx_set_profiling")

    def phase_times(self):
        """(work-list build, class kernels, expansion) of the last call, milliseconds."""
        ms = np.zeros(3)
        check(lib().gbx_phase_times(self.handle, _ptr(ms)), "gbx_phase_times")
        return ms

    def blocks(self):
        """[(class (la, lb, lc, ld), team, mean primitive quartets, quartets)] per class block."""
        n = ctypes.c_int()
        check(lib().gbx_num_blocks(self.handle, ctypes.byref(n)))
        out = []
        for k in range(n.value):
            c4 = np.zeros(4, dtype=np.int32)
            t, ap, nq = ctypes.c_int(), ctypes.c_double(), ctypes.c_int64()
            check(lib().gbx_block_info(self.handle, k, _ptr(c4), ctypes.byref(t), ctypes.byref(ap),
                                       ctypes.byref(nq)))
            out.append((tuple(int(v) for v in c4), t.value, ap.value, nq.value))
        return out

    def set_team(self, k, team):
        check(lib().gbx_set_team(self.handle, int(k), int(team)), "gbx_set_team")

    def set_block_config(self, k, variant=0, ctas_per_sm=8):
        check(lib().gbx_set_block_config(self.handle, int(k), int(variant), int(ctas_per_sm)),
              "gbx_set_block_config")

    def set_streams(self, n):
        check(lib().gbx_basis_set_streams(self.handle, int(n)), "gbx_basis_set_streams")

    def block_times(self):
        n = ctypes.c_int()
        check(lib().gbx_num_blocks(self.handle, ctypes.byref(n)))
        ms = np.zeros(n.value)
        check(lib().gbx_block_times(self.handle, _ptr(ms), n.value), "gbx_block_times")
        return ms

    def last_counts(self):
        a, b = ctypes.c_int64(), ctypes.c_int64()
        check(lib().gbx_last_counts(self.handle, ctypes.byref(a), ctypes.byref(b)))
        return int(a.value), int(b.value)

    def set_fp32_lists(self, min_quartets=65536, share=4):
        """Mixed form: the smallest FP32 list (quartets, and share of its block) that gets
        its own FP32 launch; smaller ones stay in the FP64 list."""
        check(lib().gbx_basis_set_fp32_lists(self.handle, int(min_quartets), int(share)),
              "gbx_basis_set_fp32_lists")

    def mixed_counts(self):
        """(FP64, FP32, left out) quartets of the last full-tensor or unique-integral call."""
        a, b, c = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        check(lib().gbx_mixed_counts(self.handle, ctypes.byref(a), ctypes.byref(b),
                                     ctypes.byref(c)), "gbx_mixed_counts")
        return int(a.value), int(b.value), int(c.value)

    def set_potential(self, potential=0, omega=0.0):
        """Operator of later integral calls: 0 = 1/r, 1 = erf(omega r)/r, 2 = erfc(omega r)/r."""
        check(lib().gbx_basis_set_potential(self.handle, int(potential), float(omega)),
              "gbx_basis_set_potential")

    def close(self):
        if getattr(self, "handle", None):
            lib().gbx_basis_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def release_cached_memory():
    """Free the device memory that closed bases left for reuse (up to 2 GiB per device)."""
    check(lib().gbx_release_cached_memory(), "gbx_release_cached_memory")


def _current_device():
    try:
        import torch
        if torch.cuda.is_available():
            return torch.cuda.current_device()
    except Exception:
        pass
    return 0


def fp64_peak(device=0):
    v = ctypes.c_double()
    check(lib().gbx_fp64_peak(int(device), ctypes.byref(v)), "gbx_fp64_peak")
    return float(v.value)


def pipe_peak(pipe, device=0):
    """Measured TFLOP/s of pipe 0 (FP64 FMA), 1 (FP64 mma.sync) or 2 (FP32 FMA)."""
    v = ctypes.c_double()
    check(lib().gbx_pipe_peak(int(device), int(pipe), ctypes.byref(v)), "gbx_pipe_peak")
    return float(v.value)


def boys_eval(m_max, T):
    """F_0..F_{m_max}(T) for each T (n x (m_max + 1)) from the device Boys function the class
    kernels use (``gbx_boys_eval``)."""
    T = np.ascontiguousarray(T, dtype=np.float64).reshape(-1)
    F = np.empty((T.size, int(m_max) + 1), dtype=np.float64)
    check(lib().gbx_boys_eval(int(m_max), T.size, _ptr(T), _ptr(F)), "gbx_boys_eval")
    return F
