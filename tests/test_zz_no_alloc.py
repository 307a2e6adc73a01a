"""The allocation-free entry point ``gbx_eri_full_noalloc`` (through the C ABI).

It serves callers that cannot call cudaMalloc while the library runs (their device memory
is owned by another allocator, or they cannot take cudaFree's device-wide synchronisation):
they pass host arrays for the basis and a device tensor they own, and every intermediate
lives in the library's static 64 MiB device array.  Checked against the regular entry point
``gbx_eri_full`` at the parity tolerance of the other tests (1e-12 absolute), on two calls
in a row with different bases (the array keeps the previous call's contents), and for the
size limit.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from gbasis_b200 import _engine
from gbasis_b200.contractions import GeneralizedContractionShell
from gbasis_b200.synthetic import make_workload

pytestmark = pytest.mark.gpu
ATOL = 1e-12


def _noalloc(shells, out, notation=_engine.GBX_CHEMIST, stream=None):
    pk = _engine.pack_basis(shells)
    p = _engine._ptr
    return _engine.lib().gbx_eri_full_noalloc(
        len(pk["angmom"]), p(pk["angmom"]), p(pk["nprim"]), p(pk["center"]), p(pk["exps"]),
        p(pk["coefs"]), p(pk["nout"]), p(pk["sph"]), p(pk["pos"]), p(pk["scl"]), notation,
        ctypes.c_void_p(out.data_ptr()), stream)


def _mixed_small():
    rng = np.random.default_rng(21)
    out = []
    for l, K, ct in ((2, 2, "spherical"), (0, 3, "cartesian"), (1, 2, "spherical"),
                     (2, 1, "cartesian"), (1, 1, "cartesian")):
        out.append(GeneralizedContractionShell(l, rng.uniform(-1.5, 1.5, 3),
                                               rng.uniform(0.1, 1.0, K),
                                               np.exp(rng.uniform(np.log(0.3), np.log(6.0), K)), ct))
    return out


def test_noalloc_matches_regular_entry_on_consecutive_calls():
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    for shells, notation in ((make_workload("tiny4"), "chemist"), (_mixed_small(), "physicist"),
                             (make_workload("tiny4"), "physicist")):
        db = _engine.DeviceBasis(shells)
        n = db.nbf
        ref = torch.empty(n ** 4, dtype=torch.float64, device=dev)
        got = torch.full((n ** 4,), float("nan"), dtype=torch.float64, device=dev)
        db.full_device(ref.data_ptr(), notation)
        code = _engine.GBX_PHYSICIST if notation == "physicist" else _engine.GBX_CHEMIST
        _engine.check(_noalloc(shells, got, code), "gbx_eri_full_noalloc")
        torch.cuda.synchronize()
        err = float((got - ref).abs().max())
        assert err <= ATOL, err
        db.close()


def test_noalloc_rejects_bases_beyond_its_scratch():
    import torch
    out = torch.empty(8, dtype=torch.float64, device="cuda")
    rc = _noalloc(make_workload("medium8"), out)
    assert rc == _engine.GBX_ERR_INVALID
    assert "limited to 64 MiB" in _engine.last_error()


def test_noalloc_takes_no_device_memory_and_does_not_wait_for_other_streams():
    """After a first call (set-up and kernel loading), a call leaves the device's free memory
    unchanged, and it returns while a bounded kernel queued earlier on another stream is still
    running: it makes no cudaMalloc/cudaFree and no device-wide synchronisation."""
    import torch
    shells = make_workload("tiny4")
    n = _engine.DeviceBasis(shells).nbf
    out = torch.empty(n ** 4, dtype=torch.float64, device="cuda")
    work = torch.cuda.Stream()
    side = torch.cuda.Stream()
    sp = ctypes.c_void_p(work.cuda_stream)
    _engine.check(_noalloc(shells, out, stream=sp), "gbx_eri_full_noalloc")
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    _engine.check(_noalloc(shells, out, stream=sp), "gbx_eri_full_noalloc")
    work.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    # about a second of spinning on the side stream (2e9 clock cycles: a bounded kernel)
    with torch.cuda.stream(side):
        torch.cuda._sleep(2_000_000_000)
    _engine.check(_noalloc(shells, out, stream=sp), "gbx_eri_full_noalloc")
    still_running = not side.query()
    torch.cuda.synchronize()
    assert still_running, "the call waited for work queued on another stream"
