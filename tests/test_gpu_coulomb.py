"""Direct Coulomb matrix, and Coulomb plus exchange from the unique integrals (through the C
ABI), against the contractions of the full tensor."""
import numpy as np
import pytest

from conftest import load_npz, shells_from_json
from gbasis_b200 import electron_repulsion as er
from gbasis_b200 import _engine
from gbasis_b200.coulomb import coulomb_exchange, coulomb_matrix
from gbasis_b200.synthetic import density_matrix, make_workload

pytestmark = pytest.mark.gpu


def _check(shells, thr):
    eri = er.electron_repulsion_integral(shells, notation="chemist")
    n = eri.shape[0]
    D = density_matrix(n, seed=n)
    J = coulomb_matrix(shells, D, schwarz_threshold=0.0)
    ref = np.einsum("abcd,cd->ab", eri, D)
    np.testing.assert_allclose(J, ref, rtol=0, atol=1e-12 * max(1.0, np.abs(ref).max()))
    np.testing.assert_allclose(J, J.T, rtol=0, atol=1e-13)
    if thr:
        Jt = coulomb_matrix(shells, D, schwarz_threshold=thr)
        eri_t = er.electron_repulsion_integral_improved(shells, notation="chemist",
                                                        schwarz_threshold=thr)
        np.testing.assert_allclose(Jt, np.einsum("abcd,cd->ab", eri_t, D), rtol=0,
                                   atol=1e-12 * max(1.0, np.abs(ref).max()))


def test_coulomb_tiny4():
    _check(make_workload("tiny4"), 1e-4)


def test_coulomb_mixed_with_f_shells():
    z = load_npz("mixed.npz")
    _check(shells_from_json(z["shells"]), 1e-3)


def test_coulomb_medium8():
    _check(make_workload("medium8")[:18], 1e-8)


def _check_jk(shells, thr, symmetric):
    eri = er.electron_repulsion_integral(shells, notation="chemist")
    n = eri.shape[0]
    rng = np.random.default_rng(n)
    D = rng.standard_normal((n, n))
    if symmetric:
        D = D + D.T
    J, K = coulomb_exchange(shells, D)
    Jr, Kr = np.einsum("abcd,cd->ab", eri, D), np.einsum("abcd,bd->ac", eri, D)
    tol = 1e-12 * max(1.0, np.abs(Jr).max(), np.abs(Kr).max())
    np.testing.assert_allclose(J, Jr, rtol=0, atol=tol)
    np.testing.assert_allclose(K, Kr, rtol=0, atol=tol)
    if thr:
        eri_t = er.electron_repulsion_integral_improved(shells, notation="chemist",
                                                        schwarz_threshold=thr)
        Jt, Kt = coulomb_exchange(shells, D, schwarz_threshold=thr)
        np.testing.assert_allclose(Jt, np.einsum("abcd,cd->ab", eri_t, D), rtol=0, atol=tol)
        np.testing.assert_allclose(Kt, np.einsum("abcd,bd->ac", eri_t, D), rtol=0, atol=tol)


def test_jk_tiny4_general_density():
    _check_jk(make_workload("tiny4"), 1e-4, symmetric=False)


def test_jk_mixed_with_f_shells():
    z = load_npz("mixed.npz")
    _check_jk(shells_from_json(z["shells"]), 1e-3, symmetric=True)


def test_jk_medium8_subset():
    _check_jk(make_workload("medium8")[:18], 0.0, symmetric=False)


def test_jk_rows_beyond_shared_memory():
    """255 functions: a row of unique integrals (32,640 values) exceeds shared memory, so the
    kernel reads the compact store directly; reference contractions of the device tensor."""
    import torch
    from gbasis_b200.synthetic import box_atoms, random_shell
    rng = np.random.default_rng(77)
    recipe = [(0, 6), (0, 3), (0, 1), (1, 3), (1, 1), (2, 1)]
    shells = [random_shell(rng, l, k, c, "cartesian") for c in box_atoms(rng, 17, 13.0)
              for l, k in recipe]
    db = _engine.DeviceBasis(shells)
    try:
        n = db.nbf
        assert n * (n + 1) // 2 * 8 > 227 * 1024
        g = torch.Generator(device="cuda").manual_seed(5)
        D = torch.randn((n, n), dtype=torch.float64, device="cuda", generator=g)
        T = torch.empty(n ** 4, dtype=torch.float64, device="cuda")
        db.full_device(T.data_ptr(), "chemist")   # [a, b, c, d]
        Jr = (T.view(n * n, n * n) @ D.reshape(-1)).view(n, n)
        db.full_device(T.data_ptr(), "physicist")  # [a, c, b, d]
        Kr = (T.view(n * n, n * n) @ D.reshape(-1)).view(n, n)
        del T
        J = torch.empty((n, n), dtype=torch.float64, device="cuda")
        K = torch.empty((n, n), dtype=torch.float64, device="cuda")
        _engine.check(_engine.lib().gbx_eri_jk(db.handle, D.data_ptr(), 0.0, J.data_ptr(),
                                               K.data_ptr(), None), "gbx_eri_jk")
        torch.cuda.synchronize()
        tol = 1e-12 * max(1.0, float(Jr.abs().max()), float(Kr.abs().max()))
        assert float((J - Jr).abs().max()) <= tol
        assert float((K - Kr).abs().max()) <= tol
    finally:
        db.close()
        torch.cuda.empty_cache()


def test_jk_rejects_bad_arguments():
    import torch
    db = _engine.DeviceBasis(make_workload("tiny4"))
    try:
        n = db.nbf
        D, J = (torch.zeros((n, n), dtype=torch.float64, device="cuda") for _ in range(2))
        L = _engine.lib()
        with pytest.raises(ValueError):
            _engine.check(L.gbx_eri_jk(db.handle, D.data_ptr(), 0.0, J.data_ptr(), 0, None))
        with pytest.raises(ValueError):
            _engine.check(L.gbx_eri_jk(db.handle, D.data_ptr(), 0.0, J.data_ptr(), J.data_ptr(),
                                       None))
        with pytest.raises(ValueError):
            _engine.check(L.gbx_eri_jk(db.handle, D.data_ptr(), -1.0, J.data_ptr(),
                                       D.data_ptr(), None))
    finally:
        db.close()


def test_direct_coulomb_large64_subset_against_oracle_rows():
    """The 64-atom box's first 16 atoms (160 spherical shells with f, N = 480): direct J
    without screening against J rows assembled from oracle blocks, J_ab = sum_cd (ab|cd) D_cd
    over every ket shell pair (both orders of an off-diagonal ket pair, D symmetric), for bra
    shell pairs s(8)s(8), p-d and f-f on different atoms.  The screened J (1e-12) and the mixed
    form's J stay within 1e-10 of it."""
    import os
    from oracle import parallel as opar
    wl = "large64:160"
    shells = opar.workload_shells(wl)
    sizes = [2 * s.angmom + 1 if s.coord_type in ("spherical", "p") else
             len(s.angmom_components_cart) for s in shells]
    off = np.concatenate([[0], np.cumsum(sizes)])
    n = int(off[-1])
    assert n == 480
    D = density_matrix(n)
    J = coulomb_matrix(shells, D, schwarz_threshold=0.0)
    byl = {}
    for x, s in enumerate(shells):
        byl.setdefault((s.angmom, len(s.exps)), []).append(x)
    bra = [(byl[(0, 8)][0], byl[(0, 8)][3]), (byl[(1, 3)][1], byl[(2, 2)][5]),
           (byl[(3, 1)][2], byl[(3, 1)][9])]
    kets = [(k, l) for k in range(len(shells)) for l in range(k, len(shells))]
    quart = np.array([(i, j, k, l) for i, j in bra for k, l in kets])
    vals = opar.oracle_blocks(wl, quart, processes=min(os.cpu_count() or 1, 32), chunk=64)
    pos = 0
    scale = max(1.0, float(np.abs(J).max()))
    for i, j in bra:
        ref = np.zeros((sizes[i], sizes[j]))
        for k, l in kets:
            m = sizes[i] * sizes[j] * sizes[k] * sizes[l]
            blk = vals[pos:pos + m].reshape(sizes[i], sizes[j], sizes[k], sizes[l])
            pos += m
            dcd = D[off[k]:off[k + 1], off[l]:off[l + 1]]
            ref += (1.0 if k == l else 2.0) * np.einsum("abcd,cd->ab", blk, dcd)
        got = J[off[i]:off[i + 1], off[j]:off[j + 1]]
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-12 * scale)
    assert pos == vals.size
    Jt = coulomb_matrix(shells, D, schwarz_threshold=1e-12)
    assert np.abs(Jt - J).max() <= 1e-10
    Jm = coulomb_matrix(shells, D, precision="mixed")
    assert np.abs(Jm - J).max() <= 1e-10
