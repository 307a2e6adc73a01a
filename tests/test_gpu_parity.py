"""GPU parity of the engine (through its C ABI) against the oracle and the golden fixtures.

Tolerance: 1e-12 absolute (the bar for the FP64 form), or, for the few diffuse high-l
quartets on which the reference itself loses digits, four times the reference's own
distance from the 40-digit values.
"""
import json

import numpy as np
import pytest

from conftest import expand_unique, load_npz, shell_from_record, shells_from_json
from gbasis_b200 import electron_repulsion as er
from gbasis_b200 import _engine
from gbasis_b200.contractions import GeneralizedContractionShell
from gbasis_b200.synthetic import make_workload
from oracle import eri_oracle as orc

pytestmark = pytest.mark.gpu
ATOL = 1e-12


def _max_l(shells):
    return max(s.angmom for s in shells)


def _need(shells, lmax=3):
    if _max_l(shells) > lmax:
        pytest.skip("classes above the compiled angular momentum")


def test_tiny4_against_reference_tensor():
    z = load_npz("tiny4.npz")
    shells = shells_from_json(z["shells"])
    chem = er.electron_repulsion_integral(shells, notation="chemist")
    idx = z["index"].astype(int)
    vals = chem[idx[:, 0], idx[:, 1], idx[:, 2], idx[:, 3]]
    np.testing.assert_allclose(vals, z["values"], rtol=0, atol=ATOL)
    np.testing.assert_allclose(chem, expand_unique(chem.shape[0], z["values"]), rtol=0, atol=ATOL)
    phys = er.electron_repulsion_integral(shells)
    assert phys.shape == chem.shape
    np.testing.assert_array_equal(phys, np.transpose(chem, (0, 2, 1, 3)))


def test_tiny4_physicist_layout_from_device():
    shells = make_workload("tiny4")
    db = _engine.DeviceBasis(shells)
    chem = db.full_host("chemist")
    phys = db.full_host("physicist")
    np.testing.assert_array_equal(phys, np.ascontiguousarray(np.transpose(chem, (0, 2, 1, 3))))


def test_horton_bec_sto6g():
    z = load_npz("horton_bec_sto6g.npz")
    shells = shells_from_json(z["shells"])
    got = er.electron_repulsion_integral(shells)
    np.testing.assert_allclose(got, z["reference"], rtol=0, atol=ATOL)
    np.testing.assert_allclose(got, z["horton"], rtol=1e-10, atol=1e-15)


def test_quartet_blocks_every_class():
    z = load_npz("quartets.npz")
    recs = json.loads(str(z["shells"]))
    split = np.cumsum(z["sizes"])[:-1]
    blocks, truth, improved = (np.split(z[k], split) for k in ("blocks", "truth", "improved"))
    n_done = 0
    for rq, ref, tru, imp in zip(recs, blocks, truth, improved):
        sh = [shell_from_record(r) for r in rq]
        got = er.ElectronRepulsionIntegral.construct_array_contraction(*sh).ravel()
        # accurate against the 40-digit values, and equal to the reference to within 1e-12
        # plus the reference's own error
        assert np.max(np.abs(got - tru)) <= ATOL, [s.angmom for s in sh]
        assert np.max(np.abs(got - ref)) <= ATOL + float(np.max(np.abs(ref - tru))), \
            [s.angmom for s in sh]
        n_done += 1
    assert n_done == len(recs)


@pytest.mark.parametrize("kind", ["cart", "sph", "mix", "lincomb", "screened"])
def test_mixed_basis(kind):
    z = load_npz("mixed.npz")
    shells = shells_from_json(z["shells"])
    _need(shells)
    cts = [s.coord_type for s in shells]
    obj = er.ElectronRepulsionIntegral(shells)
    if kind == "cart":
        got = obj.construct_array_cartesian()
    elif kind == "sph":
        got = obj.construct_array_spherical()
    elif kind == "mix":
        got = obj.construct_array_mix(cts)
    elif kind == "lincomb":
        got = er.electron_repulsion_integral(shells, transform=z["transform"], notation="chemist")
    else:
        got = er.electron_repulsion_integral_improved(shells, notation="chemist",
                                                      schwarz_threshold=1e-3)
    n = int(z[kind + "_n"])
    ref = expand_unique(n, z[kind])
    truth = expand_unique(n, z[kind + "_truth"])
    tol = max(ATOL, 4 * float(np.max(np.abs(ref - truth))))
    assert np.max(np.abs(got - truth)) <= tol


def _small_mixed_l2(seed=11, ctypes_=("spherical", "cartesian", "spherical", "spherical")):
    rng = np.random.default_rng(seed)
    shells = []
    for l, K, M, ct in zip((0, 1, 2, 2), (3, 2, 2, 1), (1, 1, 2, 1), ctypes_):
        exps = np.exp(rng.uniform(np.log(0.5), np.log(5.0), size=K))
        coeffs = rng.uniform(0.1, 1.0, size=(K, M)) if M > 1 else rng.uniform(0.1, 1.0, size=K)
        shells.append(GeneralizedContractionShell(l, rng.uniform(-0.6, 0.6, 3), coeffs, exps, ct))
    return shells


@pytest.mark.parametrize("mode", ["cartesian", "spherical", "mix"])
def test_small_basis_modes_against_oracle(mode):
    shells = _small_mixed_l2()
    if mode == "mix":
        types = [s.coord_type for s in shells]
    else:
        types = [mode] * len(shells)
    ref = orc.construct_array(shells, types, reorder="exponent")
    got = er.electron_repulsion_integral(shells, notation="chemist", coord_type=types)
    np.testing.assert_allclose(got, ref, rtol=0, atol=ATOL)


def test_lincomb_against_oracle():
    shells = _small_mixed_l2(5)
    types = [s.coord_type for s in shells]
    ref_ao = orc.construct_array(shells, types, reorder="exponent")
    n = ref_ao.shape[0]
    T = np.random.default_rng(3).normal(size=(n - 2, n))
    got = er.electron_repulsion_integral(shells, transform=T)
    ref = np.transpose(orc.construct_array_lincomb(ref_ao, T), (0, 2, 1, 3))
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-10)


def test_schwarz_screened_against_oracle():
    shells = make_workload("tiny4")
    for thr in (1e-6, 1e-3, 1e-1):
        ref = orc.electron_repulsion_integral_screened(shells, thr, notation="chemist",
                                                       reorder="exponent")
        got = er.electron_repulsion_integral_improved(shells, notation="chemist",
                                                      schwarz_threshold=thr)
        np.testing.assert_allclose(got, ref, rtol=0, atol=ATOL)
    db = _engine.DeviceBasis(shells)
    q = db.schwarz_bounds()
    qref = orc.schwarz_bounds(shells)
    np.testing.assert_allclose(q, qref, rtol=1e-12)


def test_medium8_full_size_sampled_parity_and_symmetry():
    """The 8-atom, 120-function workload (1.66 GB tensor): oracle blocks of a seeded sample of
    shell quartets, 8-fold symmetry, positive diagonal and the Schwarz inequality."""
    shells = make_workload("medium8")
    T = er.electron_repulsion_integral(shells, notation="chemist")
    n = T.shape[0]
    assert n == 120
    off = np.cumsum([0] + [len(s.angmom_components_cart) for s in shells])
    rng = np.random.default_rng(0)
    for _ in range(40):
        i, j, k, l = rng.integers(0, len(shells), size=4)
        blk = orc.construct_array_contraction(shells[i], shells[j], shells[k], shells[l],
                                              reorder="exponent")[0, :, 0, :, 0, :, 0, :]
        nc = [shells[x].norm_cont[0] for x in (i, j, k, l)]
        blk = np.einsum("abcd,a,b,c,d->abcd", blk, *nc)
        got = T[off[i]:off[i + 1], off[j]:off[j + 1], off[k]:off[k + 1], off[l]:off[l + 1]]
        np.testing.assert_allclose(got, blk, rtol=0, atol=ATOL)
    a, b, c, d = rng.integers(0, n, size=(4, 200000))
    v = T[a, b, c, d]
    for perm in [(b, a, c, d), (a, b, d, c), (c, d, a, b), (d, c, b, a)]:
        # exact except inside diagonal shell blocks, where (ab| and (ba| are computed apart
        np.testing.assert_allclose(T[perm], v, rtol=1e-13, atol=1e-14)
    diag = T[np.arange(n), np.arange(n), np.arange(n), np.arange(n)]
    assert np.all(diag > 0)
    D2 = np.einsum("abab->ab", T)
    assert np.all(v * v <= D2[a, b] * D2[c, d] * (1 + 1e-10) + 1e-24)


@pytest.mark.parametrize("notation", ["chemist", "physicist"])
def test_streamed_host_tensor_equals_device_tensor(notation):
    """Host output is expanded slab by slab (30 staging slabs for N = 120) and copied out
    while later slabs expand; it must equal the device-resident tensor bit for bit."""
    import torch
    shells = make_workload("medium8")
    db = _engine.DeviceBasis(shells)
    n = db.nbf
    dev = torch.empty(n ** 4, dtype=torch.float64, device="cuda")
    db.full_device(dev.data_ptr(), notation)
    torch.cuda.synchronize()
    host = db.full_host(notation)
    np.testing.assert_array_equal(host.reshape(-1), dev.cpu().numpy())
    pinned = torch.empty(n ** 4, dtype=torch.float64, pin_memory=True).numpy().reshape((n,) * 4)
    db.full_host(notation, out=pinned)
    np.testing.assert_array_equal(pinned, host)
    db.close()


def test_errors_match_reference_behaviour():
    shells = make_workload("tiny4")
    with pytest.raises(ValueError):
        er.electron_repulsion_integral(shells, notation="bad")
    with pytest.raises(TypeError):
        er.ElectronRepulsionIntegral.construct_array_contraction(None, shells[0], shells[0],
                                                                 shells[0])
    with pytest.raises(TypeError):
        er.ElectronRepulsionIntegral([shells[0], 3])
    with pytest.raises(ValueError):
        er.ElectronRepulsionIntegral([])
    with pytest.raises(ValueError):
        er.ElectronRepulsionIntegral(shells).construct_array_mix(["cartesian"])


def test_horton_large_exponent_quartet():
    """gbasis tests/test_two_elec_int.py ``test_compute_two_elec_integrals_overflow_horton``,
    an xfail in the reference (its double path loses every digit of this (ss|ff) quartet):
    the engine runs the recursions from the f pair and matches the 40-digit value and HORTON's
    value, in both pair orders."""
    from conftest import horton_overflow_case
    shells, i, rec = horton_overflow_case()
    truth = rec["truth_40_digits"]
    blk = er.ElectronRepulsionIntegral.construct_array_contraction(*shells)
    assert blk.shape == (1, 1, 1, 1, 1, 10, 1, 10)
    got = blk[0, i[0], 0, i[1], 0, i[2], 0, i[3]]
    assert abs(got - truth) <= ATOL
    assert np.allclose(got, rec["horton"])  # the reference test's tolerance
    blk = er.ElectronRepulsionIntegral.construct_array_contraction(shells[2], shells[3],
                                                                   shells[0], shells[1])
    assert abs(blk[0, i[2], 0, i[3], 0, i[0], 0, i[1]] - truth) <= ATOL
