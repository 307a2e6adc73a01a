"""Argument checks of the ERI drop-in (no GPU needed: every case raises before a device is
touched).  The cases follow the reference's own tests of the same checks:
``tests/test_electron_repulsion.py:24-35,304-310`` (shell types, notation),
``tests/test_base_four_symm.py:10-20,518-530,733-736`` (contractions, ``coord_types`` of
``construct_array_mix``, ``coord_type`` of ``construct_array_lincomb``)."""
import numpy as np
import pytest

from conftest import load_npz, shells_from_json
from gbasis_b200 import electron_repulsion as er
from gbasis_b200.contractions import GeneralizedContractionShell


def _s_shell():
    return GeneralizedContractionShell(0, np.zeros(3), np.array([1.0]), np.array([0.1]),
                                       "spherical")


@pytest.mark.parametrize("cls", [er.ElectronRepulsionIntegral,
                                 er.ElectronRepulsionIntegralImproved])
def test_construct_array_contraction_rejects_non_shells(cls):
    # gbasis/integrals/electron_repulsion.py:157-164
    c = _s_shell()
    for slot in range(4):
        args = [c, c, c, c]
        args[slot] = None
        with pytest.raises(TypeError):
            cls.construct_array_contraction(*args)


def test_contractions_checks():
    # gbasis/base.py:49-62
    c = _s_shell()
    assert er.ElectronRepulsionIntegral([c]).contractions == (c,)
    with pytest.raises(TypeError):
        er.ElectronRepulsionIntegral(c)
    with pytest.raises(ValueError):
        er.ElectronRepulsionIntegral([])
    with pytest.raises(TypeError):
        er.ElectronRepulsionIntegral([c, object()])
    with pytest.raises(TypeError):
        er.ElectronRepulsionIntegral([c], [c])
    with pytest.raises(TypeError):
        er.electron_repulsion_integral([c, "not a shell"])


def test_notation_and_precision_checks():
    # gbasis/integrals/electron_repulsion.py:265-266 and 494-495
    basis = shells_from_json(load_npz("tiny4.npz")["shells"])
    with pytest.raises(ValueError):
        er.electron_repulsion_integral(basis, notation="bad")
    with pytest.raises(ValueError):
        er.electron_repulsion_integral_improved(basis, notation="bad")
    with pytest.raises(ValueError):
        er.electron_repulsion_integral(basis, precision="fp16")
    with pytest.raises(NotImplementedError):
        er.electron_repulsion_integral(basis, precision="mixed", potential="erf", omega=0.5)
    with pytest.raises(ValueError):
        er.electron_repulsion_integral(basis, potential="erfc")


def test_construct_array_mix_checks():
    # gbasis/base_four_symm.py:422-432
    basis = shells_from_json(load_npz("tiny4.npz")["shells"])
    obj = er.ElectronRepulsionIntegral(basis)
    n = len(basis)
    with pytest.raises(TypeError):
        obj.construct_array_mix(np.array(["cartesian"] * n))
    with pytest.raises(ValueError):
        obj.construct_array_mix(["cartesian"] * (n - 1) + ["something"])
    with pytest.raises(ValueError):
        obj.construct_array_mix(["cartesian"] * (n + 1))


def test_construct_array_lincomb_coord_type_checks():
    # gbasis/base_four_symm.py:601-610: a bare string other than one made of a single
    # repeated coordinate type is not a list/tuple of types
    basis = shells_from_json(load_npz("tiny4.npz")["shells"])
    obj = er.ElectronRepulsionIntegral(basis)
    t = np.eye(3, 20)
    with pytest.raises(TypeError):
        obj.construct_array_lincomb(t, "bad")
    with pytest.raises(TypeError):
        obj.construct_array_lincomb(t, "spherical", bad_keyword=3)
    with pytest.raises(ValueError):
        obj.construct_array_lincomb(t, ["cartesian"] * len(basis) + ["spherical"])
