"""Host-side argument handling of the added entry points (no GPU needed: every case raises
before a device is touched)."""
import numpy as np
import pytest

from conftest import load_npz, shells_from_json
from gbasis_b200 import point_charge as pc
from gbasis_b200.electron_repulsion import potential_code


def test_potential_names_follow_get_boys_function():
    # gbasis/integrals/boys_functions.py:283-350
    for name in ("coulomb", "standard", "1/r", "Coulomb"):
        assert potential_code(name) == (0, 0.0)
    assert potential_code("erf", 0.4) == (1, 0.4)
    assert potential_code("erf_coulomb", 0.4) == (1, 0.4)
    assert potential_code("erfc", 1.5) == (2, 1.5)
    assert potential_code("ERFC_COULOMB", 1.5) == (2, 1.5)
    with pytest.raises(ValueError, match="omega parameter is required for erf-attenuated"):
        potential_code("erf")
    with pytest.raises(ValueError, match="omega parameter is required for erfc-attenuated"):
        potential_code("erfc")
    with pytest.raises(ValueError, match="Unknown potential type"):
        potential_code("yukawa", 1.0)


def test_point_charge_argument_checks():
    # gbasis/integrals/point_charge.py:180-218
    basis = shells_from_json(load_npz("tiny4.npz")["shells"])
    with pytest.raises(TypeError):
        pc.point_charge_integral(basis, [[0.0, 0.0, 0.0]], np.ones(1))
    with pytest.raises(TypeError):
        pc.point_charge_integral(basis, np.zeros((2, 2)), np.ones(2))
    with pytest.raises(TypeError):
        pc.point_charge_integral(basis, np.zeros((2, 3)), np.ones((2, 1)))
    with pytest.raises(TypeError):
        pc.point_charge_integral(basis, np.zeros((2, 3), dtype=complex), np.ones(2))
    with pytest.raises(ValueError):
        pc.nuclear_electron_attraction_integral(basis, np.zeros((2, 3)), np.ones(3))
    with pytest.raises(TypeError):
        pc.point_charge_integral([object()], np.zeros((1, 3)), np.ones(1))


def test_reference_module_paths():
    # gbasis.integrals.<module> -> gbasis_b200.integrals.<module>, same names, same objects
    import importlib
    from gbasis_b200 import electron_repulsion, point_charge, schwarz_screening
    expect = {
        "electron_repulsion": (electron_repulsion, ["ElectronRepulsionIntegral",
                                                    "ElectronRepulsionIntegralImproved",
                                                    "electron_repulsion_integral",
                                                    "electron_repulsion_integral_improved"]),
        "_schwarz_screening": (schwarz_screening, ["compute_schwarz_bound_shell_pair",
                                                   "compute_schwarz_bounds",
                                                   "shell_pair_significant", "SchwarzScreener"]),
        "point_charge": (point_charge, ["point_charge_integral"]),
        "nuclear_electron_attraction": (point_charge, ["nuclear_electron_attraction_integral"]),
    }
    for mod, (src, names) in expect.items():
        m = importlib.import_module(f"gbasis_b200.integrals.{mod}")
        for name in names:
            assert getattr(m, name) is getattr(src, name)
    from gbasis_b200.contractions import GeneralizedContractionShell  # gbasis.contractions
    assert GeneralizedContractionShell.__name__ == "GeneralizedContractionShell"


def test_no_cpu_fallback_without_library_or_device():
    """The engine has no CPU path: without its library the call raises ImportError, and where
    the library loads but no CUDA device answers (as on a CPU-only machine) it raises
    EngineError instead of returning anything."""
    import subprocess
    import sys
    code = r'''
import sys
sys.path.insert(0, sys.argv[1])
from gbasis_b200 import _engine
from gbasis_b200 import electron_repulsion as er
from gbasis_b200.synthetic import make_workload
shells = make_workload("tiny4")
_engine.LIB_PATH = "/nonexistent/libgbx_eri.so"
_engine._lib = None
try:
    er.electron_repulsion_integral(shells)
    print("RETURNED")
except ImportError:
    print("IMPORTERROR")
'''
    import os
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = subprocess.run([sys.executable, "-c", code, root], capture_output=True, text=True,
                         timeout=300)
    assert out.stdout.strip().splitlines()[-1] == "IMPORTERROR", out.stdout + out.stderr
    from gbasis_b200 import _engine
    import torch
    if os.path.exists(_engine.LIB_PATH) and not torch.cuda.is_available():
        from gbasis_b200 import electron_repulsion as er
        from gbasis_b200.synthetic import make_workload
        with pytest.raises(_engine.EngineError):
            er.electron_repulsion_integral(make_workload("tiny4"))


def test_class_hierarchy_mirrors_gbasis():
    """ElectronRepulsionIntegral is a BaseFourIndexSymmetric / BaseGaussianRelatedArray with the
    reference's constructor contract (gbasis/base.py:32-65, gbasis/base_four_symm.py:70-93)."""
    import pytest
    from gbasis_b200.base import BaseGaussianRelatedArray
    from gbasis_b200.base_four_symm import BaseFourIndexSymmetric
    from gbasis_b200.electron_repulsion import (ElectronRepulsionIntegral,
                                                ElectronRepulsionIntegralImproved)
    from gbasis_b200.synthetic import make_workload
    shells = make_workload("tiny4")
    for cls in (ElectronRepulsionIntegral, ElectronRepulsionIntegralImproved):
        obj = cls(shells)
        assert isinstance(obj, BaseFourIndexSymmetric) and isinstance(obj, BaseGaussianRelatedArray)
        assert obj.contractions == tuple(shells)
        assert obj._axes_contractions == (tuple(shells),)
    with pytest.raises(TypeError, match="list or tuple"):
        ElectronRepulsionIntegral(shells[0])
    with pytest.raises(ValueError, match="At least one"):
        ElectronRepulsionIntegral([])
    with pytest.raises(TypeError, match="must be instances"):
        ElectronRepulsionIntegral([shells[0], 1.0])
    with pytest.raises(TypeError):
        BaseFourIndexSymmetric(shells)  # abstract, as in the reference


def test_virtual_subclass_of_gbasis_base_classes():
    """With gbasis importable, isinstance checks against its own base classes accept the
    engine's objects (a stand-in gbasis package here: two ABCs)."""
    import abc
    import sys
    import types
    from gbasis_b200.base_four_symm import register_with_gbasis
    from gbasis_b200.electron_repulsion import ElectronRepulsionIntegral
    from gbasis_b200.synthetic import make_workload

    class FakeBase(abc.ABC):
        pass

    class FakeFour(FakeBase):
        pass
    pkg = types.ModuleType("gbasis")
    base = types.ModuleType("gbasis.base")
    four = types.ModuleType("gbasis.base_four_symm")
    base.BaseGaussianRelatedArray = FakeBase
    four.BaseFourIndexSymmetric = FakeFour
    saved = {k: sys.modules.get(k) for k in ("gbasis", "gbasis.base", "gbasis.base_four_symm")}
    sys.modules.update({"gbasis": pkg, "gbasis.base": base, "gbasis.base_four_symm": four})
    try:
        assert register_with_gbasis(ElectronRepulsionIntegral)
        obj = ElectronRepulsionIntegral(make_workload("tiny4"))
        assert isinstance(obj, FakeFour) and isinstance(obj, FakeBase)
    finally:
        for k, v in saved.items():
            if v is None:
                sys.modules.pop(k, None)
            else:
                sys.modules[k] = v
