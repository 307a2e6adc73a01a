"""GPU tests of the device block cache: a closed basis gives its device blocks back for the
next basis of the process (the public call builds and drops one per call).  Reused blocks hold
the previous basis's values, so every result must match a computation on fresh allocations."""
import numpy as np
import pytest

from gbasis_b200 import _engine
from gbasis_b200.synthetic import batch_molecule

pytestmark = pytest.mark.gpu


def _tensor(shells, host):
    import torch
    db = _engine.DeviceBasis(shells)
    n = db.nbf
    if host:
        out = db.full_host("chemist")
    else:
        dev = torch.full((n ** 4,), np.nan, dtype=torch.float64, device="cuda")
        db.full_device(dev.data_ptr(), "chemist")
        torch.cuda.synchronize()
        out = dev.cpu().numpy().reshape((n,) * 4)
    db.close()
    return out


@pytest.mark.parametrize("host", [False, True])
def test_reused_blocks_give_the_same_tensors(host):
    mols = [batch_molecule(k) for k in (3, 7, 3, 11, 7)]
    _engine.release_cached_memory()
    fresh = {}
    for k, m in zip((3, 7, 11), (mols[0], mols[1], mols[3])):
        fresh[k] = _tensor(m, host)
        _engine.release_cached_memory()  # next basis allocates anew
    # one after another: each basis takes the blocks the previous one left
    for k, m in zip((3, 7, 3, 11, 7), mols):
        np.testing.assert_array_equal(_tensor(m, host), fresh[k])
    _engine.release_cached_memory()
    np.testing.assert_array_equal(_tensor(mols[3], host), fresh[11])
