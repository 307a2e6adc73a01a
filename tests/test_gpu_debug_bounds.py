"""GPU test of the bounds-checking build (``libgbx_eri_debug.so``, made by
``python -m gbasis_b200.build --debug-bounds`` and selected with ``GBX_DEBUG_BOUNDS=1``).

In that build every store of the class kernels (register, split, line and queue kernels), of
the work-list build and the zero fill, of the expansions (device tensor, host-copy slabs,
batch) and of the J / K scatter, and every compact-store read of the expansions, is checked
against the array it addresses; an out-of-range index is recorded instead of written and the
call returns an error.  The device-side checker of such stores (compute-sanitizer) is not
available here, so this build stands in for it.  The calls below cover each of those sites in
a child process (one library per process) and must run clean and give the checkers' values.
"""
import json
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DEBUG_LIB = os.path.join(ROOT, "gbasis_b200", "_lib", "libgbx_eri_debug.so")

CHILD = r"""
import ctypes, json, sys
import numpy as np
import torch
sys.path.insert(0, "tests")
from conftest import expand_unique, load_npz, shells_from_json
from gbasis_b200 import _engine
from gbasis_b200 import electron_repulsion as er
from gbasis_b200.batch import EriBatch
from gbasis_b200.coulomb import coulomb_exchange, coulomb_matrix
from gbasis_b200.electron_repulsion import MIXED_FP32, MIXED_SKIP
from gbasis_b200.synthetic import batch_molecule, make_workload
from oracle import eri_oracle as orc

res = {}
on = ctypes.c_int(0)
_engine.check(_engine.lib().gbx_debug_bounds(ctypes.byref(on)))
res["lib"] = _engine.LIB_PATH
res["checks_on"] = on.value

# tiny4 (s, p): device tensor and the host-streamed default call (slab expansion)
tiny = make_workload("tiny4")
ref = orc.electron_repulsion_integral(tiny, notation="chemist", reorder="exponent")
res["tiny4"] = float(np.abs(er.electron_repulsion_integral(tiny, notation="chemist") - ref).max())

# every class with l <= 3 (s, p, d, f; Cartesian and spherical shells)
z = load_npz("mixed.npz")
mixed_shells = shells_from_json(z["shells"])
got = er.ElectronRepulsionIntegral(mixed_shells).construct_array_spherical()
truth = expand_unique(int(z["sph_n"]), z["sph_truth"])
ref_err = float(np.abs(expand_unique(int(z["sph_n"]), z["sph"]) - truth).max())
res["mixed_sph"] = float(np.abs(got - truth).max())
res["mixed_sph_bar"] = max(1e-12, 4.0 * ref_err)  # the reference's own error on this basis

# mixed form with left-out quartets (work-list build, FP32 list, zero fill)
box = make_workload("large64")[:30]
db = _engine.DeviceBasis(box)
n = db.nbf
a64 = torch.empty(n ** 4, dtype=torch.float64, device="cuda")
amx = torch.empty_like(a64)
db.full_device(a64.data_ptr())
db.full_device(amx.data_ptr(), mixed=(MIXED_SKIP, MIXED_FP32))
torch.cuda.synchronize()
res["mixed_form_left_out"] = db.mixed_counts()[2]
res["mixed_form"] = float((amx - a64).abs().max())
T = a64.view(n, n, n, n)
rng = np.random.default_rng(5)
X = rng.standard_normal((n, n // 4))
D = X @ X.T / n
Dt = torch.from_numpy(D).cuda()
j_ref = torch.einsum("abcd,cd->ab", T, Dt).cpu().numpy()
k_ref = torch.einsum("abcd,bd->ac", T, Dt).cpu().numpy()
db.close()
J, K = coulomb_exchange(box, D)
res["jk"] = max(float(np.abs(J - j_ref).max()), float(np.abs(K - k_ref).max()))
res["direct_j"] = float(np.abs(coulomb_matrix(box, D, schwarz_threshold=0.0) - j_ref).max())

# a batch: per-type kernels and the multi-class queue
mols = [batch_molecule(m) for m in range(6)]
outs = {}
for queue in (False, True):
    b = EriBatch(mols)
    b.set_queue(queue)
    o = [torch.empty((k,) * 4, dtype=torch.float64, device="cuda") for k in b.nbf]
    b.run(o)
    torch.cuda.synchronize()
    outs[queue] = o
    b.close()
single = []
for shells, t in zip(mols, outs[False]):
    single.append(float(np.abs(t.cpu().numpy() - er.electron_repulsion_integral(shells, notation="chemist")).max()))
res["batch_vs_single"] = max(single)
res["queue_vs_per_type"] = max(float((a - b).abs().max()) for a, b in zip(outs[True], outs[False]))
print(json.dumps(res))
"""


def test_debug_bounds_build_runs_clean():
    if not os.path.exists(DEBUG_LIB):
        pytest.skip("libgbx_eri_debug.so is not built (python -m gbasis_b200.build --debug-bounds)")
    env = dict(os.environ, GBX_DEBUG_BOUNDS="1")
    r = subprocess.run([sys.executable, "-c", CHILD], env=env, cwd=ROOT, capture_output=True,
                       text=True, timeout=1200)
    assert r.returncode == 0, (r.stdout[-3000:], r.stderr[-3000:])
    res = json.loads(r.stdout.strip().splitlines()[-1])
    print(res)
    assert res["lib"].endswith("libgbx_eri_debug.so") and res["checks_on"] == 1
    assert res["tiny4"] <= 1e-12
    assert res["mixed_sph"] <= res["mixed_sph_bar"]
    assert res["mixed_form_left_out"] > 0 and res["mixed_form"] <= 1e-10
    assert res["jk"] <= 1e-10 and res["direct_j"] <= 1e-10
    assert res["batch_vs_single"] <= 1e-12
    assert res["queue_vs_per_type"] <= 1e-7
