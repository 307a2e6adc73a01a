"""Throughput of the ERI engine on the 8-atom, 120-function workload (FP64 form).

One step = one full-tensor call: the 120^4 float64 ERI tensor (1.66 GB) of the ``medium8``
synthetic basis (8 atoms in a 10-bohr box; per atom s(6), s(3), s(1), p(3), p(1), d(1);
Cartesian; physicist notation as a view of the chemist array, as gbasis returns it).

* ``value``: unique contracted ERIs per second with the basis resident in HBM (device time of
  K steps with CUDA events, max over ranks).
* ``e2e``: the same metric through the public API ``electron_repulsion_integral`` with host
  buffers: basis packing + upload (H2D) and the full tensor copied back to page-locked host
  memory (D2H) inside every step.
* ``roofline``: the dominant kernel phase against its bound (class kernels: FP64 FMA pipe,
  peak measured live by ``gbx_fp64_peak``; expansion: HBM, peak from MEASURED_PEAKS.json).
* ``cpu_baseline``: the CPU oracle (a NumPy restatement of gbasis's algorithm) on 1 core over
  one interleaved 1/64 slice of the workload's unique shell quartets, measured (unique ERIs of
  the slice over its time; chain20's line in ``configs`` samples random quartets instead).

``--impl reference`` times that CPU implementation on all host cores instead (every step a
measured slice of the workload) and prints the same metric with ``"impl": "reference"``.  For N > 1 GPUs every rank computes the
same workload (independent replicas: a full-tensor call needs no exchange between GPUs) and
``value`` aggregates.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "medium8"
METRIC = "unique contracted ERIs/s (FP64 full tensor)"
UNIT = "ERI/s"
# DRAM bytes of one expand_rows launch on medium8 from an ncu capture (404.8 MB read +
# 1,599.4 MB written); the algorithmic bytes are 1,913.5 MB
EXPAND_TRAFFIC_BYTES = 404.778752e6 + 1599.436e6


HBM_FALLBACK_GBS = 6650.0  # copy bandwidth measured earlier on a B200 of the same kind
REF_SLICES = 64  # CPU legs: one step = one interleaved 1/64 slice of the unique shell quartets


def _peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        return {}


class ClockSampler:
    """SM clock and clock-event (throttle) reasons of the benchmarked GPU, sampled every
    ``period`` seconds through NVML from a background thread during the timed region (the
    GPU is matched to the CUDA device by UUID).  Read-only: no clock or setting changes."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, index, period=0.005):
        self.index, self.period = index, period
        self.samples, self.reasons, self.max_mhz = [], set(), None
        self._stop = None
        self._thread = None

    def _handle(self, nv):
        import torch
        want = str(torch.cuda.get_device_properties(self.index).uuid).lower()
        for i in range(nv.nvmlDeviceGetCount()):
            h = nv.nvmlDeviceGetHandleByIndex(i)
            u = nv.nvmlDeviceGetUUID(h)
            u = (u.decode() if isinstance(u, bytes) else u).lower()
            if want and want in u:
                return h
        return nv.nvmlDeviceGetHandleByIndex(self.index)

    def _run(self, nv, h):
        masks = [(name, getattr(nv, attr)) for name, attr in self.REASONS]
        while not self._stop.is_set():
            try:
                self.samples.append(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM))
                r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                for name, m in masks:
                    if r & m:
                        self.reasons.add(name)
            except Exception:
                pass
            self._stop.wait(self.period)

    def __enter__(self):
        import threading
        try:
            import pynvml as nv
            nv.nvmlInit()
            h = self._handle(nv)
            self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            self._stop = threading.Event()
            self._thread = threading.Thread(target=self._run, args=(nv, h), daemon=True)
            self._thread.start()
            t0 = time.perf_counter()
            while not self.samples and time.perf_counter() - t0 < 1.0:
                time.sleep(0.001)
        except Exception:
            self._thread = None
        return self

    def __exit__(self, *a):
        if self._thread is not None:
            self._stop.set()
            self._thread.join(timeout=5)

    def summary(self):
        sm = self.samples
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": self.max_mhz,
                "reasons": sorted(self.reasons), "samples": len(sm), "source": "NVML"}


def max_over_ranks(x, dist, device):
    """The largest of every rank's ``x`` (a time); every rank of the group must call it, in the
    same order.  ``dist`` is ``torch.distributed`` or None for a single process."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_throughput(world, units_per_rank, ms):
    """Whole-job units per second of ``world`` independent replicas, each processing
    ``units_per_rank`` units, timed by the slowest rank (``ms`` per step)."""
    return world * units_per_rank / (ms * 1e-3)


def _cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    return ln.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.machine()


def cpu_baseline_slice(shells, n_slices=REF_SLICES, s=0):
    """The oracle on 1 core over one interleaved 1/``n_slices`` slice of the workload's unique
    shell quartets (about 11,000 quartets, 10-15 s for medium8): measured unique ERIs over
    measured time, no extrapolation."""
    from oracle import eri_oracle as orc
    from oracle import parallel as opar
    pairs = opar.unique_pairs(len(shells))
    nq = opar.quartet_count(len(shells))
    q = opar.slice_quartets(pairs, nq, s, n_slices)
    t0 = time.perf_counter()
    for i, j, k, l in q:
        blk = orc.construct_array_contraction(shells[i], shells[j], shells[k], shells[l])
        for ax, x in enumerate((i, j, k, l)):  # norm_cont, as base_four_symm.py:195-205
            shape = [1] * 8
            shape[2 * ax:2 * ax + 2] = np.shape(shells[x].norm_cont)
            blk = blk * np.asarray(shells[x].norm_cont).reshape(shape)
    dt = time.perf_counter() - t0
    eris = opar.unique_eri_count(shells, q)
    return {"value": eris / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "host_cpus": os.cpu_count(), "cpu_model": _cpu_model(),
            "sample": f"slice {s} of {n_slices} of the {nq} unique shell quartets ({len(q)} "
                      f"quartets, {eris} unique ERIs, {dt:.1f} s; oracle "
                      f"construct_array_contraction, 1 core), measured"}


def cpu_baseline(shells, seconds=12.0, seed=0, n_functions=None):
    """Oracle on a seeded random sample of unique shell quartets, extrapolated (unique ERIs
    counted over ``n_functions``, default the Cartesian functions)."""
    import itertools
    from oracle import eri_oracle as orc
    pairs = list(itertools.combinations_with_replacement(range(len(shells)), 2))
    npair = len(pairs)
    nq = npair * (npair + 1) // 2
    rng = np.random.default_rng(seed)
    t0 = time.perf_counter()
    done = 0
    while time.perf_counter() - t0 < seconds:
        p, q = sorted(rng.integers(0, npair, size=2))
        (i, j), (k, l) = pairs[p], pairs[q]
        orc.construct_array_contraction(shells[i], shells[j], shells[k], shells[l])
        done += 1
    dt = time.perf_counter() - t0
    n = n_functions or sum(len(s.angmom_components_cart) for s in shells)
    from gbasis_b200.flops import unique_eris
    est_total = dt / done * nq
    return {"value": unique_eris(n) / est_total, "unit": UNIT, "cores": 1, "kind": "port",
            "host_cpus": os.cpu_count(), "cpu_model": _cpu_model(),
            "sample": f"{done} random unique shell quartets of {nq} ({dt:.1f} s, "
                      f"oracle construct_array_contraction, 1 core), extrapolated"}


def engine_config(n, nq, n_unique, compact_bytes=None, world=1):
    """The ``config`` of the headline line, shared by both arms."""
    cfg = {"workload": WORKLOAD, "n_functions": n, "shell_quartets": nq, "unique_eris": n_unique,
           "notation": "physicist", "coord_type": "cartesian", "form": "fp64",
           "parallelism": "replicas" if world > 1 else "single"}
    if compact_bytes is not None:
        cfg["l2"] = ("working set above L2 (1.66 GB tensor, "
                     f"{compact_bytes / 1e6:.0f} MB compact store)")
    return cfg


def run_reference(a, rank, world):
    """The CPU implementation of the path (the oracle port of gbasis's per-quartet integrals,
    with gbasis's norm_cont scaling) on every host core.  Each step is measured, not
    extrapolated: step s computes slice s mod 64 of the workload's unique shell quartets (the
    quartets at loop positions congruent to s, so every slice has the workload's class mix)
    over a spawned process pool, and the step's unique ERIs are counted exactly.  ``value``
    = unique ERIs of the timed steps / their wall time."""
    if rank != 0:
        return
    from gbasis_b200.synthetic import make_workload
    from gbasis_b200.flops import unique_eris
    from oracle import parallel as opar
    shells = make_workload(WORKLOAD)
    n = sum(len(s.angmom_components_cart) for s in shells)
    pairs = opar.unique_pairs(len(shells))
    nq = opar.quartet_count(len(shells))
    pool = opar.SlicePool(WORKLOAD)
    cores = pool.processes
    times, eris, quartets = [], 0, 0
    try:
        for step in range(a.warmup + a.steps):
            q = opar.slice_quartets(pairs, nq, step, REF_SLICES)
            dt = pool.run(q)
            if step >= a.warmup:
                times.append(dt)
                eris += opar.unique_eri_count(shells, q)
                quartets += len(q)
    finally:
        pool.close()
    total = float(sum(times))
    v = eris / total
    cfg = engine_config(n, nq, unique_eris(n), world=world)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": world,
            "steps": a.steps, "warmup": a.warmup, "ms_per_step": total / len(times) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                             "cpu_model": _cpu_model(),
                             "sample": f"{a.steps} timed steps, each one interleaved 1/{REF_SLICES} "
                                       f"slice of the {nq} unique shell quartets ({quartets} "
                                       f"quartets, {eris} unique ERIs in all), measured, "
                                       f"{cores} processes"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def extra_configs(local, reps=2, large_atoms=16,
                  which=("chain20", "batch512", "large64")):
    """The other configurations of the path, each timed on the device with CUDA events on the
    launching stream (one warm-up call, then ``reps`` calls):

    * ``chain20_unique``: 20-atom random-walk chain, 140 spherical shells (s,s,s,p,p,d,f per
      atom), N = 420; the 8-fold unique integrals only (no N^4 tensor), FP64 and mixed form,
      with the mixed form's max error over the whole compact store;
    * ``batch512``: 512 molecules of 2-14 atoms, one CUDA graph per run (every molecule's full
      Cartesian tensor, device resident), FP64 and mixed form side by side;
    * ``large64_coulomb``: direct Coulomb matrix of the 64-atom box's first ``large_atoms``
      atoms (default 16: 160 spherical shells, N = 480; 64 is the whole box, 640 shells,
      N = 1920), FP64 and mixed form, with the screened fraction and the mixed J's error.
    """
    import ctypes
    import torch
    from gbasis_b200 import _engine
    from gbasis_b200.autotune import light_class
    from gbasis_b200.batch import EriBatch
    from gbasis_b200.electron_repulsion import MIXED_FP32, MIXED_SKIP
    from gbasis_b200.flops import basis_flops, unique_eris
    from gbasis_b200.synthetic import density_matrix, make_workload
    dev = torch.device("cuda", local)
    st = torch.cuda.current_stream(dev)
    sp = ctypes.c_void_p(st.cuda_stream)
    peak64 = _engine.fp64_peak(local)

    def timed(fn, n=None, warm=True):
        n = reps if n is None else n
        if warm:
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(st)
        for _ in range(n):
            fn()
        e1.record(st)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n

    out = {}
    if "chain20" in which:
        shells = make_workload("chain20")
        db = _engine.DeviceBasis(shells, device=local)
        uq, fl = unique_eris(db.nbf), basis_flops(shells)
        ms64 = timed(lambda: db.unique(stream=sp))
        ref = db.compact_view().clone()
        msmx = timed(lambda: db.unique((MIXED_SKIP, MIXED_FP32), stream=sp))
        cur = db.compact_view()
        max_abs = max_rel = 0.0
        for c0 in range(0, ref.numel(), 1 << 27):
            r, x = ref[c0:c0 + (1 << 27)], cur[c0:c0 + (1 << 27)]
            d = (x - r).abs()
            max_abs = max(max_abs, float(d.max()))
            max_rel = max(max_rel, float((d / r.abs().clamp_min(1e-8)).max()))
        out["chain20_unique"] = {
            "n_functions": db.nbf, "unique_eris": uq, "shell_quartets": db.stats()[0],
            "fp64": {"ms": ms64, "value": uq / (ms64 * 1e-3), "unit": UNIT,
                     "achieved_tflops": fl / (ms64 * 1e-3) / 1e12, "frac_fp64_peak": fl / (ms64 * 1e-3) / 1e12 / peak64},
            "mixed": {"ms": msmx, "value": uq / (msmx * 1e-3), "unit": UNIT, "speedup_vs_fp64": ms64 / msmx,
                      "max_abs_err_vs_fp64": max_abs, "max_rel_err_vs_fp64": max_rel,
                      "error_over": "every unique integral", "skip_bound": MIXED_SKIP,
                      "fp32_bound": MIXED_FP32}}
        del ref, cur, r, x, d
        try:  # the oracle's Cartesian blocks on a sample of this workload's quartets, 1 core
            out["chain20_unique"]["cpu_baseline"] = cpu_baseline(shells, seconds=8.0, seed=3,
                                                                 n_functions=db.nbf)
        except Exception as exc:
            out["chain20_unique"]["cpu_baseline"] = {"error": str(exc)[:300]}
        db.close()
        torch.cuda.empty_cache()

    if "batch512" in which:
        mols = make_workload("batch512")
        t0 = time.perf_counter()
        b = EriBatch(mols, device=local)
        t_create = time.perf_counter() - t0
        outs = [torch.empty((n,) * 4, dtype=torch.float64, device=dev) for n in b.nbf]
        ms = timed(lambda: b.run(outs, stream=sp))
        uq = sum(unique_eris(n) for n in b.nbf)
        fl = sum(basis_flops(m) for m in mols)
        out["batch512"] = {
            "molecules": len(mols), "unique_eris": uq, "shell_quartets": b.n_quartets,
            "tensor_bytes": 8 * sum(n ** 4 for n in b.nbf), "ms": ms,
            "value": uq / (ms * 1e-3), "unit": UNIT, "molecules_per_s": len(mols) / (ms * 1e-3),
            "achieved_tflops": fl / (ms * 1e-3) / 1e12, "frac_fp64_peak": fl / (ms * 1e-3) / 1e12 / peak64,
            "create_s": t_create, "launch": "one CUDA graph replay per run"}
        try:  # the same block types one after another with events between them (no overlap)
            Lb = _engine.lib()
            _engine.check(Lb.gbx_batch_set_profiling(b.handle, 1))
            b.run(outs, stream=sp)
            torch.cuda.synchronize()
            tms = np.zeros(len(b.types()))
            _engine.check(Lb.gbx_batch_type_times(b.handle, tms.ctypes.data_as(ctypes.c_void_p), len(tms)))
            _engine.check(Lb.gbx_batch_set_profiling(b.handle, 0))
            out["batch512"]["types_serial_ms"] = float(tms.sum())
            out["batch512"]["heavy_types_serial_ms"] = float(sum(
                t for (c4, _, _, _), t in zip(b.types(), tms) if not light_class(c4)))
        except Exception as exc:
            out["batch512"]["types_serial_ms"] = {"error": str(exc)[:200]}
        # mixed form of the same batch, side by side (its own graph); error against the FP64
        # tensors of every 8th molecule with N <= 80
        try:
            th = (MIXED_SKIP, MIXED_FP32)
            sample = [m for m in range(0, len(mols), 8) if b.nbf[m] <= 80]
            ref = {m: outs[m].clone() for m in sample}
            t0 = time.perf_counter()
            b.run(outs, stream=sp, mixed=th)  # first mixed run: bounds and lists
            torch.cuda.synchronize()
            t_setup = time.perf_counter() - t0
            ms_mx = timed(lambda: b.run(outs, stream=sp, mixed=th))
            err = max(float((outs[m] - ref[m]).abs().max()) for m in sample)
            n64, n32, nskip = b.mixed_counts()
            out["batch512"]["mixed"] = {
                "ms": ms_mx, "value": uq / (ms_mx * 1e-3), "unit": UNIT,
                "speedup_vs_fp64": ms / ms_mx, "max_abs_err_vs_fp64": err,
                "error_over": f"full tensors of {len(sample)} molecules (every 8th with N <= 80)",
                "quartets_fp64": n64, "quartets_fp32": n32, "quartets_left_out": nskip,
                "first_run_s": t_setup, "skip_bound": MIXED_SKIP, "fp32_bound": MIXED_FP32}
            del ref
        except Exception as exc:  # keep the rest of the line
            out["batch512"]["mixed"] = {"error": str(exc)[:300]}
        # the multi-class queue form: one persistent launch for every block type (then the
        # batched expansion), captured and replayed like the per-type graph; its largest
        # difference from the per-type kernels' tensors over the same sampled molecules
        try:
            sample = [m for m in range(0, len(mols), 8) if b.nbf[m] <= 80]
            b.run(outs, stream=sp)
            torch.cuda.synchronize()
            ref = {m: outs[m].clone() for m in sample}
            b.set_queue(True)
            ms_q = timed(lambda: b.run(outs, stream=sp))
            diff = max(float((outs[m] - ref[m]).abs().max()) for m in sample)
            b.set_queue(False)
            out["batch512"]["queue"] = {
                "ms": ms_q, "value": uq / (ms_q * 1e-3), "unit": UNIT,
                "speedup_vs_per_type_graph": ms / ms_q, "max_abs_diff_vs_per_type": diff,
                "launch": "one persistent multi-class queue kernel + expansion, one graph replay",
                "default": "per-type graph" if ms <= ms_q else "queue"}
            del ref
        except Exception as exc:
            out["batch512"]["queue"] = {"error": str(exc)[:300]}
        b.close()
        del outs
        torch.cuda.empty_cache()

    if "large64" in which:
        # config 5: the 64-atom box (its first `large_atoms` atoms unless 64), direct J only (the
        # unique integrals of the whole box would take 13.6 TB)
        shells = make_workload("large64")[: 10 * large_atoms]
        t0 = time.perf_counter()
        db = _engine.DeviceBasis(shells, device=local)
        t_create = time.perf_counter() - t0
        n = db.nbf
        D = torch.from_numpy(density_matrix(n)).to(dev)
        J = torch.empty((n, n), dtype=torch.float64, device=dev)
        Jm = torch.empty((n, n), dtype=torch.float64, device=dev)
        L = _engine.lib()
        tau = 1e-12

        def coulomb():
            _engine.check(L.gbx_eri_coulomb_j(db.handle, ctypes.c_void_p(D.data_ptr()), tau,
                                              ctypes.c_void_p(J.data_ptr()), sp), "gbx_eri_coulomb_j")

        def coulomb_mixed():
            _engine.check(L.gbx_eri_coulomb_j_mixed(
                db.handle, ctypes.c_void_p(D.data_ptr()), MIXED_SKIP, MIXED_FP32,
                ctypes.c_void_p(Jm.data_ptr()), sp), "gbx_eri_coulomb_j_mixed")
        # the whole box (minutes per call) is timed on its first call: that call also computes the
        # Schwarz bounds and allocates the work buffers, well under a second of it
        warm = large_atoms <= 16
        ms = timed(coulomb, 1, warm)
        computed, screened = db.last_counts()
        ms_mx = timed(coulomb_mixed, 1, warm)
        computed_mx, skipped_mx = db.last_counts()
        dj = float((Jm - J).abs().max())
        out["large64_coulomb"] = {
            "atoms": large_atoms, "shells": len(shells), "n_functions": n, "coord_type": "spherical",
            "candidate_quartets": computed + screened, "schwarz_threshold": tau,
            "fp64": {"ms": ms, "quartets_computed": computed,
                     "screened_fraction": screened / max(1, computed + screened),
                     "quartets_per_s": computed / (ms * 1e-3),
                     "unit": "screened unique shell quartets/s"},
            "mixed": {"ms": ms_mx, "quartets_computed": computed_mx,
                      "quartets_per_s": computed_mx / (ms_mx * 1e-3), "speedup_vs_fp64": ms / ms_mx,
                      "max_abs_J_err_vs_fp64": dj, "max_abs_J": float(J.abs().max()),
                      "skip_bound": MIXED_SKIP, "fp32_bound": MIXED_FP32},
            "density": "D = X X^T / ||X X^T||, X seeded normal N x N/4", "create_s": t_create,
            "warm_up_call": warm}
        db.close()
        torch.cuda.empty_cache()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-extra-configs", action="store_true",
                    help="skip the chain20 / batch512 / large64 measurements")
    ap.add_argument("--configs", default="chain20,batch512,large64",
                    help="which secondary configurations to measure (comma-separated)")
    ap.add_argument("--large64-atoms", type=int, default=16,
                    help="atoms of the 64-atom box in the direct-J configuration (64: the whole "
                         "box: 6 minutes per J on one B200, FP64 and mixed)")
    a = ap.parse_args()

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if a.impl == "reference":
        return run_reference(a, rank, world)

    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    from gbasis_b200 import _engine
    from gbasis_b200 import electron_repulsion as er
    from gbasis_b200.flops import basis_flops, unique_eris
    from gbasis_b200.synthetic import make_workload

    shells = make_workload(WORKLOAD)
    n = sum(len(s.angmom_components_cart) for s in shells)
    n_unique = unique_eris(n)
    flops = basis_flops(shells)
    dev = torch.device("cuda", local)
    db = _engine.DeviceBasis(shells, device=local)
    nq, compact_bytes = db.stats()
    out = torch.empty(n ** 4, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    sp = __import__("ctypes").c_void_p(stream.cuda_stream)

    def step():
        db.full_device(out.data_ptr(), "chemist", 0.0, stream=sp)

    for _ in range(max(3, a.warmup)):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        e0.record(stream)
        for _ in range(a.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1) / a.steps, dist, dev)
    value = replica_throughput(world, n_unique, ms)

    # mixed-precision form on the same workload, and its error against the FP64 tensor
    from gbasis_b200.electron_repulsion import MIXED_FP32, MIXED_SKIP
    ref = out.clone()
    mixed_args = (MIXED_SKIP, MIXED_FP32)

    def step_mixed():
        db.full_device(out.data_ptr(), "chemist", 0.0, stream=sp, mixed=mixed_args)

    for _ in range(max(3, a.warmup)):
        step_mixed()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(a.steps):
        step_mixed()
    e1.record(stream)
    torch.cuda.synchronize()
    ms_mixed = e0.elapsed_time(e1) / a.steps
    q64, q32, qleft = db.mixed_counts()
    err = (out - ref).abs()
    mixed = {"value": world * n_unique / (ms_mixed * 1e-3), "unit": UNIT, "ms_per_step": ms_mixed,
             "speedup_vs_fp64": ms / ms_mixed, "max_abs_err_vs_fp64": float(err.max()),
             "max_rel_err_vs_fp64": float((err / ref.abs().clamp_min(1e-8)).max()),
             "skip_bound": MIXED_SKIP, "fp32_bound": MIXED_FP32,
             "quartets_fp64": q64, "quartets_fp32": q32, "quartets_left_out": qleft}
    del ref, err

    # per-phase device times (events on the same stream), a separate pass of the same call
    db.set_profiling(True)
    ph = np.zeros(3)
    for _ in range(a.steps):
        step()
        ph += db.phase_times()
    ph /= a.steps
    db.set_profiling(False)
    peak64 = _engine.fp64_peak(local)
    peaks = _peaks()
    hbm = peaks.get("hbm_gbs")
    hbm_source = "MEASURED_PEAKS.json hbm_gbs (of measured)"
    if not hbm:
        # no measured copy bandwidth on this machine: the earlier B200 measurement
        hbm, hbm_source = HBM_FALLBACK_GBS, "fallback 6650 GB/s copy bandwidth (of fallback)"
    compute_tf = flops / (ph[1] * 1e-3) / 1e12
    exp_bytes = 8.0 * n ** 4 + compact_bytes  # tensor written + compact store read once
    exp_gbs = exp_bytes / (ph[2] * 1e-3) / 1e9
    roof_compute = {"kernel": "class kernels (eri_block, eri_split, eri_lines; all class blocks, concurrent)", "bound": "fp64", "achieved": compute_tf,
                    "peak": peak64, "unit": "TFLOP/s", "frac": compute_tf / peak64,
                    "peak_source": "gbx_fp64_peak dependent-FMA probe, measured live",
                    "traffic": None, "ms": ph[1], "algorithmic_flops": flops}
    roof_expand = {"kernel": "expand_rows", "bound": "hbm", "achieved": exp_gbs, "peak": hbm,
                   "unit": "GB/s", "frac": (exp_gbs / hbm) if hbm else None,
                   "peak_source": hbm_source,
                   "traffic": EXPAND_TRAFFIC_BYTES if WORKLOAD == "medium8" else None,
                   "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of one "
                                     "expand_rows launch on this workload (--set full capture)",
                   "ms": ph[2], "algorithmic_bytes": exp_bytes}
    roof = roof_compute if ph[1] >= ph[2] else roof_expand

    # end to end through the public API with host buffers
    pinned = torch.empty(n ** 4, dtype=torch.float64, pin_memory=True).numpy().reshape((n,) * 4)
    pk = _engine.pack_basis(shells)
    h2d = sum(int(v.nbytes) for v in pk.values())
    er.electron_repulsion_integral(shells, out=pinned)  # warm
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(a.e2e_steps):
        res = er.electron_repulsion_integral(shells, out=pinned)
    e2e_s = max_over_ranks((time.perf_counter() - t0) / a.e2e_steps, dist, dev)
    assert res.shape == (n, n, n, n)
    # floor of the host-output path on this machine: one plain device-to-host copy of the
    # tensor's bytes into the same page-locked buffer
    src = out.view(-1)[: n ** 4]
    host = torch.from_numpy(pinned.reshape(-1))
    host.copy_(src, non_blocking=True)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    host.copy_(src, non_blocking=True)
    torch.cuda.synchronize()
    d2h_s = time.perf_counter() - t1
    e2e = {"value": replica_throughput(world, n_unique, e2e_s * 1e3), "unit": UNIT,
           "h2d_bytes_per_step": h2d,
           "d2h_bytes_per_step": 8 * n ** 4, "ms_per_step": e2e_s * 1e3,
           "d2h_copy_floor_ms": d2h_s * 1e3,
           "d2h_copy_gbs": 8 * n ** 4 / d2h_s / 1e9,
           "out": "page-locked array passed as out="}
    # the default call: no out=, the tensor comes back as a new pageable NumPy array
    del res
    t0 = time.perf_counter()
    for _ in range(max(1, a.e2e_steps)):
        res = er.electron_repulsion_integral(shells)
    pg_s = max_over_ranks((time.perf_counter() - t0) / max(1, a.e2e_steps), dist, dev)
    del res
    e2e["pageable_default"] = {"value": replica_throughput(world, n_unique, pg_s * 1e3),
                               "unit": UNIT, "ms_per_step": pg_s * 1e3,
                               "out": "new pageable array (electron_repulsion_integral(basis))"}
    # per-quartet drop-in: one construct_array_contraction call (host shells in, NumPy out)
    cac = {}
    by_l = {}
    for sh in shells:
        by_l.setdefault(sh.angmom, sh)
    for name, q in (("(ss|ss) K=6", [s for s in shells if s.angmom == 0][0]),
                    ("(dd|dd)", by_l[2])):
        quartet = [q] * 4
        er.ElectronRepulsionIntegral.construct_array_contraction(*quartet)
        t0 = time.perf_counter()
        for _ in range(20):
            er.ElectronRepulsionIntegral.construct_array_contraction(*quartet)
        cac[name] = (time.perf_counter() - t0) / 20 * 1e3
    e2e["construct_array_contraction_ms"] = cac

    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": engine_config(n, nq, n_unique, compact_bytes, world),
            "phases_ms": {"work_list": ph[0], "class_kernels": ph[1], "expand": ph[2]},
            "roofline": roof, "roofline_kernels": [roof_compute, roof_expand],
            "e2e": e2e, "clocks": clk.summary(), "mixed": mixed,
            "gpu_launches": None}
    # our kernels per step: work-list build + one per class block + expansion
    line["gpu_launches"] = a.steps * (2 + len(db.blocks()))
    db.close()
    if world == 1 and not a.no_extra_configs:
        del out
        torch.cuda.empty_cache()
        try:  # the secondary configurations never cost the headline line
            line["configs"] = extra_configs(local, large_atoms=a.large64_atoms,
                                           which=tuple(a.configs.split(",")))
        except Exception as exc:
            line["configs"] = {"error": str(exc)[:300]}
    if rank == 0 and not a.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_slice(shells)
    if rank == 0:
        print(json.dumps(line), flush=True)
    db.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
