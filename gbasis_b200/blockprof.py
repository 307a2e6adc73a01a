"""Per-class-block device times of the synthetic workloads, as Markdown tables.

Run: ``python -m gbasis_b200.blockprof medium8 chain20 batch512``.

Each class block (bra pair class x ket pair class; a block type of the batch) is timed with
CUDA events while the blocks run one after another on one stream (profiling level 2; the
batch's per-type events), so a row is the block's kernel time alone.  ``frac`` is the block's
algorithmic FLOPs (``gbasis_b200.flops``: primitive-quartet work times the mean primitive
quartets, plus the HRR) over its time, as a fraction of the FP64 FMA rate measured on the same
device (``gbx_pipe_peak``).  Workloads: ``medium8`` full Cartesian tensor, ``chain20`` unique
integrals (spherical), ``batch512`` every molecule's full tensor (one graph of block types).
"""
from __future__ import annotations

import ctypes
import os
import sys

import numpy as np

from . import _engine
from .flops import canonical, hrr_flops, prim_flops
from .synthetic import make_workload

__all__ = ["block_rows", "kernel_of", "markdown"]


def kernel_of(cls4):
    """Which kernel runs a class's store mode: ``register`` (light classes), ``split``
    (heavy classes whose row ranges fit threads) or ``line``."""
    from .autotune import light_class
    if light_class(cls4):
        return "register"
    here = os.path.join(os.path.dirname(os.path.abspath(__file__)), "csrc")
    if here not in sys.path:
        sys.path.insert(0, here)
    import gen_lines  # the generator that chose the kernels at build time
    return "split" if gen_lines.split_ok(tuple(cls4)) else "line"


def _row(cls4, team, avg, nq, ms, peak):
    c = canonical(*cls4)
    fl = nq * (avg * prim_flops(*c) + hrr_flops(*c))
    return {"class": cls4, "kernel": kernel_of(cls4), "team": team, "avg_prims": avg,
            "quartets": nq, "ms": ms, "tflops": fl / (ms * 1e-3) / 1e12 if ms > 0 else 0.0,
            "frac": fl / (ms * 1e-3) / 1e12 / peak if ms > 0 else 0.0}


def block_rows(workload, peak, device=0):
    """One dict per class block (block type for ``batch512``), slowest first."""
    import torch
    rows = []
    if workload == "batch512":
        from .batch import EriBatch
        b = EriBatch(make_workload("batch512"), device=device)
        outs = [torch.empty((n,) * 4, dtype=torch.float64, device=f"cuda:{device}") for n in b.nbf]
        sp = ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)
        L = _engine.lib()
        b.run(outs, stream=sp)
        _engine.check(L.gbx_batch_set_profiling(b.handle, 1))
        b.run(outs, stream=sp)
        torch.cuda.synchronize(device)
        types = b.types()
        ms = np.zeros(len(types))
        _engine.check(L.gbx_batch_type_times(b.handle, ms.ctypes.data_as(ctypes.c_void_p), len(ms)))
        rows = [_row(c4, t, ap, nq, m, peak) for (c4, t, ap, nq), m in zip(types, ms)]
        b.close()
    elif workload.startswith("large64_j"):
        # direct Coulomb matrix of the 64-atom box's first n atoms (all 64 by default)
        from .synthetic import density_matrix
        atoms = int(workload.split(":")[1]) if ":" in workload else 64
        db = _engine.DeviceBasis(make_workload("large64")[: 10 * atoms], device=device)
        n = db.nbf
        D = torch.from_numpy(density_matrix(n)).to(f"cuda:{device}")
        J = torch.empty((n, n), dtype=torch.float64, device=f"cuda:{device}")
        sp = ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)

        def call():
            _engine.check(_engine.lib().gbx_eri_coulomb_j(
                db.handle, ctypes.c_void_p(D.data_ptr()), 1e-12, ctypes.c_void_p(J.data_ptr()),
                sp), "gbx_eri_coulomb_j")
        call()
        db.set_profiling(2)
        call()
        torch.cuda.synchronize(device)
        ms = db.block_times()
        # block sizes here are the quartets that passed the screening, not the candidates
        rows = [_row(c4, t, ap, nq, m, peak) for (c4, t, ap, nq), m in zip(db.blocks(), ms)]
        db.set_profiling(0)
        db.close()
    else:
        db = _engine.DeviceBasis(make_workload(workload), device=device)
        if workload == "medium8":
            out = torch.empty(db.nbf ** 4, dtype=torch.float64, device=f"cuda:{device}")
            call = lambda: db.full_device(out.data_ptr())  # noqa: E731
        else:
            call = db.unique
        call()
        db.set_profiling(2)
        call()
        torch.cuda.synchronize(device)
        ms = db.block_times()
        rows = [_row(c4, t, ap, nq, m, peak) for (c4, t, ap, nq), m in zip(db.blocks(), ms)]
        db.set_profiling(0)
        db.close()
    torch.cuda.empty_cache()
    return sorted(rows, key=lambda r: -r["ms"])


def markdown(workload, rows, peak):
    tot = sum(r["ms"] for r in rows)
    out = [f"### {workload}: {len(rows)} class blocks, {tot:.3f} ms one after another "
           f"(FP64 FMA peak {peak:.2f} TF/s, measured)", "",
           "| class (bra pair, ket pair) | kernel | lanes per quartet | mean primitive quartets "
           "| shell quartets | ms | share | TF/s | frac of FP64 peak |",
           "|---|---|---|---|---|---|---|---|---|"]
    for r in rows:
        team = r["team"] if r["kernel"] == "register" else "-"
        out.append(f"| {r['class']} | {r['kernel']} | {team} | {r['avg_prims']:.1f} | "
                   f"{r['quartets']} | {r['ms']:.3f} | {r['ms'] / tot:.1%} | {r['tflops']:.2f} | "
                   f"{r['frac']:.3f} |")
    by = {}
    for r in rows:
        by.setdefault(r["kernel"], [0.0, 0.0])
        by[r["kernel"]][0] += r["ms"]
        by[r["kernel"]][1] += r["tflops"] * r["ms"]
    out += ["", "| kernel | blocks' ms | share | TF/s | frac of FP64 peak |", "|---|---|---|---|---|"]
    for k, (ms, tfms) in sorted(by.items(), key=lambda kv: -kv[1][0]):
        out.append(f"| {k} | {ms:.3f} | {ms / tot:.1%} | {tfms / ms:.2f} | {tfms / ms / peak:.3f} |")
    return "\n".join(out) + "\n"


def main(argv):
    peak = _engine.pipe_peak(0)
    for w in argv or ["medium8", "chain20", "batch512"]:
        print(markdown(w, block_rows(w, peak), peak), flush=True)


if __name__ == "__main__":
    main(sys.argv[1:])
