"""Generate recursion programs for the cooperative (warp-per-quartet) ERI kernel.

Heavy classes — whose [e0|f0] accumulators and HRR intermediates do not fit in one thread's
registers — are evaluated by a warp that interprets a per-class program level by level in
shared memory.  For each class this writes, into ``coop_programs.cu``:

* the VRR program (Obara-Saika on centre A, nodes (e, m)) and the electron-transfer program
  (nodes (e, f)) as lists of instructions grouped by dependency level;
* the target list mapping every contracted [e0|f0] (e in [la, la+lb], f in [lc, lc+ld]) to
  its node;
* the ket HRR program (per row e: nodes (c, d), leaves f) and the bra HRR program (per
  column: nodes (a, b), leaves e), with the node of every final component.

Instruction (8 x int16): dst, s1, s2, s3, s4, dir, k1, k2 — see ``coop_kernel.cu`` for the
three formulas.  The recursion choices (directions) are the same closures as ``gen_eri.py``.
"""
from __future__ import annotations

import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import gen_eri as G  # noqa: E402


def _levels(nodes_order, depth):
    """Group instructions by dependency depth; returns (instrs sorted, level offsets)."""
    by = {}
    for ins in nodes_order:
        by.setdefault(depth[ins[0]], []).append(ins)
    out, lv = [], [0]
    for d in sorted(by):
        out += by[d]
        lv.append(len(out))
    return out, lv


def program(la, lb, lc, ld):
    g = G.best_prim(la, lb, lc, ld)
    L = la + lb + lc + ld
    # ---- VRR nodes: (e, m); leaves (0, m) get indices 0..L
    vidx = {}
    for m in range(L + 1):
        if ((0, 0, 0), m) in g.vrr:
            vidx[((0, 0, 0), m)] = m
    # ensure leaves 0..L exist as slots even if unused
    nxt = L + 1
    vorder = sorted((k for k, v in g.vrr.items() if v is not None),
                    key=lambda k: (sum(k[0]), -k[1]))
    for k in vorder:
        vidx[k] = nxt
        nxt += 1
    nV = nxt
    vdepth = {}
    vins = []
    for (e, m) in vorder:
        i = g.vrr[(e, m)]
        e1 = G.add(e, i, -1)
        d = vidx[(e, m)]
        s1, s2 = vidx[(e1, m)], vidx[(e1, m + 1)]
        if e1[i] > 0:
            e2 = G.add(e1, i, -1)
            s3, s4, k = vidx[(e2, m)], vidx[(e2, m + 1)], e1[i]
        else:
            s3 = s4 = -1
            k = 0
        dep = 1 + max(vdepth.get(s, 0) for s in (s1, s2, s3, s4) if s >= 0)
        vdepth[d] = dep
        vins.append((d, s1, s2, s3, s4, i, k, 0))
    vins, vlv = _levels(vins, vdepth)
    # ---- ETR nodes: (e, f), leaves (e, 0) are VRR nodes (e, 0)
    def xidx(e, f):
        if sum(f) == 0:
            return vidx[(e, 0)]
        return tidx[(e, f)]
    tidx = {}
    torder = sorted((k for k, v in g.etr.items() if v is not None), key=lambda k: sum(k[1]))
    for k in torder:
        tidx[k] = nxt
        nxt += 1
    nX = nxt
    tdepth = {}
    tins = []
    for (e, f) in torder:
        i = g.etr[(e, f)]
        f1 = G.add(f, i, -1)
        d = tidx[(e, f)]
        s1 = xidx(e, f1)
        s2 = xidx(G.add(e, i), f1)
        s3 = xidx(G.add(e, i, -1), f1) if e[i] > 0 else -1
        s4 = xidx(e, G.add(f1, i, -1)) if f1[i] > 0 else -1
        dep = 1 + max(tdepth.get(s, 0) for s in (s1, s2, s3, s4) if s >= 0)
        tdepth[d] = dep
        tins.append((d, s1, s2, s3, s4, i, e[i] if s3 >= 0 else 0, f1[i] if s4 >= 0 else 0))
    tins, tlv = _levels(tins, tdepth)
    targets = [xidx(e, f) for e in g.E for f in g.F]
    # ---- ket HRR (per row): leaves f in F order, nodes (c, d)
    kn = G.HrrGen.closure(lc, G.comps(lc), G.comps(ld), G.pick_first)
    kidx = {(c, (0, 0, 0)): j for j, c in enumerate(g.F)}
    knxt = len(g.F)
    korder = sorted((k for k, v in kn.items() if v is not None), key=lambda k: sum(k[1]))
    for k in korder:
        kidx[k] = knxt
        knxt += 1
    kdepth, kins = {}, []
    for (c, d) in korder:
        i = kn[(c, d)]
        d1 = G.add(d, i, -1)
        s1, s2 = kidx[(G.add(c, i), d1)], kidx[(c, d1)]
        dep = 1 + max(kdepth.get(s1, 0), kdepth.get(s2, 0))
        kdepth[kidx[(c, d)]] = dep
        kins.append((kidx[(c, d)], s1, s2, -1, -1, i, 0, 0))
    kins, klv = _levels(kins, kdepth)
    kfin = [kidx[(c, d)] for c in G.comps(lc) for d in G.comps(ld)]
    # ---- bra HRR (per column): leaves e in E order, nodes (a, b)
    bn = G.HrrGen.closure(la, G.comps(la), G.comps(lb), G.pick_first)
    bidx = {(e, (0, 0, 0)): j for j, e in enumerate(g.E)}
    bnxt = len(g.E)
    border = sorted((k for k, v in bn.items() if v is not None), key=lambda k: sum(k[1]))
    for k in border:
        bidx[k] = bnxt
        bnxt += 1
    bdepth, bins = {}, []
    for (a, b) in border:
        i = bn[(a, b)]
        b1 = G.add(b, i, -1)
        s1, s2 = bidx[(G.add(a, i), b1)], bidx[(a, b1)]
        dep = 1 + max(bdepth.get(s1, 0), bdepth.get(s2, 0))
        bdepth[bidx[(a, b)]] = dep
        bins.append((bidx[(a, b)], s1, s2, -1, -1, i, 0, 0))
    bins, blv = _levels(bins, bdepth)
    bfin = [bidx[(a, b)] for a in G.comps(la) for b in G.comps(lb)]
    return dict(cls=(la, lb, lc, ld), L=L, NE=len(g.E), NF=len(g.F), nV=nV, nX=nX,
                vins=vins, vlv=vlv, tins=tins, tlv=tlv, targets=targets,
                kins=kins, klv=klv, nK=knxt, kfin=kfin, bins=bins, blv=blv, nB=bnxt, bfin=bfin)


def emit(classes, path, n_heavy=None):
    """Programs of ``classes``; the first ``n_heavy`` (default: all) are the heavy classes that
    the cooperative kernels run per class block; the rest serve the multi-class queue kernel."""
    n_heavy = len(classes) if n_heavy is None else n_heavy
    ins, lv, idx = [], [], []
    metas = []
    for c in classes:
        p = program(*c)
        m = {"cls": c, "L": p["L"], "NE": p["NE"], "NF": p["NF"], "nX": p["nX"],
             "nK": p["nK"], "nB": p["nB"]}
        for key in ("v", "t", "k", "b"):
            m[key + "_ins"] = len(ins)
            ins += p[key + "ins"]
            m[key + "_lv"] = len(lv)
            m[key + "_nlv"] = len(p[key + "lv"]) - 1
            lv += p[key + "lv"]
        for key in ("targets", "kfin", "bfin"):
            m[key] = len(idx)
            idx += p[key]
        m["n_ins"] = len(ins) - m["v_ins"]
        m["n_idx"] = len(idx) - m["targets"]
        metas.append(m)
    import math
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
    from gbasis_b200.spherical import engine_sph_matrix
    sph = list(engine_sph_matrix(2).ravel()) + list(engine_sph_matrix(3).ravel())
    cn = []
    for l in range(4):
        v = [1.0 / math.sqrt(G._dfact(2 * a - 1) * G._dfact(2 * b - 1) * G._dfact(2 * c - 1))
             for a, b, c in G.comps(l)]
        cn += v + [0.0] * (10 - len(v))
    lines = ["// Generated by gen_coop.py: recursion programs of the cooperative ERI kernel.",
             "#pragma once",
             '#include "coop.cuh"', "namespace gbx {",
             f"__device__ const double kCoopSph[{len(sph)}] = {{{', '.join(repr(float(v)) for v in sph)}}};",
             f"__device__ const double kCoopCn[40] = {{{', '.join(repr(float(v)) for v in cn)}}};",
             f"__device__ const short kCoopIns[{max(1, len(ins))}][8] = {{"]
    lines += ["  {" + ", ".join(str(v) for v in i) + "}," for i in ins] or ["  {0},"]
    lines.append("};")
    lines.append(f"__device__ const int kCoopLv[{max(1, len(lv))}] = {{{', '.join(map(str, lv)) or '0'}}};")
    lines.append(f"__device__ const short kCoopIdx[{max(1, len(idx))}] = {{{', '.join(map(str, idx)) or '0'}}};")
    lines.append(f"const int kCoopNumClasses = {len(metas)};")
    lines.append(f"const int kCoopNumHeavy = {n_heavy};")
    lines.append("const CoopMeta kCoopMeta[] = {")
    for m in metas:
        la, lb, lc, ld = m["cls"]
        lines.append(
            "  {%d, %d, %d, %d, %d, %d, %d, %d, %d, %d, "
            "%d, %d, %d, %d, %d, %d, %d, %d, %d, %d, %d, %d, %d, %d, %d, %d, %d}," % (
                la, lb, lc, ld, m["L"], m["NE"], m["NF"], m["nX"], m["nK"], m["nB"],
                m["v_ins"], m["v_lv"], m["v_nlv"], m["t_ins"], m["t_lv"], m["t_nlv"],
                m["k_ins"], m["k_lv"], m["k_nlv"], m["b_ins"], m["b_lv"], m["b_nlv"],
                m["targets"], m["kfin"], m["bfin"], m["n_ins"], m["n_idx"]))
    lines.append("};")
    lines.append("}  // namespace gbx")
    text = "\n".join(lines) + "\n"
    if not (os.path.exists(path) and open(path).read() == text):
        with open(path, "w") as f:
            f.write(text)
    return metas
