"""Schedules of the line-factorised cooperative kernel for heavy classes (``lines_kernel.cuh``).

One warp evaluates one contracted quartet.  Every recursion of a primitive quartet couples
neighbours along one Cartesian axis only, so it splits into independent 1-D "lines" that a
lane runs entirely in registers:

* VRR x then y (one lane per e_x):  [(ex,ey,0)]^(m)              -> Y
* VRR z, lines (ex, ey):            [(ex,ey,ez)]^(0)              -> W block f = 0
* transfer x, lines (ey, ez):       [e, (fx,0,0)]   table (ex, fx) -> W blocks (fx, 0)
* transfer y, lines (ex, ez), fx:   [e, (fx,fy,0)]  table (ey, fy) -> W blocks (fx, fy)
* transfer z, lines (ex,ey,fx,fy):  [e, f]          table (ez, fz) -> targets, added to ACC

Between stages the values cross shared memory once (W, Y); inside a line they stay in
registers.  The recursion formulas are gbasis's (``gbasis/integrals/_two_elec_int.py:350-526``):
the direction of each step is z if the z component is non-zero, else y, else x.

W holds one tetrahedral block per (fx, fy), fx + fy <= lc + ld, with g = L - fx - fy:
index Zb(fx,fy) + toff(ex, ey, g) + ez over ex + ey + ez <= g, where
toff(ex, ey, g) = tet(g+1) - tet(g+1-ex) + ey (g+1-ex) - ey (ey-1)/2 and tet(k) = k(k+1)(k+2)/6.
Y uses the same layout with m in place of ez (g = L).

A line's extent is pruned to the cells its targets depend on; lanes take lines in rounds of 32
sorted by extent, and each round runs code unrolled to the round's largest extent, with
per-lane predicates.  ``emulate`` runs the same schedule on the host (tests); ``emit`` writes
the per-class device code.
"""
from __future__ import annotations

import functools
import math


def ncart(l):
    return (l + 1) * (l + 2) // 2


def tet(k):
    return k * (k + 1) * (k + 2) // 6


def toff(ex, ey, g):
    u = g + 1
    return tet(u) - tet(u - ex) + ey * (u - ex) - ey * (ey - 1) // 2


def comps(l):
    return [(x, y, l - x - y) for x in range(l, -1, -1) for y in range(l - x, -1, -1)]


def comp_index(c):
    """Index of c within comps(|c|) (canonical order: x descending, then y descending)."""
    ey, ez = c[1], c[2]
    return (ey + ez) * (ey + ez + 1) // 2 + ez


def _rounds(items, key):
    """Lines sorted by extent (descending), cut into rounds of 32."""
    items = sorted(items, key=key, reverse=True)
    return [items[i:i + 32] for i in range(0, len(items), 32)]


class Schedule:
    def __init__(self, la, lb, lc, ld):
        self.cls = (la, lb, lc, ld)
        self.la, self.lb, self.lc, self.ld = la, lb, lc, ld
        L = self.L = la + lb + lc + ld
        F = self.F = lc + ld
        self.emax = la + lb
        self.NE = sum(ncart(l) for l in range(la, la + lb + 1))
        self.NF = sum(ncart(l) for l in range(lc, F + 1))
        # W blocks
        self.zb = {}
        off = 0
        for fx in range(F + 1):
            for fy in range(F + 1 - fx):
                self.zb[(fx, fy)] = off
                off += tet(L - fx - fy + 1)
        self.w_size = off
        self.y_size = tet(L + 1)
        emax = self.emax
        # --- transfer z lines: (ex, ey, fx, fy) with ex+ey <= emax; extent n (ez at fz = 0)
        # and fzmax.  Inputs [e,(fx,fy,0)] for ez <= n where n = min(L - s - t, emax - s + F - t).
        zl = []
        for fx in range(F + 1):
            for fy in range(F + 1 - fx):
                t = fx + fy
                for ex in range(emax + 1):
                    for ey in range(emax + 1 - ex):
                        s = ex + ey
                        n = min(L - s - t, emax - s + (F - t))
                        zl.append((ex, ey, fx, fy, n, F - t))
        self.z_rounds = _rounds(zl, key=lambda r: (r[4], r[5]))
        # --- transfer y lines (ex, ez) per fx: table (ey, fy), fy <= F - fx.  Only ex <= emax
        # feeds a transfer-z line; cell (ey, fy) is needed for ey <= n - fy with
        # n = min(emax + F - fx - ex, L - fx - ex - ez) (targets' cone and |e| + |f| <= L).
        self.y_rounds = {}
        for fx in range(F + 1):
            yl = []
            for ex in range(emax + 1):
                for ez in range(L - fx - ex + 1):
                    n = min(emax + F - fx - ex, L - fx - ex - ez)
                    yl.append((ex, ez, n))
            self.y_rounds[fx] = _rounds(yl, key=lambda r: r[2])
        # --- transfer x lines (ey, ez): table (ex, fx), fx <= F.  Cell (ex, fx) needed when
        # ex <= emax + F - fx.
        xl = []
        for ey in range(L + 1):
            for ez in range(L + 1 - ey):
                n = min(L - ey - ez, emax + F)
                if ey + ez > emax + F:
                    continue
                xl.append((ey, ez, n))
        self.x_rounds = _rounds(xl, key=lambda r: r[2])
        # --- VRR z lines (ex, ey): ez <= L - ex - ey, only those with ex + ey <= emax + F
        vl = [(ex, ey, L - ex - ey) for ex in range(L + 1) for ey in range(L + 1 - ex)
              if ex + ey <= emax + F]
        self.v_rounds = _rounds(vl, key=lambda r: r[2])

    def widx(self, ex, ey, ez, fx, fy):
        g = self.L - fx - fy
        assert ex + ey + ez <= g, (ex, ey, ez, fx, fy)
        return self.zb[(fx, fy)] + toff(ex, ey, g) + ez

    def yidx(self, ex, ey, m):
        return toff(ex, ey, self.L) + m

    def acc_index(self, e, f):
        la, lc = self.la, self.lc
        ie = tet(sum(e)) - tet(la) + comp_index(e)
        jf = tet(sum(f)) - tet(lc) + comp_index(f)
        return ie * self.NF + jf

    def rounds_summary(self):
        return {"v": len(self.v_rounds), "x": len(self.x_rounds),
                "y": sum(len(r) for r in self.y_rounds.values()), "z": len(self.z_rounds)}


# ------------------------------------------------------------------- host emulation
def emulate(S, Fm, PA, WP, o2z, rz, CE, ze, o2e, ACC):
    """One primitive quartet through the schedule (lanes emulated one by one), adding its
    [e0|f0] to ACC (a list of NE*NF floats in target order).  Mirrors the device code."""
    L, F, emax = S.L, S.F, S.emax
    W = [math.nan] * S.w_size
    Y = [math.nan] * S.y_size
    # VRR x then y: lane ex
    for ex in range(L + 1):
        c = list(Fm) + [0.0]
        p = [0.0] * (L + 2)
        for k in range(1, ex + 1):
            nw = [0.0] * (L + 2)
            for m in range(L - k + 1):
                v = PA[0] * c[m] + WP[0] * c[m + 1]
                if k >= 2:
                    v += (k - 1) * o2z * (p[m] - rz * p[m + 1])
                nw[m] = v
            p, c = c, nw
        py = [0.0] * (L + 2)
        for ey in range(0, L - ex + 1):
            if ey >= 1:
                nw = [0.0] * (L + 2)
                for m in range(L - ex - ey + 1):
                    v = PA[1] * c[m] + WP[1] * c[m + 1]
                    if ey >= 2:
                        v += (ey - 1) * o2z * (py[m] - rz * py[m + 1])
                    nw[m] = v
                py, c = c, nw
            for m in range(L - ex - ey + 1):
                Y[S.yidx(ex, ey, m)] = c[m]
    # VRR z lines
    for rnd in S.v_rounds:
        for (ex, ey, n) in rnd:
            c = [Y[S.yidx(ex, ey, m)] for m in range(n + 1)] + [0.0]
            p = [0.0] * (n + 2)
            W[S.widx(ex, ey, 0, 0, 0)] = c[0]
            for ez in range(1, n + 1):
                nw = [0.0] * (n + 2)
                for m in range(n - ez + 1):
                    v = PA[2] * c[m] + WP[2] * c[m + 1]
                    if ez >= 2:
                        v += (ez - 1) * o2z * (p[m] - rz * p[m + 1])
                    nw[m] = v
                p, c = c, nw
                W[S.widx(ex, ey, ez, 0, 0)] = c[0]

    def transfer(r1, r0, i, k, ext):
        # r1 = [.., f], r0 = [.., f - 1_i]; k = f_i (before the step); ext = cells of result
        out = []
        for a in range(ext + 1):
            v = CE[i] * r1[a] - ze * r1[a + 1]
            if a >= 1:
                v += a * o2e * r1[a - 1]
            if k >= 1:
                v += k * o2e * r0[a]
            out.append(v)
        return out + [math.nan]

    # transfer x lines (ey, ez): cells ex <= n - fx (and ex <= emax + F - fx)
    for rnd in S.x_rounds:
        for (ey, ez, n) in rnd:
            r1 = [W[S.widx(ex, ey, ez, 0, 0)] for ex in range(n + 1)] + [math.nan]
            r0 = None
            for fx in range(1, F + 1):
                ext = min(n - fx, emax + F - fx)
                if ext < 0:
                    break
                nw = transfer(r1, r0, 0, fx - 1, ext)
                for ex in range(ext + 1):
                    W[S.widx(ex, ey, ez, fx, 0)] = nw[ex]
                r0, r1 = r1, nw
    # transfer y lines (ex, ez) per fx: cells ey <= n - fy
    for fx in range(F + 1):
        for rnd in S.y_rounds[fx]:
            for (ex, ez, n) in rnd:
                r1 = [W[S.widx(ex, ey, ez, fx, 0)] for ey in range(n + 1)] + [math.nan]
                r0 = None
                for fy in range(1, F - fx + 1):
                    ext = min(n - fy, emax + (F - fx - fy) - ex)
                    if ext < 0:
                        break
                    nw = transfer(r1, r0, 1, fy - 1, ext)
                    for ey in range(ext + 1):
                        W[S.widx(ex, ey, ez, fx, fy)] = nw[ey]
                    r0, r1 = r1, nw
    # transfer z lines: targets
    la, lc = S.la, S.lc
    for rnd in S.z_rounds:
        for (ex, ey, fx, fy, n, fzmax) in rnd:
            s, t = ex + ey, fx + fy
            r1 = [W[S.widx(ex, ey, ez, fx, fy)] for ez in range(n + 1)] + [math.nan]
            r0 = None
            for fz in range(0, fzmax + 1):
                if fz >= 1:
                    ext = min(n - fz, emax - s + (F - t - fz))
                    if ext < 0:
                        break
                    nw = transfer(r1, r0, 2, fz - 1, ext)
                    r0, r1 = r1, nw
                else:
                    ext = n
                if lc <= t + fz <= F:
                    for ez in range(ext + 1):
                        if la <= s + ez <= emax:
                            ACC[S.acc_index((ex, ey, ez), (fx, fy, fz))] += r1[ez]


# ------------------------------------------------------------------- device code
def _tag(cls):
    return "".join(str(v) for v in cls)


def emit_class(S, tab_name, tab_off):
    """Struct LinesCls_<tag> with prim() for schedule S; returns (code, table ints)."""
    la, lb, lc, ld = S.cls
    L, F, emax = S.L, S.F, S.emax
    tab = []
    body = []
    off = tab_off

    def row(vals, width=32):
        nonlocal off
        vals = list(vals)
        vals = vals + [-1] * (width - len(vals))
        tab.extend(vals)
        o = off
        off += width
        return o

    body.append(f"    lines_vrr_xy<{L}>(lane, Fs, s, Y);")
    body.append("    __syncwarp();")
    for rnd in S.v_rounds:
        o = row(ex | (ey << 8) for (ex, ey, n) in rnd)
        nmax = max(n for (_, _, n) in rnd)
        body.append(f"    lines_vrr_z<{L}, {nmax}>(__ldg({tab_name} + {o} + lane), s, Y, W);")
    body.append("    __syncwarp();")
    for rnd in S.x_rounds:
        o = row(ey | (ez << 8) for (ey, ez, n) in rnd)
        nmax = max(n for (_, _, n) in rnd)
        body.append(f"    lines_etr_x<{L}, {F}, {nmax}>(__ldg({tab_name} + {o} + lane), s, W);")
    body.append("    __syncwarp();")
    for fx in range(F):  # at fx = F there is no y step left
        for rnd in S.y_rounds[fx]:
            if not rnd:
                continue
            o = row(ex | (ez << 8) for (ex, ez, n) in rnd)
            nmax = max(max(n for (_, _, n) in rnd), 0)
            body.append(f"    lines_etr_y<{L}, {F}, {emax}, {fx}, {nmax}>"
                        f"(__ldg({tab_name} + {o} + lane), s, W);")
    body.append("    __syncwarp();")
    for rnd in S.z_rounds:
        o1 = row(ex | (ey << 4) | (fx << 8) | (fy << 12) for (ex, ey, fx, fy, n, fz) in rnd)
        o2 = row(S.widx(ex, ey, 0, fx, fy) for (ex, ey, fx, fy, n, fz) in rnd)
        nmax = max(n for r in rnd for n in [r[4]])
        fzmax = max(r[5] for r in rnd)
        body.append(f"    lines_etr_z<{L}, {F}, {la}, {emax}, {lc}, {S.NF}, {nmax}, {fzmax}>"
                    f"(make_int2(__ldg({tab_name} + {o1} + lane), __ldg({tab_name} + {o2} + lane)), "
                    "s, W, ACC, first);")
    tag = _tag(S.cls)
    reg = tail_fits(S.cls)
    # the group form (a CTA of GROUP_W warps per quartet, classes with the interpreted tail):
    # vrr_xy on warp 0; each stage's rounds given to the warps longest first, each to the warp
    # with the least work so far (a round's cost: its longest line); a CTA barrier between stages
    body_g = []
    if not reg:
        stage = []

        def flush():
            load = [0] * GROUP_W
            for cost, ln in sorted(stage, key=lambda x: -x[0]):
                w = load.index(min(load))
                load[w] += cost
                body_g.append(f"    if (wq == {w})" + ln[3:])
            stage.clear()
        for ln in body:
            if "__syncwarp();" in ln:
                flush()
                body_g.append("    __syncthreads();")
            elif "lines_vrr_xy<" in ln:
                body_g.append("    if (wq == 0)" + ln[3:])
            else:
                tmpl = ln[ln.index("<") + 1:ln.index(">")].split(",")
                stage.append((int(tmpl[-1]) + 1 if "etr_z" not in ln else
                              (int(tmpl[-2]) + 1) * (int(tmpl[-1]) + 1), ln))
        flush()
    code = ([emit_tail(S.cls)] if reg else []) + [
            f"struct LinesCls_{tag} {{",
            f"  static constexpr int L = {L}, NE = {S.NE}, NF = {S.NF}, kW = {S.w_size}, "
            f"kY = {S.y_size};",
            f"  static constexpr int LA = {la}, LB = {lb}, LC = {lc}, LD = {ld};",
            f"  static constexpr bool kRegTail = {'true' if reg else 'false'};",
            f"  static constexpr bool kGroup = {'false' if reg else 'true'};",
            f"  using Tail = {'TailCls_' + tag if reg else 'void'};",
            "  static __device__ __forceinline__ void prim(int lane, const double* Fs,",
            "                                              const LinePS& s, double* __restrict__ W,",
            "                                              double* __restrict__ Y,",
            "                                              double* __restrict__ ACC, bool first) {",
            *body,
            "  }",
            *([] if reg else [
                "  static __device__ __forceinline__ void prim_g(int wq, int lane, const double* Fs,",
                "                                                const LinePS& s, double* __restrict__ W,",
                "                                                double* __restrict__ Y,",
                "                                                double* __restrict__ ACC, bool first) {",
                *body_g,
                "  }"]),
            "};"]
    return "\n".join(code), tab


def emit_sources(outdir, heavy, nfiles=12):
    """Write lines_XX.cu (each with its own program tables for its classes) and return
    (file names, {class: launcher name})."""
    import os
    import gen_coop
    cost = {}
    for c in heavy:
        S = Schedule(*c)
        cost[c] = S.w_size + 4 * sum(len(r) for r in S.z_rounds) + S.NE * S.NF
    bins = [[] for _ in range(nfiles)]
    load = [0] * nfiles
    for c in sorted(heavy, key=lambda c: -cost[c]):
        k = load.index(min(load))
        bins[k].append(c)
        load[k] += cost[c]
    files, launchers = [], {}
    for k, mine in enumerate(b for b in bins if b):
        mine = sorted(mine)
        prog = f"coop_programs_l{k:02d}.cuh"
        gen_coop.emit(mine, os.path.join(outdir, prog))
        tab_name = "kLinesTab"
        tab = []
        structs = []
        for c in mine:
            code, t = emit_class(Schedule(*c), tab_name, len(tab))
            tab += t
            structs.append(code)
            if split_ok(c):
                structs.append(emit_split(c))
        out = ["// Generated by gen_lines.py: line-factorised cooperative kernels of heavy classes.",
               f'#include "{prog}"',
               '#include "../lines_kernel.cuh"',
               '#include "../errors.h"',
               "namespace gbx {",
               f"__device__ const int {tab_name}[{max(1, len(tab))}] = {{"
               + ", ".join(str(v) for v in tab) + "};"]
        out += structs
        for j, c in enumerate(mine):
            tag = _tag(c)
            name = f"launch_lines_{tag}"
            launchers[c] = name
            out.append(f"int {name}(const EriLaunch& a, cudaStream_t st) {{")
            if split_ok(c):
                out.append(f"  if (a.variant == 0) return launch_split_t<SplitCls_{tag}>(a, st);")
            out.append(f"  return launch_lines_t<LinesCls_{tag}>(a, kCoopMeta[{j}], st);")
            out.append("}")
        out.append("}  // namespace gbx")
        text = "\n".join(out) + "\n"
        name = f"lines_{k:02d}.cu"
        path = os.path.join(outdir, name)
        if not (os.path.exists(path) and open(path).read() == text):
            with open(path, "w") as f:
                f.write(text)
        files.append(name)
    return files, launchers


# ------------------------------------------------------------------- register tail
def tail_fits(cls):
    """The register tail holds one ket row (NCD) and one bra column (NAB) per lane."""
    la, lb, lc, ld = cls
    return ncart(la) * ncart(lb) <= 36 and ncart(lc) * ncart(ld) <= 36


def _hrr_code(lo, hi_shell, targets_a, targets_b, leaf, coef):
    """Straight-line horizontal recursion (x, y+1_i) = (x+1_i, y) + coef_i (x, y) for the
    targets (a, b), leaves (x, 0) = leaf(x); returns (lines, {(a, b): expression})."""
    import gen_eri as G
    best = None
    for pk in (G.pick_first, G.pick_last, G.pick_max):
        nodes = G.HrrGen.closure(lo, targets_a, targets_b, pk)
        n = sum(1 for v in nodes.values() if v is not None)
        if best is None or n < best[0]:
            best = (n, nodes)
    nodes = best[1]
    order = sorted(((k, v) for k, v in nodes.items() if v is not None), key=lambda kv: sum(kv[0][1]))

    def name(x, y):
        if sum(y) == 0:
            return leaf(x)
        return f"h_{G.tname(x)}_{G.tname(y)}"
    lines = []
    for (x, y), i in order:
        y1 = G.add(y, i, -1)
        lines.append(f"    const double {name(x, y)} = fma({coef}{'xyz'[i]}, {name(x, y1)}, "
                     f"{name(G.add(x, i), y1)});")
    return lines, {(a, b): name(a, b) for a in targets_a for b in targets_b}


def emit_tail(cls):
    """Struct TailCls_<tag>: ket(row) -> out[NCD] and bra(col, stride) -> out[NAB]."""
    import gen_eri as G
    la, lb, lc, ld = cls
    E = G.comps_range(la, la + lb)
    F = G.comps_range(lc, lc + ld)
    Fi = {f: j for j, f in enumerate(F)}
    Ei = {e: j for j, e in enumerate(E)}
    klines, kmap = _hrr_code(lc, ld, G.comps(lc), G.comps(ld), lambda f: f"row[{Fi[f]}]", "CD")
    blines, bmap = _hrr_code(la, lb, G.comps(la), G.comps(lb), lambda e: f"col[{Ei[e]} * stride]",
                             "AB")
    out = [f"struct TailCls_{_tag(cls)} {{",
           "  static __device__ __forceinline__ void ket(const double* __restrict__ row, double CDx,",
           "                                             double CDy, double CDz, double* out) {",
           *klines]
    out += [f"    out[{k}] = {kmap[(c, d)]};" for k, (c, d) in
            enumerate((c, d) for c in G.comps(lc) for d in G.comps(ld))]
    out += ["  }",
            "  static __device__ __forceinline__ void bra(const double* __restrict__ col, int stride,",
            "                                             double ABx, double ABy, double ABz, double* out) {",
            *blines]
    out += [f"    out[{k}] = {bmap[(a, b)]};" for k, (a, b) in
            enumerate((a, b) for a in G.comps(la) for b in G.comps(lb))]
    out += ["  }", "};"]
    return "\n".join(out)


# ------------------------------------------------------------------- split register kernel
GROUP_W = 4         # warps of the group form's CTA (one quartet per CTA)
SPLITS = (4, 8)     # warps of a CTA, each computing one part of the targets
SPLIT_MAX_ACC = 64  # accumulators per thread in a part
SPLIT_MAX_OPS = 500  # recursion operations per part with 4 parts
# with 8 parts: every class of 620 < ops <= 750 (and every one of 500 < ops <= 620 with more
# than 40 accumulators) was checked spill-free with ptxas on sm_100a (226-252 registers);
# 906 ops spilled 220-530 bytes
SPLIT_MAX_OPS_8 = 750
SPLIT_MAX_L = 7


def split_parts(cls, S):
    """Contiguous ranges of bra rows e (in target order), one per warp."""
    import gen_eri as G
    la, lb, lc, ld = cls
    NE = len(G.comps_range(la, la + lb))
    return [(r * NE // S, (r + 1) * NE // S) for r in range(S)]


def split_ok(cls):
    """Number of parts (warps) of the split kernel for the class, or 0: the smallest S whose
    parts fit a thread's registers (at most SPLIT_MAX_ACC accumulators and SPLIT_MAX_OPS
    recursion operations per part, or 620 operations with at most 40 accumulators, or with 8
    parts SPLIT_MAX_OPS_8; beyond that the parts spill, as measured with ptxas on sm_100a)."""
    return _split_ok(tuple(cls))


@functools.lru_cache(maxsize=None)
def _split_ok(cls):
    import gen_eri as G
    la, lb, lc, ld = cls
    E = G.comps_range(la, la + lb)
    F = G.comps_range(lc, lc + ld)
    if not (sum(cls) <= SPLIT_MAX_L and tail_fits(cls)):
        return 0
    for S in SPLITS:
        parts = split_parts(cls, S)
        if not all(e1 > e0 for e0, e1 in parts):
            continue
        acc = max(e1 - e0 for e0, e1 in parts) * len(F)
        if acc > SPLIT_MAX_ACC:
            continue
        ops = max(_part_gen(cls, E[e0:e1], F).op_count() for e0, e1 in parts)
        if ops <= SPLIT_MAX_OPS or (acc <= 40 and ops <= 620) or (S == 8 and ops <= SPLIT_MAX_OPS_8):
            return S
    return 0


def _part_gen(cls, E, F):
    """Cheapest recursion closure (over the step-direction choices) for targets E x F."""
    import gen_eri as G
    la, lb, lc, ld = cls
    best = None
    for vp in (G.pick_first, G.pick_last, G.pick_max):
        for ep in (G.pick_etr_first, G.pick_etr_last, G.pick_etr_max, G.pick_etr_min_e):
            g = G.PrimGen.__new__(G.PrimGen)
            g.la, g.lb, g.lc, g.ld = la, lb, lc, ld
            g.L = sum(cls)
            g.E, g.F = E, F
            g.vrr_pick, g.etr_pick = vp, ep
            g.vrr, g.etr = {}, {}
            for e in E:
                for f in F:
                    g._need_etr(e, f)
            n = g.op_count()
            if best is None or n < best[0]:
                best = (n, g)
    return best[1]


def emit_split(cls):
    """Struct SplitCls_<tag>: part(r, ...) adds part r's [e0|f0] (rows e0(r)..e1(r)) of one
    primitive quartet to acc (row-major within the part)."""
    import gen_eri as G
    la, lb, lc, ld = cls
    E = G.comps_range(la, la + lb)
    F = G.comps_range(lc, lc + ld)
    S = split_ok(cls)
    parts = split_parts(cls, S)
    kacc = max(e1 - e0 for e0, e1 in parts) * len(F)
    tag = _tag(cls)
    out = [f"struct SplitCls_{tag} {{",
           f"  static constexpr int L = {sum(cls)}, NE = {len(E)}, NF = {len(F)}, kAcc = {kacc}, "
           f"kS = {S};",
           f"  static constexpr int LA = {la}, LB = {lb}, LC = {lc}, LD = {ld};",
           f"  using Tail = TailCls_{tag};",
           "  static __device__ __forceinline__ int e0(int r) { return "
           + " ".join(f"r == {r} ? {e0} :" for r, (e0, _) in enumerate(parts[:-1]))
           + f" {parts[-1][0]}; }}",
           "  static __device__ __forceinline__ int ne(int r) { return "
           + " ".join(f"r == {r} ? {e1 - e0} :" for r, (e0, e1) in enumerate(parts[:-1]))
           + f" {parts[-1][1] - parts[-1][0]}; }}"]
    for r, (e0, e1) in enumerate(parts):
        g = _part_gen(cls, E[e0:e1], F)
        body = []
        g.emit(body)
        out.append(f"  static __device__ __forceinline__ void part{r}(const double* __restrict__ F,")
        out.append("      double PAx, double PAy, double PAz, double WPx, double WPy, double WPz,")
        out.append("      double o2z, double rz, double CEx, double CEy, double CEz, double ze, double o2e,")
        out.append("      double* __restrict__ acc) {")
        out += ["    " + b.replace("const R ", "const double ").replace("R(", "double(") for b in body]
        out.append("    (void)PAx; (void)PAy; (void)PAz; (void)WPx; (void)WPy; (void)WPz; (void)o2z;")
        out.append("    (void)rz; (void)CEx; (void)CEy; (void)CEz; (void)ze; (void)o2e;")
        out.append("  }")
    out.append("  static __device__ __forceinline__ void part(int r, const double* F, double PAx,")
    out.append("      double PAy, double PAz, double WPx, double WPy, double WPz, double o2z, double rz,")
    out.append("      double CEx, double CEy, double CEz, double ze, double o2e, double* acc) {")
    out.append("    switch (r) {")
    for r in range(S):
        out.append(f"      case {r}: part{r}(F, PAx, PAy, PAz, WPx, WPy, WPz, o2z, rz, CEx, CEy, CEz, "
                   "ze, o2e, acc); break;")
    out.append("      default: break;")
    out.append("    }")
    out.append("  }")
    out.append("};")
    return "\n".join(out)
