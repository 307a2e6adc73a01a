"""Generate class-specialised recursion code for the ERI kernels (writes ``eri_gen.cuh``).

For every class (la, lb | lc, ld) — ordered pair types, the bra pair type not below the ket
pair type in the order (la + lb, max(la, lb), la) — this emits straight-line device code for

* ``prim``: one primitive quartet of the Obara-Saika vertical recursion on centre A
  ([e0|00]^(m), e <= L) followed by the electron-transfer recursion onto centre C
  ([e0|f0], la <= |e| <= la+lb, lc <= |f| <= lc+ld), accumulated into ``acc``;
* ``hrr``: the horizontal recursions (ket first, then bra) that turn the contracted
  [e0|f0] into the Cartesian block (ab|cd).

Only the intermediates the targets depend on are emitted (dependency closure), and the
recursion direction at every node is chosen per class to minimise the operation count.
The mathematics is that of gbasis (``gbasis/integrals/_two_elec_int.py:350-526`` for
VRR/ETR, ``:549-788`` for HRR); the code organisation is this project's.

Usage: ``python gen_eri.py [LMAX] > eri_gen.cuh`` (default LMAX = 3).
"""
from __future__ import annotations

import itertools
import sys

DIRS = "xyz"


def ncart(l):
    return (l + 1) * (l + 2) // 2


def comps(l):
    return [(x, y, l - x - y) for x in range(l, -1, -1) for y in range(l - x, -1, -1)]


def comps_range(lo, hi):
    return [c for n in range(lo, hi + 1) for c in comps(n)]


def add(t, i, k=1):
    u = list(t)
    u[i] += k
    return tuple(u)


def tname(t):
    return "".join(str(v) for v in t)


def pair_types(lmax):
    """Ordered pair types (lA, lB) sorted by (lA + lB, max, lA): the engine's pair classes."""
    return sorted(((a, b) for a in range(lmax + 1) for b in range(lmax + 1)),
                  key=lambda t: (t[0] + t[1], max(t), t[0]))


def canonical_classes(lmax):
    """(lA, lB, lC, lD) with the bra pair class not below the ket pair class."""
    pts = pair_types(lmax)
    return [bra + ket for i, bra in enumerate(pts) for ket in pts[: i + 1]]


# --------------------------------------------------------------------------- VRR/ETR
class PrimGen:
    """Dependency closure and code for one class's primitive recursion."""

    def __init__(self, la, lb, lc, ld, vrr_pick, etr_pick):
        self.la, self.lb, self.lc, self.ld = la, lb, lc, ld
        self.L = la + lb + lc + ld
        self.E = comps_range(la, la + lb)
        self.F = comps_range(lc, lc + ld)
        self.vrr_pick, self.etr_pick = vrr_pick, etr_pick
        self.vrr = {}  # (e, m) -> (i, deps)
        self.etr = {}  # (e, f) -> (i, deps)
        for e in self.E:
            for f in self.F:
                self._need_etr(e, f)

    def _need_vrr(self, e, m):
        key = (e, m)
        if key in self.vrr:
            return
        if sum(e) == 0:
            self.vrr[key] = None
            return
        i = self.vrr_pick(e)
        e1 = add(e, i, -1)
        self.vrr[key] = i
        self._need_vrr(e1, m)
        self._need_vrr(e1, m + 1)
        if e1[i] > 0:
            e2 = add(e1, i, -1)
            self._need_vrr(e2, m)
            self._need_vrr(e2, m + 1)

    def _need_etr(self, e, f):
        key = (e, f)
        if key in self.etr:
            return
        if sum(f) == 0:
            self.etr[key] = None
            self._need_vrr(e, 0)
            return
        i = self.etr_pick(e, f)
        f1 = add(f, i, -1)
        self.etr[key] = i
        self._need_etr(e, f1)
        self._need_etr(add(e, i), f1)
        if e[i] > 0:
            self._need_etr(add(e, i, -1), f1)
        if f1[i] > 0:
            self._need_etr(e, add(f1, i, -1))

    def op_count(self):
        n = 0
        for (e, m), i in self.vrr.items():
            if i is None:
                continue
            e1 = add(e, i, -1)
            n += 2 + (2 if e1[i] > 0 else 0)
        for (e, f), i in self.etr.items():
            if i is None:
                continue
            f1 = add(f, i, -1)
            n += 2 + (1 if e[i] > 0 else 0) + (1 if f1[i] > 0 else 0)
        return n

    @staticmethod
    def vname(e, m):
        return f"v{tname(e)}_{m}"

    @staticmethod
    def ename(e, f):
        if sum(f) == 0:
            return PrimGen.vname(e, 0)
        return f"t{tname(e)}_{tname(f)}"

    def emit(self, out):
        """Emit the body; inputs F[m], PA*, WP*, o2z, rz, CE*, ze, o2e; output acc[]."""
        order = sorted(self.vrr.items(), key=lambda kv: (sum(kv[0][0]), -kv[0][1]))
        for (e, m), i in order:
            nm = self.vname(e, m)
            if i is None:
                out.append(f"const R {nm} = F[{m}];")
                continue
            e1 = add(e, i, -1)
            d = DIRS[i]
            expr = f"fma(PA{d}, {self.vname(e1, m)}, WP{d} * {self.vname(e1, m + 1)})"
            if e1[i] > 0:
                e2 = add(e1, i, -1)
                k = e1[i]
                expr = (f"fma(R({k}) * o2z, fma(-rz, {self.vname(e2, m + 1)}, {self.vname(e2, m)}), "
                        f"{expr})")
            out.append(f"const R {nm} = {expr};")
        order = sorted(((k, v) for k, v in self.etr.items() if v is not None),
                       key=lambda kv: sum(kv[0][1]))
        for (e, f), i in order:
            f1 = add(f, i, -1)
            d = DIRS[i]
            expr = (f"fma(CE{d}, {self.ename(e, f1)}, -ze * {self.ename(add(e, i), f1)})")
            if e[i] > 0:
                expr = f"fma(R({e[i]}) * o2e, {self.ename(add(e, i, -1), f1)}, {expr})"
            if f1[i] > 0:
                expr = f"fma(R({f1[i]}) * o2e, {self.ename(e, add(f1, i, -1))}, {expr})"
            out.append(f"const R {self.ename(e, f)} = {expr};")
        nf = len(self.F)
        for ie, e in enumerate(self.E):
            for jf, f in enumerate(self.F):
                out.append(f"acc[{ie * nf + jf}] += {self.ename(e, f)};")


def pick_first(t, *_):
    return next(i for i in range(3) if t[i] > 0)


def pick_last(t, *_):
    return next(i for i in (2, 1, 0) if t[i] > 0)


def pick_max(t, *_):
    return max(range(3), key=lambda i: (t[i], -i))


def pick_etr_first(e, f):
    return pick_first(f)


def pick_etr_last(e, f):
    return pick_last(f)


def pick_etr_max(e, f):
    return pick_max(f)


def pick_etr_min_e(e, f):
    # prefer the direction where e is small (fewer [e-1] terms)
    cands = [i for i in range(3) if f[i] > 0]
    return min(cands, key=lambda i: (e[i], -f[i], i))


def best_prim(la, lb, lc, ld):
    best = None
    for vp in (pick_first, pick_last, pick_max):
        for ep in (pick_etr_first, pick_etr_last, pick_etr_max, pick_etr_min_e):
            g = PrimGen(la, lb, lc, ld, vp, ep)
            n = g.op_count()
            if best is None or n < best[0]:
                best = (n, g)
    return best[1]


# ---------------------------------------------------------------------------- HRR
class HrrGen:
    """(ab|cd) from contracted [e0|f0]: ket HRR with CD, then bra HRR with AB."""

    def __init__(self, la, lb, lc, ld):
        self.la, self.lb, self.lc, self.ld = la, lb, lc, ld
        self.E = comps_range(la, la + lb)
        self.F = comps_range(lc, lc + ld)

    @staticmethod
    def closure(lo, tgt_a, tgt_b, pick):
        nodes = {}

        def need(a, b):
            if (a, b) in nodes:
                return
            if sum(b) == 0:
                nodes[(a, b)] = None
                return
            i = pick(b)
            b1 = add(b, i, -1)
            nodes[(a, b)] = i
            need(add(a, i), b1)
            need(a, b1)

        for a in tgt_a:
            for b in tgt_b:
                need(a, b)
        return nodes

    def emit(self, out):
        la, lb, lc, ld = self.la, self.lb, self.lc, self.ld
        NF = len(self.F)
        Fidx = {f: j for j, f in enumerate(self.F)}
        Eidx = {e: j for j, e in enumerate(self.E)}
        cd_t = [(c, d) for c in comps(lc) for d in comps(ld)]
        ab_t = [(a, b) for a in comps(la) for b in comps(lb)]
        NCD = len(cd_t)
        best = None
        for pk in (pick_first, pick_last, pick_max):
            kn = self.closure(lc, comps(lc), comps(ld), pk)
            bn = self.closure(la, comps(la), comps(lb), pk)
            n = len(self.E) * sum(1 for v in kn.values() if v is not None) + \
                NCD * sum(1 for v in bn.values() if v is not None)
            if best is None or n < best[0]:
                best = (n, kn, bn)
        _, kn, bn = best
        korder = sorted(((k, v) for k, v in kn.items() if v is not None), key=lambda kv: sum(kv[0][1]))
        border = sorted(((k, v) for k, v in bn.items() if v is not None), key=lambda kv: sum(kv[0][1]))
        # ket side: for every e, h[e][cd]
        for ie, e in enumerate(self.E):
            def kname(c, d):
                if sum(d) == 0:
                    return f"acc[{ie * NF + Fidx[c]}]"
                return f"k{ie}_{tname(c)}_{tname(d)}"
            for (c, d), i in korder:
                dd = DIRS[i]
                d1 = add(d, i, -1)
                out.append(f"const double {kname(c, d)} = fma(CD{dd}, {kname(c, d1)}, "
                           f"{kname(add(c, i), d1)});")
            for icd, (c, d) in enumerate(cd_t):
                out.append(f"double h{ie}_{icd} = {kname(c, d)};")
        # bra side: for every cd, (ab|cd)
        NB = ncart(lb)
        for icd in range(NCD):
            def bname(a, b):
                if sum(b) == 0:
                    return f"h{Eidx[a]}_{icd}"
                return f"b{icd}_{tname(a)}_{tname(b)}"
            for (a, b), i in border:
                dd = DIRS[i]
                b1 = add(b, i, -1)
                out.append(f"const double {bname(a, b)} = fma(AB{dd}, {bname(a, b1)}, "
                           f"{bname(add(a, i), b1)});")
            for iab, (a, b) in enumerate(ab_t):
                out.append(f"out[{iab * NCD + icd}] = {bname(a, b)};")
        del NB


def _dfact(n):
    r = 1
    while n > 1:
        r *= n
        n -= 2
    return r


def emit_sph_and_norms(w, lmax):
    """Constant Cartesian->spherical code per l (engine_sph_matrix) and the Cartesian
    component norms 1/sqrt(prod (2a_i-1)!!) in canonical order."""
    import math
    import os
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))))
    from gbasis_b200.spherical import engine_sph_matrix
    w("template <int L> struct Sph;")
    for l in range(2, lmax + 1):
        K = engine_sph_matrix(l)
        w(f"template <> struct Sph<{l}> {{")
        w(f"  static __device__ __forceinline__ void apply(const double* x, double* y) {{")
        for u in range(K.shape[0]):
            terms = [(c, float(K[u, c])) for c in range(K.shape[1]) if K[u, c] != 0.0]
            expr = f"{terms[0][1]!r} * x[{terms[0][0]}]"
            for c, v in terms[1:]:
                expr = f"fma({v!r}, x[{c}], {expr})"
            w(f"    y[{u}] = {expr};")
        w("  }")
        w("};")
    w("template <int L> __device__ __forceinline__ double cnorm(int c);")
    for l in range(lmax + 1):
        vals = [1.0 / math.sqrt(_dfact(2 * a - 1) * _dfact(2 * b - 1) * _dfact(2 * c - 1))
                for a, b, c in comps(l)]
        w(f"template <> __device__ __forceinline__ double cnorm<{l}>(int c) {{")
        w(f"  constexpr double v[{len(vals)}] = {{{', '.join(repr(v) for v in vals)}}};")
        w("  return v[c];")
        w("}")


LIGHT_LIMIT = 170  # doubles of [e0|f0] + (ab|cd) one thread may hold


def is_light(c):
    """Classes evaluated by one thread in registers; the rest run on the cooperative kernel."""
    la, lb, lc, ld = c
    ne = sum(ncart(e) for e in range(la, la + lb + 1))
    nf = sum(ncart(f) for f in range(lc, lc + ld + 1))
    return ne * nf + ncart(la) * ncart(lb) * ncart(lc) * ncart(ld) <= LIGHT_LIMIT


# Largest total angular momentum for which the straight-line register code is emitted: the CPU
# tests execute it against the oracle for every class up to L = 8, and the device compiles it
# for classes up to L = 6 only (light classes and the (ab|ss) structs).  Executed on the CPU, the
# VRR/transfer code emitted for the L >= 11 heavy f classes disagrees with a direct recursion.
MAX_EMIT_L = 8


def emit_all(lmax, classes=None):
    if classes is None:
        classes = [c for c in canonical_classes(lmax) if is_light(c)]
    lines = []
    w = lines.append
    w("// Generated by gen_eri.py — class-specialised ERI recursions. Do not edit by hand.")
    w("#pragma once")
    w(f"#define GBX_GEN_LMAX {lmax}")
    w("namespace gbx { namespace gen {")
    emit_sph_and_norms(w, lmax)
    w("template <int LA, int LB, int LC, int LD> struct Cls;")
    for la, lb, lc, ld in classes:
        if la + lb + lc + ld > MAX_EMIT_L:
            raise ValueError(f"straight-line register code is emitted up to L = {MAX_EMIT_L}; "
                             f"class {(la, lb, lc, ld)} runs the line, split or cooperative kernel")
        g = best_prim(la, lb, lc, ld)
        h = HrrGen(la, lb, lc, ld)
        NE, NF = len(g.E), len(g.F)
        NAB, NCD = ncart(la) * ncart(lb), ncart(lc) * ncart(ld)
        w(f"template <> struct Cls<{la},{lb},{lc},{ld}> {{")
        w(f"  static constexpr int L = {la + lb + lc + ld}, NE = {NE}, NF = {NF}, "
          f"NAB = {NAB}, NCD = {NCD}, PRIM_OPS = {g.op_count()};")
        w("  template <typename R>")
        w("  static __device__ __forceinline__ void prim(const R* __restrict__ F, R PAx, R PAy, R PAz,")
        w("      R WPx, R WPy, R WPz, R o2z, R rz, R CEx, R CEy, R CEz, R ze, R o2e,")
        w("      R* __restrict__ acc) {")
        body = []
        g.emit(body)
        for b in body:
            w("    " + b)
        w("    (void)PAx; (void)PAy; (void)PAz; (void)WPx; (void)WPy; (void)WPz; (void)o2z; (void)rz;")
        w("    (void)CEx; (void)CEy; (void)CEz; (void)ze; (void)o2e;")
        w("  }")
        w("  static __device__ __forceinline__ void hrr(const double* __restrict__ acc,")
        w("      double ABx, double ABy, double ABz, double CDx, double CDy, double CDz,")
        w("      double* __restrict__ out) {")
        body = []
        h.emit(body)
        for b in body:
            w("    " + b)
        w("    (void)ABx; (void)ABy; (void)ABz; (void)CDx; (void)CDy; (void)CDz;")
        w("  }")
        w("};")
    w("}}  // namespace gbx::gen")
    return "\n".join(lines) + "\n"


def emit_sources(outdir, lmax):
    """Write eri_gen.cuh (light classes), their instantiation files, the cooperative programs
    of the heavy classes (coop_programs.cuh) and the class dispatch."""
    import os
    import gen_coop
    os.makedirs(outdir, exist_ok=True)

    def put(name, text):
        path = os.path.join(outdir, name)
        if not (os.path.exists(path) and open(path).read() == text):
            with open(path, "w") as f:
                f.write(text)

    every = canonical_classes(lmax)
    light = [c for c in every if is_light(c)]
    heavy = [c for c in every if not is_light(c)]
    # the point-charge kernel uses the (ab|ss) structs of every pair class, heavy ones included
    one_e = [(la, lb, 0, 0) for la in range(lmax + 1) for lb in range(lmax + 1)]
    put("eri_gen.cuh", emit_all(lmax, light + [c for c in one_e if c not in light]))
    # heavy classes first (their cooperative kernels index the table by position), then the
    # light classes, whose programs only the multi-class queue kernel runs
    gen_coop.emit(heavy + light, os.path.join(outdir, "coop_programs.cuh"), n_heavy=len(heavy))
    files = []
    # spread the light classes over translation units of similar compile cost (code size)
    nbins = 12
    bins = [[] for _ in range(nbins)]
    load = [0] * nbins
    cost = {c: best_prim(*c).op_count() + 4 * ncart(c[0]) * ncart(c[1]) * ncart(c[2]) * ncart(c[3])
            for c in light}
    for c in sorted(light, key=lambda c: -cost[c]):
        k = load.index(min(load))
        bins[k].append(c)
        load[k] += cost[c]
    for k, mine in enumerate(b for b in bins if b):
        lines = ["// Generated by gen_eri.py: explicit instantiations of the class kernels.",
                 '#include "../eri_kernels.cuh"',
                 '#include "../errors.h"',
                 "namespace gbx {",
                 "template <int LA, int LB, int LC, int LD>",
                 "int launch_t(const EriLaunch& a, int grid, cudaStream_t st) {",
                 "  if (a.fp32) eri_block<LA, LB, LC, LD, float><<<grid, kEriThreads, 0, st>>>(a);",
                 "  else if (a.potential)",
                 "    eri_block<LA, LB, LC, LD, double, true><<<grid, kEriThreads, 0, st>>>(a);",
                 "  else eri_block<LA, LB, LC, LD, double><<<grid, kEriThreads, 0, st>>>(a);",
                 '  return cuda_status(cudaGetLastError(), "eri class kernel launch");',
                 "}"]
        for c in mine:
            lines.append(f"template int launch_t<{c[0]}, {c[1]}, {c[2]}, {c[3]}>(const EriLaunch&, "
                         "int, cudaStream_t);")
        lines.append("}  // namespace gbx")
        name = f"eri_cls_{k:02d}.cu"
        put(name, "\n".join(lines) + "\n")
        files.append(name)
    import gen_lines
    lfiles, launchers = gen_lines.emit_sources(outdir, heavy)
    files += lfiles
    lines = ["// Generated by gen_eri.py: (la,lb,lc,ld) -> class kernel launcher.",
             "#include <cstdlib>",
             "#include <cstring>",
             '#include "../coop.cuh"',
             '#include "../runtime.h"',
             "namespace gbx {",
             "template <int LA, int LB, int LC, int LD>",
             "int launch_t(const EriLaunch& a, int grid, cudaStream_t st);"]
    for c in light:
        lines.append(f"extern template int launch_t<{c[0]}, {c[1]}, {c[2]}, {c[3]}>(const EriLaunch&, "
                     "int, cudaStream_t);")
    for c in heavy:
        lines.append(f"int {launchers[c]}(const EriLaunch& a, cudaStream_t st);")
    lines.append("// Heavy classes run the line-factorised kernel; GBX_HEAVY_KERNEL=interp selects the")
    lines.append("// program-interpreting cooperative kernel instead (read once per process).")
    lines.append("static bool heavy_interp() {")
    lines.append('  static const bool v = [] { const char* e = std::getenv("GBX_HEAVY_KERNEL");')
    lines.append('                             return e && std::strcmp(e, "interp") == 0; }();')
    lines.append("  return v;")
    lines.append("}")
    lines.append(f"int compiled_lmax() {{ return {lmax}; }}")
    lines.append("int launch_class(int la, int lb, int lc, int ld, const EriLaunch& a, int grid, "
                 "cudaStream_t st) {")
    lines.append("  switch (((la * 8 + lb) * 8 + lc) * 8 + ld) {")
    for c in light:
        key = ((c[0] * 8 + c[1]) * 8 + c[2]) * 8 + c[3]
        lines.append(f"    case {key}: return launch_t<{c[0]}, {c[1]}, {c[2]}, {c[3]}>(a, grid, st);")
    for j, c in enumerate(heavy):
        key = ((c[0] * 8 + c[1]) * 8 + c[2]) * 8 + c[3]
        lines.append(f"    case {key}: return heavy_interp() ? launch_coop({j}, a, st) : "
                     f"{launchers[c]}(a, st);")
    lines.append("    default: break;")
    lines.append("  }")
    lines.append('  return set_error(GBX_ERR_UNSUPPORTED, "no kernel for class (%d %d|%d %d)", '
                 "la, lb, lc, ld);")
    lines.append("}")
    lines.append("}  // namespace gbx")
    put("eri_dispatch.cu", "\n".join(lines) + "\n")
    files.append("eri_dispatch.cu")
    return files


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "--emit-dir":
        lmax = int(sys.argv[3]) if len(sys.argv) > 3 else 2
        print("\n".join(emit_sources(sys.argv[2], lmax)))
    else:
        lmax = int(sys.argv[1]) if len(sys.argv) > 1 else 3
        sys.stdout.write(emit_all(lmax))
