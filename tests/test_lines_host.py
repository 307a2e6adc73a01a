"""Host checks of the line-factorised heavy-class kernel (``csrc/lines_kernel.cuh``).

The generated per-class code (``gen_lines.emit_class``: a list of template calls with their
lane tables) is executed on the CPU by a line-for-line Python transcription of the device
templates, lane by lane, and the accumulated [e0|f0] are compared with a direct memoised
evaluation of the vertical and transfer recursions (same step directions).  A schedule error,
a table error or an index error in the templates shows up here, without a GPU.
"""
import os
import re
import sys
from functools import lru_cache

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "gbasis_b200", "csrc"))
import gen_eri  # noqa: E402
import gen_lines  # noqa: E402

tet = gen_lines.tet


def zb(L, F, fx, fy):
    off = 0
    for a in range(F + 1):
        for b in range(F + 1 - a):
            if (a, b) == (fx, fy):
                return off
            off += tet(L - a - b + 1)
    return off


def toff(ex, ey, g):
    return tet(g + 1) - tet(g + 1 - ex) + ey * (g + 1 - ex) - ey * (ey - 1) // 2


class Dev:
    """Python transcription of the device templates (same loops, predicates and indices)."""

    def __init__(self, s):
        self.s = s

    def vstep(self, M, c, p, k, PA, WP):
        s = self.s
        a = (k - 1) * s["o2z"]
        for m in range(M + 1):
            if m <= M - k:
                v = PA * c[m] + WP * c[m + 1]
                v = a * (p[m] - s["rz"] * p[m + 1]) + v
                p[m] = c[m]
                c[m] = v

    def tstep(self, M, r1, r0, k, ext, CE, lim):
        s = self.s
        kk = k * s["o2e"]
        nw = [0.0] * (M + 1)
        for a in range(M + 1):
            if a > lim:
                continue
            v = CE * r1[a] - s["ze"] * r1[a + 1]
            if a >= 1:
                v = a * s["o2e"] * r1[a - 1] + v
            v = kk * r0[a] + v
            nw[a] = v if a <= ext else 0.0
        for a in range(M + 1):
            r0[a] = r1[a]
            r1[a] = nw[a]

    def vrr_xy(self, L, lane, Fs, Y):
        s = self.s
        ex = lane
        if ex > L:
            return
        c = [Fs[m] for m in range(L + 1)] + [0.0]
        p = [0.0] * (L + 2)
        for k in range(1, L + 1):
            if k <= ex:
                self.vstep(L, c, p, k, s["PA"][0], s["WP"][0])
        u = L + 1 - ex
        b0 = tet(L + 1) - tet(u)
        for m in range(L + 1):
            if m <= L - ex:
                Y[b0 + m] = c[m]
        p = [0.0] * (L + 2)
        for ey in range(1, L + 1):
            if ey <= L - ex:
                self.vstep(L, c, p, ey, s["PA"][1], s["WP"][1])
                bo = b0 + ey * u - ey * (ey - 1) // 2
                for m in range(L - ey + 1):
                    if m <= L - ex - ey:
                        Y[bo + m] = c[m]

    def vrr_z(self, L, NMAX, ent, Y, W):
        s = self.s
        if ent < 0:
            return
        ex, ey = ent & 255, ent >> 8
        n = L - ex - ey
        b = toff(ex, ey, L)
        c = [Y[b + m] if m <= n else 0.0 for m in range(NMAX + 1)] + [0.0]
        p = [0.0] * (NMAX + 2)
        W[b] = c[0]
        for ez in range(1, NMAX + 1):
            if ez <= n:
                self.vstep(NMAX, c, p, ez, s["PA"][2], s["WP"][2])
                W[b + ez] = c[0]

    def etr_x(self, L, F, NMAX, ent, W):
        s = self.s
        if ent < 0:
            return
        ey, ez = ent & 255, ent >> 8
        n = L - ey - ez
        q = ey * (ey - 1) // 2
        r1 = [W[tet(L + 1) - tet(L + 1 - ex) + ey * (L + 1 - ex) - q + ez] if ex <= n else 0.0
              for ex in range(NMAX + 1)] + [0.0]
        r0 = [0.0] * (NMAX + 2)
        for fx in range(1, F + 1):
            if fx > NMAX:
                break
            ext = n - fx
            self.tstep(NMAX, r1, r0, fx - 1, ext, s["CE"][0], NMAX - fx)
            g = L - fx
            z = zb(L, F, fx, 0)
            for ex in range(NMAX - fx + 1):
                if ex <= ext:
                    W[z + tet(g + 1) - tet(g + 1 - ex) + ey * (g + 1 - ex) - q + ez] = r1[ex]

    def etr_y(self, L, F, EMAX, FX, NMAX, ent, W):
        s = self.s
        if ent < 0:
            return
        ex, ez = ent & 255, ent >> 8
        n = min(EMAX + F - FX - ex, L - FX - ex - ez)
        g = L - FX
        b = zb(L, F, FX, 0) + tet(g + 1) - tet(g + 1 - ex) + ez
        u = g + 1 - ex
        r1 = [W[b + ey * u - ey * (ey - 1) // 2] if ey <= n else 0.0
              for ey in range(NMAX + 1)] + [0.0]
        r0 = [0.0] * (NMAX + 2)
        for fy in range(1, F - FX + 1):
            if fy > NMAX:
                break
            ext = n - fy
            self.tstep(NMAX, r1, r0, fy - 1, ext, s["CE"][1], NMAX - fy)
            g = L - FX - fy
            b = zb(L, F, FX, fy) + tet(g + 1) - tet(g + 1 - ex) + ez
            u = g + 1 - ex
            for ey in range(NMAX - fy + 1):
                if ey <= ext:
                    W[b + ey * u - ey * (ey - 1) // 2] = r1[ey]

    def etr_z(self, L, F, LA, EMAX, LC, NF, NMAX, FZMAX, ent, W, ACC, first):
        s = self.s
        if ent[0] < 0:
            return
        x = ent[0]
        ex, ey, fx, fy = x & 15, (x >> 4) & 15, (x >> 8) & 15, (x >> 12) & 15
        sl, t = ex + ey, fx + fy
        n, fzmax = L - sl - t, F - t
        r1 = [W[ent[1] + ez] if ez <= n else 0.0 for ez in range(NMAX + 1)] + [0.0]
        r0 = [0.0] * (NMAX + 2)
        for fz in range(FZMAX + 1):
            if fz > fzmax:
                break
            if fz >= 1:
                self.tstep(NMAX, r1, r0, fz - 1, n - fz, s["CE"][2], NMAX - fz)
            tf = t + fz
            if tf >= LC:
                jf = -tet(LC) + tet(tf) + (fy + fz) * (fy + fz + 1) // 2 + fz
                for ez in range(NMAX - fz + 1):
                    se = sl + ez
                    if ez <= n - fz and LA <= se <= EMAX:
                        ie = -tet(LA) + tet(se) + (ey + ez) * (ey + ez + 1) // 2 + ez
                        i = ie * NF + jf
                        ACC[i] = r1[ez] if first else ACC[i] + r1[ez]


class Buf(list):
    """Shared-memory stand-in: every index must lie inside the buffer."""

    def __getitem__(self, i):
        assert 0 <= i < len(self), i
        return list.__getitem__(self, i)

    def __setitem__(self, i, v):
        assert 0 <= i < len(self), i
        list.__setitem__(self, i, v)


def run_generated(cls, s, Fs):
    """Execute the generated prim() of `cls` (all 32 lanes) and return ACC."""
    S = gen_lines.Schedule(*cls)
    code, tab = gen_lines.emit_class(S, "kLinesTab", 0)
    dev = Dev(s)
    W = Buf([float("nan")] * S.w_size)
    Y = Buf([float("nan")] * S.y_size)
    ACC = Buf([float("nan")] * (S.NE * S.NF))
    for line in code.splitlines():
        line = line.strip()
        m = re.match(r"(lines_\w+)<([\d, ]+)>\((.*)\);", line)
        if not m:
            continue
        name, targs = m.group(1), [int(v) for v in m.group(2).split(",")]
        offs = [int(v) for v in re.findall(r"kLinesTab \+ (\d+) \+ lane", m.group(3))]
        for lane in range(32):
            if name == "lines_vrr_xy":
                dev.vrr_xy(targs[0], lane, Fs, Y)
            elif name == "lines_vrr_z":
                dev.vrr_z(*targs, tab[offs[0] + lane], Y, W)
            elif name == "lines_etr_x":
                dev.etr_x(*targs, tab[offs[0] + lane], W)
            elif name == "lines_etr_y":
                dev.etr_y(*targs, tab[offs[0] + lane], W)
            elif name == "lines_etr_z":
                dev.etr_z(*targs, (tab[offs[0] + lane], tab[offs[1] + lane]), W, ACC, True)
            else:
                raise AssertionError(name)
    return S, np.array(list(ACC))


def direct(cls, s, Fs):
    PA, WP, CE = s["PA"], s["WP"], s["CE"]

    @lru_cache(None)
    def V(e, m):
        if min(e) < 0:
            return 0.0
        if sum(e) == 0:
            return Fs[m]
        i = 2 if e[2] else (1 if e[1] else 0)
        e1 = tuple(v - (k == i) for k, v in enumerate(e))
        e2 = tuple(v - (k == i) for k, v in enumerate(e1))
        return PA[i] * V(e1, m) + WP[i] * V(e1, m + 1) + e1[i] * s["o2z"] * (V(e2, m) - s["rz"] * V(e2, m + 1))

    @lru_cache(None)
    def E(e, f):
        if min(e) < 0 or min(f) < 0:
            return 0.0
        if sum(f) == 0:
            return V(e, 0)
        i = 2 if f[2] else (1 if f[1] else 0)
        f1 = tuple(v - (k == i) for k, v in enumerate(f))
        f2 = tuple(v - (k == i) for k, v in enumerate(f1))
        ep = tuple(v + (k == i) for k, v in enumerate(e))
        em = tuple(v - (k == i) for k, v in enumerate(e))
        return CE[i] * E(e, f1) + e[i] * s["o2e"] * E(em, f1) + f1[i] * s["o2e"] * E(e, f2) - s["ze"] * E(ep, f1)
    return E


HEAVY = [c for c in gen_eri.canonical_classes(3) if not gen_eri.is_light(c)]


@pytest.mark.parametrize("cls", HEAVY)
def test_generated_line_code_matches_recursions(cls):
    assert cls in HEAVY
    from oracle import eri_oracle as orc
    rng = np.random.default_rng(sum(cls))
    L = sum(cls)
    Fs = [float(orc.boys(m, 0.9)) for m in range(L + 1)]
    s = {"PA": rng.uniform(-0.4, 0.4, 3), "WP": rng.uniform(-0.4, 0.4, 3),
         "CE": rng.uniform(-0.4, 0.4, 3), "o2z": 0.35, "rz": 0.45, "ze": 0.8, "o2e": 0.3}
    S, acc = run_generated(cls, s, Fs)
    E = direct(cls, s, Fs)
    la, lb, lc, ld = cls
    ref = np.array([E(e, f) for e in gen_eri.comps_range(la, la + lb)
                    for f in gen_eri.comps_range(lc, lc + ld)])
    assert not np.isnan(acc).any()
    np.testing.assert_allclose(acc, ref, rtol=1e-12, atol=1e-14 * np.abs(ref).max())


def test_every_heavy_class_schedules_and_fits():
    for c in HEAVY:
        S = gen_lines.Schedule(*c)
        per_warp = (S.NE * S.NF + S.w_size + S.y_size + S.L + 1) * 8
        assert per_warp < 200 * 1024, c
        code, tab = gen_lines.emit_class(S, "kLinesTab", 0)
        assert all(-1 <= v < (1 << 16) for v in tab)


SPLIT = [c for c in HEAVY if gen_lines.split_ok(c)]


@pytest.mark.parametrize("cls", SPLIT)
def test_split_parts_cover_targets(cls):
    """The split kernel's per-warp parts (generated straight-line recursions, executed here
    as Python) reassemble the full [e0|f0] at the rows e0(r).. of each part."""
    from oracle import eri_oracle as orc
    rng = np.random.default_rng(3 + sum(cls))
    L = sum(cls)
    Fs = [float(orc.boys(m, 0.6)) for m in range(L + 1)]
    s = {"PA": rng.uniform(-0.4, 0.4, 3), "WP": rng.uniform(-0.4, 0.4, 3),
         "CE": rng.uniform(-0.4, 0.4, 3), "o2z": 0.35, "rz": 0.45, "ze": 0.8, "o2e": 0.3}
    code = gen_lines.emit_split(cls)
    la, lb, lc, ld = cls
    E = gen_eri.comps_range(la, la + lb)
    F = gen_eri.comps_range(lc, lc + ld)
    parts = gen_lines.split_parts(cls, gen_lines.split_ok(cls))
    got = np.full(len(E) * len(F), np.nan)
    bodies = re.split(r"static __device__ __forceinline__ void part\d\(", code)[1:1 + len(parts)]
    for (e0, e1), body in zip(parts, bodies):
        body = body.split("{", 1)[1].split("\n  }\n", 1)[0]
        lines = [ln.strip().rstrip(";") for ln in body.split("\n")]
        lines = [re.sub(r"^const double ", "", ln) for ln in lines
                 if ln and not ln.startswith("(void)") and ln != "}"]
        acc = [0.0] * ((e1 - e0) * len(F))
        env = dict(fma=lambda x, y, w: x * y + w, double=float, F=Fs, acc=acc,
                   PAx=s["PA"][0], PAy=s["PA"][1], PAz=s["PA"][2], WPx=s["WP"][0], WPy=s["WP"][1],
                   WPz=s["WP"][2], o2z=s["o2z"], rz=s["rz"], CEx=s["CE"][0], CEy=s["CE"][1],
                   CEz=s["CE"][2], ze=s["ze"], o2e=s["o2e"])
        exec("\n".join(lines), env)
        got[e0 * len(F):e1 * len(F)] = acc
    Ed = direct(cls, s, Fs)
    ref = np.array([Ed(e, f) for e in E for f in F])
    np.testing.assert_allclose(got, ref, rtol=1e-12, atol=1e-14 * np.abs(ref).max())


def _stages(lines):
    """Split generated prim code into stages at the barriers: per stage the round calls."""
    out, cur = [], []
    for ln in lines:
        if "__syncwarp();" in ln or "__syncthreads();" in ln:
            out.append(cur)
            cur = []
        elif "lines_" in ln:
            cur.append(ln)
    out.append(cur)
    return out


def test_group_form_runs_every_round_once():
    """The line kernel's group form (prim_g, a CTA of GROUP_W warps per quartet) runs exactly
    the one-warp prim's calls, stage by stage, each on one warp in range (vrr_xy on warp 0)."""
    heavy = [c for c in gen_eri.canonical_classes(3) if not gen_eri.is_light(c)]
    grouped = 0
    for c in heavy:
        code, _ = gen_lines.emit_class(gen_lines.Schedule(*c), "kLinesTab", 0)
        has = "prim_g(" in code
        assert has == (not gen_lines.tail_fits(c)), c
        if not has:
            continue
        grouped += 1
        one = code[code.index("void prim("):code.index("prim_g(")].splitlines()
        grp = code[code.index("prim_g("):].splitlines()
        s1, s2 = _stages(one), _stages(grp)
        assert len(s1) == len(s2), c
        for a, b in zip(s1, s2):
            calls = []
            for ln in b:
                m = re.match(r"\s*if \(wq == (\d+)\) (lines_.*)$", ln)
                assert m, (c, ln)
                w = int(m.group(1))
                assert 0 <= w < gen_lines.GROUP_W
                if "lines_vrr_xy<" in ln:
                    assert w == 0
                calls.append(m.group(2).strip())
            assert sorted(x.strip() for x in a) == sorted(calls), c
    assert grouped > 0
