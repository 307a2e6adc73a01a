// Line-factorised cooperative ERI kernel for heavy classes: one warp per contracted quartet.
//
// Every step of the Obara-Saika vertical recursion and of the electron transfer couples
// neighbours along one Cartesian axis only (the step direction is z if that component is
// non-zero, else y, else x), so a primitive quartet splits into stages of independent 1-D
// lines, each run by one lane in registers:
//   vrr_xy  lane e_x:          [(ex,0,0)]^(m) by x steps, then [(ex,ey,0)]^(m) by y steps -> Y
//   vrr_z   line (ex,ey):      [(ex,ey,ez)]^(0) by z steps                              -> W(0,0)
//   etr_x   line (ey,ez):      table (ex, fx): [e,(fx,0,0)]                             -> W(fx,0)
//   etr_y   line (ex,ez), fx:  table (ey, fy): [e,(fx,fy,0)]                            -> W(fx,fy)
//   etr_z   line (ex,ey,fx,fy): table (ez, fz): [e,f], targets added to ACC[e][f]
// Values cross shared memory once between stages.  W is a set of tetrahedral blocks, one per
// (fx, fy): element (ex,ey,ez) of block (fx,fy) sits at zb(fx,fy) + toff(ex,ey,g) + ez with
// g = L - fx - fy; Y has the layout of block (0,0) with m in place of ez.  Lines come in
// rounds of 32 (one per lane, generated tables); a round's code is unrolled to its largest
// extent NMAX and each lane predicates its own cells.
//
// Recursions (gbasis/integrals/_two_elec_int.py:350-526):
//   [e+1_i]^(m) = PA_i [e]^(m) + WP_i [e]^(m+1) + e_i/(2 zeta) ([e-1_i]^(m) - rho/zeta [e-1_i]^(m+1))
//   [e, f+1_i] = CE_i [e,f] + e_i/(2 eta) [e-1_i,f] + f_i/(2 eta) [e,f-1_i] - zeta/eta [e+1_i,f]
#pragma once
#include "coop_tail.cuh"
#include "eri_kernels.cuh"  // sph_axis, gen::Sph, gen::cnorm

namespace gbx {

__host__ __device__ constexpr int lines_tet(int k) { return k * (k + 1) * (k + 2) / 6; }

// Warps per CTA of the line kernel's group form (gen_lines.py GROUP_W).
constexpr int kLinesGroupW = 4;

// Offset of (ex, ey, 0) in a tetrahedral block of extent g (ex + ey + ez <= g).
__host__ __device__ constexpr int lines_toff(int ex, int ey, int g) {
  return lines_tet(g + 1) - lines_tet(g + 1 - ex) + ey * (g + 1 - ex) - ey * (ey - 1) / 2;
}

// Start of W block (fx, fy): blocks in order fx = 0..F, fy = 0..F-fx.
__host__ __device__ constexpr int lines_zb(int L, int F, int fx, int fy) {
  int off = 0;
  for (int a = 0; a <= F; ++a)
    for (int b = 0; b <= F - a; ++b) {
      if (a == fx && b == fy) return off;
      off += lines_tet(L - a - b + 1);
    }
  return off;
}

struct LinePS {
  double PAx, PAy, PAz, WPx, WPy, WPz, CEx, CEy, CEz;
  double o2z, rz, ze, o2e;
};

// One step of the vertical recursion along an axis: c holds [k-1]^(m), p holds [k-2]^(m);
// afterwards c holds [k]^(m) for m <= M - k and p holds the old c.
template <int M>
__device__ __forceinline__ void lines_vstep(double* c, double* p, int k, double PA, double WP,
                                            double o2z, double rz) {
  const double a = (double)(k - 1) * o2z;
#pragma unroll
  for (int m = 0; m <= M; ++m) {
    if (m <= M - k) {
      double v = fma(PA, c[m], WP * c[m + 1]);
      v = fma(a, fma(-rz, p[m + 1], p[m]), v);
      p[m] = c[m];
      c[m] = v;
    }
  }
}

// One transfer step along an axis over a line's cells a <= M: r1 = [.., f] (cells a), r0 =
// [.., f - 1_i]; k = f_i of f.  Result cell a = CE r1[a] - ze r1[a+1] + a/(2 eta) r1[a-1]
// + k/(2 eta) r0[a]; r0 <- r1, r1 <- result.
template <int M>
__device__ __forceinline__ void lines_tstep(double* r1, double* r0, int k, int ext, double CE,
                                            double ze, double o2e, int lim) {
  // cells a <= lim (a compile-time bound at every unrolled call site); the rest stay zero
  double nw[M + 1];
  const double kk = (double)k * o2e;
#pragma unroll
  for (int a = 0; a <= M; ++a) {
    if (a <= lim) {
      double v = fma(CE, r1[a], -ze * r1[a + 1]);
      if (a >= 1) v = fma((double)a * o2e, r1[a - 1], v);
      v = fma(kk, r0[a], v);
      nw[a] = (a <= ext) ? v : 0.0;
    } else {
      nw[a] = 0.0;
    }
  }
#pragma unroll
  for (int a = 0; a <= M; ++a) {
    r0[a] = r1[a];
    r1[a] = nw[a];
  }
}

// VRR along x then y; lane ex <= L writes Y[toff(ex, ey, L) + m] = [(ex,ey,0)]^(m).
template <int L>
__device__ __forceinline__ void lines_vrr_xy(int lane, const double* Fs, const LinePS& s,
                                             double* __restrict__ Y) {
  const int ex = lane;
  if (ex > L) return;
  double c[L + 2], p[L + 2];
#pragma unroll
  for (int m = 0; m <= L; ++m) {
    c[m] = Fs[m];
    p[m] = 0.0;
  }
  c[L + 1] = 0.0;
  p[L + 1] = 0.0;
#pragma unroll
  for (int k = 1; k <= L; ++k)
    if (k <= ex) lines_vstep<L>(c, p, k, s.PAx, s.WPx, s.o2z, s.rz);
  const int u = L + 1 - ex;
  const int b0 = lines_tet(L + 1) - lines_tet(u);
#pragma unroll
  for (int m = 0; m <= L; ++m)
    if (m <= L - ex) Y[b0 + m] = c[m];
#pragma unroll
  for (int m = 0; m <= L + 1; ++m) p[m] = 0.0;
#pragma unroll
  for (int ey = 1; ey <= L; ++ey) {
    if (ey <= L - ex) {
      lines_vstep<L>(c, p, ey, s.PAy, s.WPy, s.o2z, s.rz);
      const int bo = b0 + ey * u - ey * (ey - 1) / 2;
#pragma unroll
      for (int m = 0; m <= L - ey; ++m)
        if (m <= L - ex - ey) Y[bo + m] = c[m];
    }
  }
}

// VRR along z for line (ex, ey) = (ent & 255, ent >> 8); n = L - ex - ey <= NMAX.
template <int L, int NMAX>
__device__ __forceinline__ void lines_vrr_z(int ent, const LinePS& s, const double* __restrict__ Y,
                                            double* __restrict__ W) {
  if (ent < 0) return;
  const int ex = ent & 255, ey = ent >> 8;
  const int n = L - ex - ey;
  const int b = lines_toff(ex, ey, L);  // same offset in Y and in W block (0, 0)
  double c[NMAX + 2], p[NMAX + 2];
#pragma unroll
  for (int m = 0; m <= NMAX; ++m) {
    c[m] = (m <= n) ? Y[b + m] : 0.0;
    p[m] = 0.0;
  }
  c[NMAX + 1] = 0.0;
  p[NMAX + 1] = 0.0;
  W[b] = c[0];
#pragma unroll
  for (int ez = 1; ez <= NMAX; ++ez) {
    if (ez <= n) {
      lines_vstep<NMAX>(c, p, ez, s.PAz, s.WPz, s.o2z, s.rz);
      W[b + ez] = c[0];
    }
  }
}

// Transfer along x for line (ey, ez) = (ent & 255, ent >> 8): cells ex <= n - fx, n = L-ey-ez.
template <int L, int F, int NMAX>
__device__ __forceinline__ void lines_etr_x(int ent, const LinePS& s, double* __restrict__ W) {
  if (ent < 0) return;
  const int ey = ent & 255, ez = ent >> 8;
  const int n = L - ey - ez;
  const int q = ey * (ey - 1) / 2;
  double r1[NMAX + 2], r0[NMAX + 2];
#pragma unroll
  for (int ex = 0; ex <= NMAX; ++ex) {
    r1[ex] = (ex <= n) ? W[lines_tet(L + 1) - lines_tet(L + 1 - ex) + ey * (L + 1 - ex) - q + ez]
                       : 0.0;
    r0[ex] = 0.0;
  }
  r1[NMAX + 1] = 0.0;
  r0[NMAX + 1] = 0.0;
#pragma unroll
  for (int fx = 1; fx <= F; ++fx) {
    if (fx > NMAX) break;
    const int ext = n - fx;
    lines_tstep<NMAX>(r1, r0, fx - 1, ext, s.CEx, s.ze, s.o2e, NMAX - fx);
    const int g = L - fx;
    const int zb = lines_zb(L, F, fx, 0);
#pragma unroll
    for (int ex = 0; ex <= NMAX - fx; ++ex)
      if (ex <= ext)
        W[zb + lines_tet(g + 1) - lines_tet(g + 1 - ex) + ey * (g + 1 - ex) - q + ez] = r1[ex];
  }
}

// Transfer along y for line (ex, ez) = (ent & 255, ent >> 8) at fx = FX: cells ey <= n - fy,
// n = min(EMAX + F - FX - ex, L - FX - ex - ez).
template <int L, int F, int EMAX, int FX, int NMAX>
__device__ __forceinline__ void lines_etr_y(int ent, const LinePS& s, double* __restrict__ W) {
  if (ent < 0) return;
  const int ex = ent & 255, ez = ent >> 8;
  const int n = min(EMAX + F - FX - ex, L - FX - ex - ez);
  double r1[NMAX + 2], r0[NMAX + 2];
  {
    constexpr int g = L - FX;
    constexpr int zb = lines_zb(L, F, FX, 0);
    const int b = zb + lines_tet(g + 1) - lines_tet(g + 1 - ex) + ez;
    const int u = g + 1 - ex;
#pragma unroll
    for (int ey = 0; ey <= NMAX; ++ey) {
      r1[ey] = (ey <= n) ? W[b + ey * u - ey * (ey - 1) / 2] : 0.0;
      r0[ey] = 0.0;
    }
  }
  r1[NMAX + 1] = 0.0;
  r0[NMAX + 1] = 0.0;
#pragma unroll
  for (int fy = 1; fy <= F - FX; ++fy) {
    if (fy > NMAX) break;
    const int ext = n - fy;
    lines_tstep<NMAX>(r1, r0, fy - 1, ext, s.CEy, s.ze, s.o2e, NMAX - fy);
    const int g = L - FX - fy;
    const int b = lines_zb(L, F, FX, fy) + lines_tet(g + 1) - lines_tet(g + 1 - ex) + ez;
    const int u = g + 1 - ex;
#pragma unroll
    for (int ey = 0; ey <= NMAX - fy; ++ey)
      if (ey <= ext) W[b + ey * u - ey * (ey - 1) / 2] = r1[ey];
  }
}

// Transfer along z for line (ex,ey,fx,fy) = 4-bit fields of ent.x, W offset of its first cell
// in ent.y; cells ez <= n - fz, n = L - s - t; targets (la <= s+ez <= EMAX, lc <= t+fz <= F)
// stored (first primitive) or added to ACC[ie * NF + jf].
template <int L, int F, int LA, int EMAX, int LC, int NF, int NMAX, int FZMAX>
__device__ __forceinline__ void lines_etr_z(int2 ent, const LinePS& s,
                                            const double* __restrict__ W, double* __restrict__ ACC,
                                            bool first) {
  if (ent.x < 0) return;
  const int ex = ent.x & 15, ey = (ent.x >> 4) & 15, fx = (ent.x >> 8) & 15, fy = (ent.x >> 12) & 15;
  const int sl = ex + ey, t = fx + fy;
  const int n = L - sl - t, fzmax = F - t;
  double r1[NMAX + 2], r0[NMAX + 2];
#pragma unroll
  for (int ez = 0; ez <= NMAX; ++ez) {
    r1[ez] = (ez <= n) ? W[ent.y + ez] : 0.0;
    r0[ez] = 0.0;
  }
  r1[NMAX + 1] = 0.0;
  r0[NMAX + 1] = 0.0;
  const int eb = -lines_tet(LA), fb = -lines_tet(LC);
#pragma unroll
  for (int fz = 0; fz <= FZMAX; ++fz) {
    if (fz > fzmax) break;
    if (fz >= 1) lines_tstep<NMAX>(r1, r0, fz - 1, n - fz, s.CEz, s.ze, s.o2e, NMAX - fz);
    const int tf = t + fz;
    if (tf >= LC) {
      const int jf = fb + lines_tet(tf) + (fy + fz) * (fy + fz + 1) / 2 + fz;
#pragma unroll
      for (int ez = 0; ez <= NMAX - fz; ++ez) {
        const int se = sl + ez;
        if (ez <= n - fz && se >= LA && se <= EMAX) {
          const int ie = eb + lines_tet(se) + (ey + ez) * (ey + ez + 1) / 2 + ez;
          double* dst = ACC + ie * NF + jf;
          *dst = first ? r1[ez] : *dst + r1[ez];
        }
      }
    }
  }
}

// Register tail of classes whose ket block (NCD) and bra block (NAB) fit a lane: lanes take
// rows e of ACC and run the ket horizontal recursion and ket transforms in registers (T::ket),
// writing HF[e][cd]; then lanes take output columns (c, d) and run the bra recursion
// (T::bra), bra transforms, scaling and the store (mode 0) or the Schwarz maximum (mode 1).
template <int LA, int LB, int LC, int LD, class T>
__device__ __forceinline__ void lines_tail(const EriLaunch& a, const double* ACC, double* HF,
                                           const int2 pq, const PairDev& P, const PairDev& Q,
                                           const int lane, int NE, int NF) {
  constexpr int NCA = ncart(LA), NCB = ncart(LB), NCC = ncart(LC), NCDD = ncart(LD);
  constexpr int NCD = NCC * NCDD, NAB = NCA * NCB;
  const ShellDev& sA = a.shells[P.shA];
  const ShellDev& sB = a.shells[P.shB];
  const ShellDev& sC = a.shells[Q.shA];
  const ShellDev& sD = a.shells[Q.shB];
  const bool schwarz = a.mode == 1;
  for (int e = lane; e < NE; e += 32) {
    double h[NCD];
    T::ket(ACC + e * NF, Q.ABx, Q.ABy, Q.ABz, h);
    if (!schwarz) {
      if (LD >= 2 && sD.sph) sph_axis<LD, NCC, 1>(h);
      if (LC >= 2 && sC.sph) sph_axis<LC, 1, NCDD>(h);
    }
#pragma unroll
    for (int i = 0; i < NCD; ++i) HF[e * NCD + i] = h[i];
  }
  __syncwarp();
  const int nAi = schwarz ? NCA : internal_count(sA), nBi = schwarz ? NCB : internal_count(sB);
  const int nCi = schwarz ? NCC : internal_count(sC), nDi = schwarz ? NCDD : internal_count(sD);
  const int ncol = nCi * nDi;
  long long bbase, bcols;
  block_dest(a, P, bbase, bcols);
  // strides of the bra and ket pair-function indices (transposed: quartet_transposed)
  const bool tr = quartet_transposed(P, Q);
  const long long sbra = tr ? 1 : bcols, sket = tr ? bcols : 1;
  const long long nBo = sB.nout, nDo = sD.nout;
  double mx = 0.0;
  for (int k = lane; k < ncol; k += 32) {
    const int uc = k / nDi, ud = k - uc * nDi;
    double o[NAB];
    T::bra(HF + uc * NCDD + ud, NCD, P.ABx, P.ABy, P.ABz, o);
    if (schwarz) {
      const double wcd = gen::cnorm<LC>(uc) * gen::cnorm<LD>(ud);
#pragma unroll
      for (int ia = 0; ia < NCA; ++ia)
#pragma unroll
        for (int ib = 0; ib < NCB; ++ib)
          mx = fmax(mx, fabs(o[ia * NCB + ib]) * (gen::cnorm<LA>(ia) * gen::cnorm<LB>(ib) * wcd));
      continue;
    }
    if (LB >= 2 && sB.sph) sph_axis<LB, NCA, 1>(o);
    if (LA >= 2 && sA.sph) sph_axis<LA, 1, NCB>(o);
    const double fcd = sC.scl[uc] * sD.scl[ud];
    const long long col = bbase + ((long long)Q.fo + sC.pos[uc] * nDo + sD.pos[ud]) * sket;
#pragma unroll
    for (int ia = 0; ia < NCA; ++ia) {
      if (ia >= nAi) break;
      const double fa = sA.scl[ia] * fcd;
      const long long ra = (long long)P.fo + sA.pos[ia] * nBo;
#pragma unroll
      for (int ib = 0; ib < NCB; ++ib) {
        if (ib >= nBi) break;
        out_store(a, col + (ra + sB.pos[ib]) * sbra, o[ia * NCB + ib] * fa * sB.scl[ib]);
      }
    }
  }
  if (schwarz) {
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) a.qout[pq.x] = sqrt(mx);
  }
  __syncwarp();
}

// The kernel: per quartet, ACC[e][f] over the primitive quartets by C::prim, then the shared
// tail (HRR, transforms, store / Schwarz / Coulomb epilogue).  Per warp shared memory:
// ACC | W | Y | Boys values, the tail's buffers overlaying W.
template <class C, bool COULOMB, bool ATT = false>
__global__ void __launch_bounds__(128, 4) eri_lines(const CoopArgs A) {
  extern __shared__ double smem[];
  const EriLaunch& a = A.a;
  const CoopMeta& M = A.m;
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  short(*s_ins)[8] = reinterpret_cast<short(*)[8]>(smem);
  short* s_idx = reinterpret_cast<short*>(smem) + 8 * M.n_ins;
  const bool staged = A.prog_doubles > 0;
  // no quartet for any warp of this CTA: leave before staging (the test is CTA-uniform)
  if ((long long)blockIdx.x * (blockDim.x >> 5) >=
      (a.work_count ? (long long)(*a.work_count) : a.nwork))
    return;
  if (staged) {
    const int4* src = reinterpret_cast<const int4*>(&kCoopIns[M.v_ins][0]);
    int4* dst4 = reinterpret_cast<int4*>(smem);
    for (int i = threadIdx.x; i < M.n_ins; i += blockDim.x) dst4[i] = src[i];
    for (int i = threadIdx.x; i < M.n_idx; i += blockDim.x) s_idx[i] = kCoopIdx[M.targets + i];
    __syncthreads();
  }
  const ProgView pv = staged ? ProgView{s_ins, s_idx, M.v_ins, M.targets}
                             : ProgView{kCoopIns, kCoopIdx, 0, 0};
  double* S = smem + A.prog_doubles + (size_t)wib * A.smem_per_warp;
  double* ACC = S;
  double* W = S + C::NE * C::NF;
  double* Y = W + C::kW;
  double* Fs = Y + C::kY;
  const long long count = a.work_count ? (long long)(*a.work_count) : a.nwork;
  const long long nwarps = (long long)gridDim.x * (blockDim.x >> 5);
  unsigned long long* const tk = a.ticket;  // one quartet per draw
  for (long long w = tk ? warp_ticket(tk, lane) : (long long)blockIdx.x * (blockDim.x >> 5) + wib;
       w < count; w = tk ? warp_ticket(tk, lane) : w + nwarps) {
    const int2 pq = a.work[a.reverse ? a.work_off + a.nwork - 1 - w : a.work_off + w];
    const PairDev P = a.pairs[pq.x];
    const PairDev Q = a.pairs[pq.y];
    // primitive quartets in one flat loop; the next pair data are loaded one step ahead
    const int np = P.nprim * Q.nprim;
    PrimPair bp = a.prims[P.prim_off], kp = a.prims[Q.prim_off];
    for (int idx = 0; idx < np; ++idx) {
      PrimPair bpn = bp, kpn = kp;
      if (idx + 1 < np) {
        const int ip = (idx + 1) / Q.nprim, jq = idx + 1 - ip * Q.nprim;
        bpn = a.prims[P.prim_off + ip];
        kpn = a.prims[Q.prim_off + jq];
      }
      const double r = rsqrt(bp.zeta + kp.zeta);
      const double inv = r * r;
      const double PQx = bp.Px - kp.Px, PQy = bp.Py - kp.Py, PQz = bp.Pz - kp.Pz;
      const double rz = kp.zeta * inv;
      const double T = bp.zeta * rz * fma(PQx, PQx, fma(PQy, PQy, PQz * PQz));
      LinePS ps;
      ps.PAx = bp.Xx;
      ps.PAy = bp.Xy;
      ps.PAz = bp.Xz;
      ps.WPx = -rz * PQx;
      ps.WPy = -rz * PQy;
      ps.WPz = -rz * PQz;
      ps.o2z = 0.5 * bp.izeta;
      ps.rz = rz;
      ps.ze = bp.zeta * kp.izeta;
      ps.o2e = 0.5 * kp.izeta;
      ps.CEx = fma(ps.ze, bp.Xx, kp.Xx);
      ps.CEy = fma(ps.ze, bp.Xy, kp.Xy);
      ps.CEz = fma(ps.ze, bp.Xz, kp.Xz);
      boys_lanes(C::L, lane, T, bp.C * kp.C * r, a.boys_tab, Fs, ATT ? a.potential : 0, a.omega,
                 bp.zeta * rz);
      __syncwarp();
      C::prim(lane, Fs, ps, W, Y, ACC, idx == 0);
      __syncwarp();
      bp = bpn;
      kp = kpn;
    }
    if (np == 0) {  // no primitive quartet (a pair left without primitives): zero targets
      for (int i = lane; i < C::NE * C::NF; i += 32) ACC[i] = 0.0;
      __syncwarp();
    }
    if constexpr (C::kRegTail && !COULOMB) {
      lines_tail<C::LA, C::LB, C::LC, C::LD, typename C::Tail>(a, S, S + C::NE * C::NF, pq, P, Q,
                                                               lane, C::NE, C::NF);
    } else {
      coop_tail(A, pv, S, pq, P, Q, lane);
    }
  }
}

// Group form of the line kernel, for classes with the interpreted tail whose per-warp buffers
// leave few warps on an SM: a CTA of kLinesGroupW warps holds one quartet in one buffer.  Per
// primitive quartet warp 0 evaluates the Boys values, then C::prim_g runs each stage's rounds of
// lines on the warps the generator gave them (vrr_xy on warp 0), with a CTA barrier between
// stages; the interpreted tail then runs on all the CTA's threads (modes 0 and 2).  Same
// arithmetic per line and per tail step as eri_lines.
template <class C>
__global__ void __launch_bounds__(32 * kLinesGroupW, 4) eri_lines_grp(const CoopArgs A) {
  extern __shared__ double smem[];
  const EriLaunch& a = A.a;
  const CoopMeta& M = A.m;
  const int lane = threadIdx.x & 31, wq = threadIdx.x >> 5;
  const long long count = a.work_count ? (long long)(*a.work_count) : a.nwork;
  if ((long long)blockIdx.x >= count) return;  // no quartet for this CTA (uniform)
  short(*s_ins)[8] = reinterpret_cast<short(*)[8]>(smem);
  short* s_idx = reinterpret_cast<short*>(smem) + 8 * M.n_ins;
  const bool staged = A.prog_doubles > 0;
  if (staged) {
    const int4* src = reinterpret_cast<const int4*>(&kCoopIns[M.v_ins][0]);
    int4* dst4 = reinterpret_cast<int4*>(smem);
    for (int i = threadIdx.x; i < M.n_ins; i += blockDim.x) dst4[i] = src[i];
    for (int i = threadIdx.x; i < M.n_idx; i += blockDim.x) s_idx[i] = kCoopIdx[M.targets + i];
  }
  const ProgView pv = staged ? ProgView{s_ins, s_idx, M.v_ins, M.targets}
                             : ProgView{kCoopIns, kCoopIdx, 0, 0};
  double* S = smem + A.prog_doubles;
  double* ACC = S;
  double* W = S + C::NE * C::NF;
  double* Y = W + C::kW;
  double* Fs = Y + C::kY;
  unsigned long long* const tk = a.ticket;  // one quartet per draw, by thread 0
  __shared__ long long s_w;
  long long w = blockIdx.x;
  for (;;) {
    if (tk) {
      if (threadIdx.x == 0) s_w = (long long)atomicAdd(tk, 1ull);
      __syncthreads();  // also: programs staged (first quartet), previous tail done
      w = s_w;
    } else {
      __syncthreads();
    }
    if (w >= count) break;  // the same for all threads of the CTA
    const int2 pq = a.work[a.reverse ? a.work_off + a.nwork - 1 - w : a.work_off + w];
    const PairDev P = a.pairs[pq.x];
    const PairDev Q = a.pairs[pq.y];
    const int np = P.nprim * Q.nprim;
    for (int idx = 0; idx < np; ++idx) {
      const int ip = idx / Q.nprim, jq = idx - ip * Q.nprim;
      const PrimPair bp = a.prims[P.prim_off + ip], kp = a.prims[Q.prim_off + jq];
      const double r = rsqrt(bp.zeta + kp.zeta);
      const double inv = r * r;
      const double PQx = bp.Px - kp.Px, PQy = bp.Py - kp.Py, PQz = bp.Pz - kp.Pz;
      const double rz = kp.zeta * inv;
      const double T = bp.zeta * rz * fma(PQx, PQx, fma(PQy, PQy, PQz * PQz));
      LinePS ps;
      ps.PAx = bp.Xx;
      ps.PAy = bp.Xy;
      ps.PAz = bp.Xz;
      ps.WPx = -rz * PQx;
      ps.WPy = -rz * PQy;
      ps.WPz = -rz * PQz;
      ps.o2z = 0.5 * bp.izeta;
      ps.rz = rz;
      ps.ze = bp.zeta * kp.izeta;
      ps.o2e = 0.5 * kp.izeta;
      ps.CEx = fma(ps.ze, bp.Xx, kp.Xx);
      ps.CEy = fma(ps.ze, bp.Xy, kp.Xy);
      ps.CEz = fma(ps.ze, bp.Xz, kp.Xz);
      if (wq == 0)
        boys_lanes(C::L, lane, T, bp.C * kp.C * r, a.boys_tab, Fs, a.potential, a.omega,
                   bp.zeta * rz);
      __syncthreads();
      C::prim_g(wq, lane, Fs, ps, W, Y, ACC, idx == 0);
      __syncthreads();
    }
    if (np == 0) {  // no primitive quartet (a pair left without primitives): zero targets
      for (int i = threadIdx.x; i < C::NE * C::NF; i += blockDim.x) ACC[i] = 0.0;
      __syncthreads();
    }
    coop_tail_g(A, pv, S, pq, P, Q, CtaGroup<kLinesGroupW>{(int)threadIdx.x});
    if (!tk) w += gridDim.x;
  }
}

// Launch of the line kernel of class C (same shared-memory plan as the interpreted kernel,
// with phase A's W, Y and Boys buffers).
template <class C>
int launch_lines_t(const EriLaunch& a, const CoopMeta& m, cudaStream_t st) {
  CoopArgs A;
  A.a = a;
  A.m = m;
  size_t smem = 0;
  int wpc = 1;
  int s = GBX_OK;
  if (C::kRegTail && a.mode != 2) {
    // register tail: per warp ACC, then W | Y | Boys values, overlaid by the tail's [e0|cd]
    // rows; no interpreter buffers and no staged programs
    constexpr long long kNCD = ncart(C::LC) * ncart(C::LD);
    constexpr long long kPhaseA = (long long)C::kW + C::kY + C::L + 1;
    constexpr long long kPerWarp =
        (long long)C::NE * C::NF + (kPhaseA > C::NE * kNCD ? kPhaseA : C::NE * kNCD);
    A.R = A.Cc = 1;
    A.prog_doubles = 0;
    A.smem_per_warp = (int)kPerWarp;
    wpc = (int)std::max<long long>(1, std::min<long long>(4, kCoopMaxSmem / (kPerWarp * 8)));
    smem = (size_t)wpc * kPerWarp * 8;
  } else {
    s = coop_plan(m, (long long)C::kW + C::kY + C::L + 1, A, smem, wpc);
  }
  if (s) return s;
  if constexpr (C::kGroup) {
    // group form (a.variant 2), or by default (a.variant 0) for classes whose ket pair has no
    // s shell first (LC >= 1); not for the Schwarz diagonal (mode 1).  Measured per class on the
    // 20-atom chain's unique integrals, blocks one after another: the group form took up to
    // 55 % off the classes with LC >= 1 ((ff|df) 107 -> 56 ms, (ff|ff) 54 -> 25, (ff|pf)
    // 84 -> 65; three within 5 % either way) and cost up to 100 % on most LC = 0 classes
    // ((df|sp) 77 -> 156 ms)
    CoopArgs G;
    G.a = a;
    G.m = m;
    size_t gsmem = 0;
    int one = 1;
    // the kernel's own 8-byte ticket slot sits in static shared memory beside the plan's
    const bool group = a.mode != 1 &&
                       (a.variant == 2 || (a.variant == 0 && C::LC >= 1)) &&
                       coop_plan(m, (long long)C::kW + C::kY + C::L + 1, G, gsmem, one,
                                 16 / kLinesGroupW, true, 1) == GBX_OK &&
                       (long long)gsmem + 64 <= kCoopMaxSmem;
    if (group) {
      s = cuda_status(cudaFuncSetAttribute(eri_lines_grp<C>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)gsmem), "eri_lines_grp shared memory attribute");
      if (s) return s;
      int dev = 0, nsm = 1;
      cudaGetDevice(&dev);
      cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
      const long long grid = std::max<long long>(
          1, std::min<long long>(a.nwork, (long long)nsm * (16 / kLinesGroupW)));
      eri_lines_grp<C><<<(int)grid, 32 * kLinesGroupW, gsmem, st>>>(G);
      return cuda_status(cudaGetLastError(), "eri_lines_grp launch");
    }
  }
  // the Coulomb epilogue (mode 2) is a separate instantiation, so that the store / Schwarz
  // kernel of a class with the register tail carries no interpreted tail
  auto kern = a.potential ? (a.mode == 2 ? eri_lines<C, true, true> : eri_lines<C, false, true>)
                          : (a.mode == 2 ? eri_lines<C, true> : eri_lines<C, false>);
  s = cuda_status(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kCoopMaxSmem), "eri_lines shared memory attribute");
  if (s) return s;
  kern<<<coop_grid(a, wpc), 32 * wpc, smem, st>>>(A);
  return cuda_status(cudaGetLastError(), "eri_lines launch");
}

// Per quartet of a split CTA's group: what the tail needs, captured in shared memory while the
// quartet's pair data are in registers (the tail then makes no dependent global loads for it).
struct SplitQuartet {
  double pab[3], qab[3];
  int shA, shB, shC, shD;
  int pfo, qfo, mol, bra;
  int tr, ket;  // stored transposed (quartet_transposed); ket pair (Coulomb mode)
};

// Row stride of the split kernel's shared accumulators: a row holds NF values of [e0|f0] and,
// after the ket recursion (done in place), NCD values of [e0|cd]; odd, so that lanes reading
// consecutive rows hit different banks.
__host__ __device__ constexpr int split_rs(int nf, int ncd) { return (nf > ncd ? nf : ncd) | 1; }

// Tail of a split CTA's group of nq quartets, spread over all its threads: first tasks (quartet,
// row e) run the ket horizontal recursion and ket transforms in registers (T::ket) and write
// [e0|cd] back over the row; then tasks (quartet, output column (c, d)) run the bra recursion
// (T::bra), bra transforms, scaling and the store (mode 0), or the Schwarz maximum (mode 1).
template <int LA, int LB, int LC, int LD, class T, int NE, int RS>
__device__ __forceinline__ void split_tail(const EriLaunch& a, double* ACC,
                                           const SplitQuartet* sq, unsigned long long* s_mx,
                                           int nq, double* JAB) {
  constexpr int NCA = ncart(LA), NCB = ncart(LB), NCC = ncart(LC), NCDD = ncart(LD);
  constexpr int NCD = NCC * NCDD, NAB = NCA * NCB;
  constexpr int QS = NE * RS;
  const bool schwarz = a.mode == 1;
  const bool coulomb = a.mode == 2;  // J: JAB[q][ab] gathers sum_cd (ab|cd) D[c][d] per quartet
  if (coulomb) {
    for (int i = threadIdx.x; i < nq * NAB; i += blockDim.x) JAB[i] = 0.0;
  }
  for (int t = threadIdx.x; t < nq * NE; t += blockDim.x) {
    const int q = t / NE, e = t - q * NE;
    const SplitQuartet& s = sq[q];
    double* row = ACC + q * QS + e * RS;
    double h[NCD];
    T::ket(row, s.qab[0], s.qab[1], s.qab[2], h);
    if (!schwarz) {
      if (LD >= 2 && a.shells[s.shD].sph) sph_axis<LD, NCC, 1>(h);
      if (LC >= 2 && a.shells[s.shC].sph) sph_axis<LC, 1, NCDD>(h);
    }
#pragma unroll
    for (int i = 0; i < NCD; ++i) row[i] = h[i];
  }
  __syncthreads();
  for (int t = threadIdx.x; t < nq * NCD; t += blockDim.x) {
    const int q = t / NCD, k = t - q * NCD;
    const SplitQuartet& s = sq[q];
    const ShellDev& sA = a.shells[s.shA];
    const ShellDev& sB = a.shells[s.shB];
    const ShellDev& sC = a.shells[s.shC];
    const ShellDev& sD = a.shells[s.shD];
    const int nAi = schwarz ? NCA : internal_count(sA), nBi = schwarz ? NCB : internal_count(sB);
    const int nCi = schwarz ? NCC : internal_count(sC), nDi = schwarz ? NCDD : internal_count(sD);
    if (k >= nCi * nDi) continue;
    const int uc = k / nDi, ud = k - uc * nDi;
    double o[NAB];
    T::bra(ACC + q * QS + uc * NCDD + ud, RS, s.pab[0], s.pab[1], s.pab[2], o);
    if (schwarz) {
      const double wcd = gen::cnorm<LC>(uc) * gen::cnorm<LD>(ud);
      double mx = 0.0;
#pragma unroll
      for (int ia = 0; ia < NCA; ++ia)
#pragma unroll
        for (int ib = 0; ib < NCB; ++ib)
          mx = fmax(mx, fabs(o[ia * NCB + ib]) * (gen::cnorm<LA>(ia) * gen::cnorm<LB>(ib) * wcd));
      // non-negative doubles order like their bit patterns
      atomicMax(s_mx + q, (unsigned long long)__double_as_longlong(mx));
      continue;
    }
    if (LB >= 2 && sB.sph) sph_axis<LB, NCA, 1>(o);
    if (LA >= 2 && sA.sph) sph_axis<LA, 1, NCB>(o);
    if (coulomb) {
      // J[a][b] += (1 + [C != D]) sum_cd (ab|cd) D[c][d] (gathered in JAB, added below) and,
      // for a quartet whose pairs differ, J[c][d] += (1 + [A != B]) sum_ab (ab|cd) D[a][b]
      const long long n = a.nbf;
      const long long fc = sC.func_off + sC.pos[uc], fd = sD.func_off + sD.pos[ud];
      const double fcd = sC.scl[uc] * sD.scl[ud];
      const double dcd = a.D[fc * n + fd] * fcd;
      double scd = 0.0;
#pragma unroll
      for (int ia = 0; ia < NCA; ++ia) {
        if (ia >= nAi) break;
#pragma unroll
        for (int ib = 0; ib < NCB; ++ib) {
          if (ib >= nBi) break;
          const double v = o[ia * NCB + ib];
          atomicAdd(JAB + q * NAB + ia * NCB + ib, v * dcd);
          scd = fma(v, a.D[(sA.func_off + sA.pos[ia]) * n + sB.func_off + sB.pos[ib]] *
                           (sA.scl[ia] * sB.scl[ib]), scd);
        }
      }
      if (s.bra != s.ket) {
        const double w = scd * ((s.shA != s.shB) ? 2.0 : 1.0) * fcd;
        j_add(a, fc * n + fd, w);
        if (s.shC != s.shD) j_add(a, fd * n + fc, w);
      }
      continue;
    }
    long long bbase, bcols;
    if (a.mol_base) {
      bbase = a.mol_base[s.mol];
      bcols = a.mol_ncols[s.mol];
    } else {
      bbase = a.base;
      bcols = a.ncols;
    }
    const long long nBo = sB.nout, nDo = sD.nout;
    const double fcd = sC.scl[uc] * sD.scl[ud];
    const long long sbra = s.tr ? 1 : bcols, sket = s.tr ? bcols : 1;
    const long long col = bbase + ((long long)s.qfo + sC.pos[uc] * nDo + sD.pos[ud]) * sket;
#pragma unroll
    for (int ia = 0; ia < NCA; ++ia) {
      if (ia >= nAi) break;
      const double fa = sA.scl[ia] * fcd;
      const long long ra = (long long)s.pfo + sA.pos[ia] * nBo;
#pragma unroll
      for (int ib = 0; ib < NCB; ++ib) {
        if (ib >= nBi) break;
        out_store(a, col + (ra + sB.pos[ib]) * sbra, o[ia * NCB + ib] * fa * sB.scl[ib]);
      }
    }
  }
  if (schwarz) {
    __syncthreads();
    for (int q = threadIdx.x; q < nq; q += blockDim.x)
      a.qout[sq[q].bra] = sqrt(__longlong_as_double((long long)s_mx[q]));
  }
  if (coulomb) {
    __syncthreads();
    const long long n = a.nbf;
    for (int t = threadIdx.x; t < nq * NAB; t += blockDim.x) {
      const int q = t / NAB, i = t - q * NAB, ia = i / NCB, ib = i - ia * NCB;
      const SplitQuartet& s = sq[q];
      const ShellDev& sA = a.shells[s.shA];
      const ShellDev& sB = a.shells[s.shB];
      if (ia >= internal_count(sA) || ib >= internal_count(sB)) continue;
      const long long fa = sA.func_off + sA.pos[ia], fb = sB.func_off + sB.pos[ib];
      const double v = JAB[t] * ((s.shC != s.shD) ? 2.0 : 1.0) * sA.scl[ia] * sB.scl[ib];
      j_add(a, fa * n + fb, v);
      if (s.shA != s.shB) j_add(a, fb * n + fa, v);
    }
  }
}

// Split register kernel for heavy classes of moderate size: a CTA of S = C::kS warps (4 or 8)
// takes 32 quartets at a time, thread t of warp r computing part r (a contiguous range of bra
// rows e) of quartet t's contracted [e0|f0] in registers (generated straight-line recursions,
// as in the light classes' kernel); the parts meet in shared memory ACC[32][NE][RS] and all
// threads of the CTA then share the group's tail (split_tail): store (mode 0), Schwarz
// maximum (mode 1) or Coulomb-matrix contributions (mode 2).
template <class C, bool ATT = false>
__global__ void __launch_bounds__(C::kS * 32) eri_split(const EriLaunch a) {
  __shared__ double s_tab[kBoysNGrid * kBoysTaylor];
  __shared__ double s_exp[kBoysNGrid];
  __shared__ SplitQuartet sq[32];
  __shared__ unsigned long long s_mx[32];
  extern __shared__ double dyn[];
  constexpr int L = C::L;
  constexpr int NCD = ncart(C::LC) * ncart(C::LD);
  constexpr int RS = split_rs(C::NF, NCD);
  constexpr int QS = C::NE * RS;
  const long long count = a.work_count ? (long long)(*a.work_count) : a.nwork;
  if ((long long)blockIdx.x * 32 >= count) return;  // no quartet for this CTA (uniform)
  stage_boys<L>(a.boys_tab, s_tab, s_exp);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  double* ACC = dyn;
  // groups of 32 quartets: from the launch's work counter (thread 0 draws, the CTA reads it
  // after the barrier; the next draw comes after the group's barriers), else every gridDim-th
  __shared__ long long s_base;
  unsigned long long* const tk = a.ticket;
  long long base = (long long)blockIdx.x * 32;
  for (;;) {
    if (threadIdx.x < 32) s_mx[threadIdx.x] = 0ull;
    if (tk && threadIdx.x == 0) s_base = (long long)atomicAdd(tk, 1ull) * 32;
    __syncthreads();  // Boys table staged (first group); previous group's tail done
    if (tk) base = s_base;
    if (base >= count) break;  // the same for all threads of the CTA
    const long long w = base + lane;
    if (w < count) {
      const int2 pq = a.work[a.reverse ? a.work_off + a.nwork - 1 - w : a.work_off + w];
      const PairDev P = a.pairs[pq.x];
      const PairDev Q = a.pairs[pq.y];
      if (warp == 0) {
        SplitQuartet& s = sq[lane];
        s.pab[0] = P.ABx;
        s.pab[1] = P.ABy;
        s.pab[2] = P.ABz;
        s.qab[0] = Q.ABx;
        s.qab[1] = Q.ABy;
        s.qab[2] = Q.ABz;
        s.shA = P.shA;
        s.shB = P.shB;
        s.shC = Q.shA;
        s.shD = Q.shB;
        s.pfo = P.fo;
        s.qfo = Q.fo;
        s.mol = P.mol;
        s.bra = pq.x;
        s.tr = quartet_transposed(P, Q) ? 1 : 0;
        s.ket = pq.y;
      }
      double acc[C::kAcc];
#pragma unroll
      for (int i = 0; i < C::kAcc; ++i) acc[i] = 0.0;
      for (int ip = 0; ip < P.nprim; ++ip) {
        const PrimPair bp = a.prims[P.prim_off + ip];
        const double o2z = 0.5 * bp.izeta;
        for (int jq = 0; jq < Q.nprim; ++jq) {
          const PrimPair kp = a.prims[Q.prim_off + jq];
          const double r = rsqrt(bp.zeta + kp.zeta);
          const double inv = r * r;
          const double PQx = bp.Px - kp.Px, PQy = bp.Py - kp.Py, PQz = bp.Pz - kp.Pz;
          const double rz = kp.zeta * inv;
          const double T = bp.zeta * rz * fma(PQx, PQx, fma(PQy, PQy, PQz * PQz));
          double F[L + 1];
          boys_eval<L>(T, s_tab, s_exp, F);
          if constexpr (ATT)
            boys_attenuate<L>(a.potential, a.omega, bp.zeta * rz, T, s_tab, s_exp, F);
          const double pref = bp.C * kp.C * r;
#pragma unroll
          for (int m = 0; m <= L; ++m) F[m] *= pref;
          const double ze = bp.zeta * kp.izeta;
          C::part(warp, F, bp.Xx, bp.Xy, bp.Xz, -rz * PQx, -rz * PQy, -rz * PQz, o2z, rz,
                  fma(ze, bp.Xx, kp.Xx), fma(ze, bp.Xy, kp.Xy), fma(ze, bp.Xz, kp.Xz), ze,
                  0.5 * kp.izeta, acc);
        }
      }
      const int nv = C::ne(warp) * C::NF;
      double* dst = ACC + lane * QS + C::e0(warp) * RS;
#pragma unroll
      for (int i = 0; i < C::kAcc; ++i)
        if (i < nv) dst[(i / C::NF) * RS + i % C::NF] = acc[i];
    }
    __syncthreads();
    const int nq = (int)(count - base < 32 ? count - base : 32);
    split_tail<C::LA, C::LB, C::LC, C::LD, typename C::Tail, C::NE, RS>(a, ACC, sq, s_mx, nq,
                                                                        ACC + 32 * QS);
    __syncthreads();
    base += (long long)gridDim.x * 32;  // static order (replaced by the next draw with a counter)
  }
}

template <class C>
int launch_split_t(const EriLaunch& a, cudaStream_t st) {
  constexpr int NCD = ncart(C::LC) * ncart(C::LD);
  constexpr int NAB = ncart(C::LA) * ncart(C::LB);
  // ACC[32][NE][RS]; the Coulomb mode adds the per-quartet sums JAB[32][NAB]
  const size_t dyn = (size_t)32 * C::NE * split_rs(C::NF, NCD) * sizeof(double) +
                     (a.mode == 2 ? (size_t)32 * NAB * sizeof(double) : 0);
  auto kern = a.potential ? eri_split<C, true> : eri_split<C>;
  int s = cuda_status(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)dyn), "eri_split shared memory attribute");
  if (s) return s;
  int dev = 0, nsm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int grid = (int)std::max<long long>(1, std::min<long long>((a.nwork + 31) / 32, (long long)nsm * (32 / C::kS)));
  kern<<<grid, 32 * C::kS, dyn, st>>>(a);
  return cuda_status(cudaGetLastError(), "eri_split launch");
}

}  // namespace gbx
