// Shared pieces of the cooperative (warp-per-quartet) kernels: launch arguments, the Boys
// evaluation by lanes, and the per-quartet tail (phases B-D: ket HRR, ket Cartesian->spherical
// transform, bra HRR + transform, permutation/scale and store, Schwarz or Coulomb epilogues)
// that runs once the contracted [e0|f0] are in shared memory ACC.  Included after a
// translation unit's recursion-program tables (kCoopIns, kCoopLv, kCoopIdx, kCoopSph, kCoopCn).
// Mathematics: gbasis/integrals/_two_elec_int.py:549-812 (HRR, component norm) and
// gbasis/base_four_symm.py:195-349 (norm_cont, spherical transform).
#pragma once
#include <algorithm>

#include "coop.cuh"
#include "errors.h"

namespace gbx {

struct CoopArgs {
  EriLaunch a;
  CoopMeta m;
  int R, Cc, smem_per_warp;  // rows / columns per HRR chunk, doubles of smem per warp
  int prog_doubles;          // shared memory taken by the staged programs (0: read globally)
  int extra_doubles = 0;     // per-CTA shared memory after the programs (line kernel: Boys table)
};

constexpr long long kCoopMaxSmem = 227 * 1024;

// Shared-memory plan of a cooperative launch.  Per warp: ACC (NE*NF) followed by the larger
// of phase A's `phase_a` doubles and the tail's buffers (rows R and columns Cc per HRR chunk);
// the class's programs are staged once per CTA when they fit 32 KB; 1 to 4 warps per CTA.
// Among the chunk sizes R, Cc in {8, 4, 2, 1}, staging or not, and 1..4 warps per CTA, the plan
// keeps the one with the most warps resident per SM (228 KB of shared memory per SM, 1 KB of it
// reserved per CTA; at most `max_warps_regs` warps by registers), then the larger chunks, then
// staged programs: shared memory, not registers, is what limits these kernels' occupancy (a
// class with f shells took 125 KB per 4-warp CTA with the largest chunks: 4 warps per SM).
inline int coop_plan(const CoopMeta& M, long long phase_a, CoopArgs& A, size_t& smem, int& wpc,
                     int max_warps_regs = 16, bool allow_staged = true, int max_wpc = 4) {
  const int NCD = ncart(M.lc) * ncart(M.ld), NAB = ncart(M.la) * ncart(M.lb);
  const int NENF = M.NE * M.NF;
  const long long warp_cap = 48 * 1024 / 8;
  auto size_for = [&](int R, int Cc) {
    long long s = NENF + phase_a;
    s = std::max<long long>(s, NENF + (long long)M.NE * NCD + (long long)R * M.nK);
    s = std::max<long long>(s, NENF + (long long)M.NE * NCD + NCD);
    s = std::max<long long>(s, NENF + (long long)M.NE * NCD + (long long)Cc * (M.nB + 2 * NAB) +
                                   2 * NAB);
    return s;
  };
  const long long prog_bytes = (long long)M.n_ins * 16 + (long long)M.n_idx * 2;
  const long long extra = (long long)A.extra_doubles * 8;
  const long long sm_bytes = 228 * 1024, reserved = 1024;
  long long best_key = -1;
  for (int R = 8; R >= 1; R /= 2)
    for (int Cc = 8; Cc >= 1; Cc /= 2) {
      const long long per_warp = size_for(R, Cc);
      if (per_warp > warp_cap && !(R == 1 && Cc == 1)) continue;
      for (int staged = 1; staged >= 0; --staged) {
        if (staged && (!allow_staged || prog_bytes > 32 * 1024)) continue;
        const long long prog = staged ? (prog_bytes + 15) / 16 * 16 : 0;
        for (int w = 1; w <= max_wpc; ++w) {
          const long long cta = prog + extra + (long long)w * per_warp * 8;
          if (cta > kCoopMaxSmem) continue;
          const long long ctas = std::min<long long>(sm_bytes / (cta + reserved),
                                                     std::max(1, max_warps_regs / w));
          const long long warps = ctas * w;
          // most resident warps, then larger chunks, then staged programs, then fewer warps
          const long long key = ((warps * 128 + R * Cc) * 2 + staged) * 8 + (4 - w);
          if (warps > 0 && key > best_key) {
            best_key = key;
            A.R = R;
            A.Cc = Cc;
            A.smem_per_warp = (int)per_warp;
            A.prog_doubles = staged ? (int)(prog / 8) : 0;
            wpc = w;
            smem = (size_t)cta;
          }
        }
      }
    }
  if (best_key < 0)
    return set_error(GBX_ERR_UNSUPPORTED, "class (%d%d|%d%d) does not fit the shared memory",
                     M.la, M.lb, M.lc, M.ld);
  return GBX_OK;
}

inline int coop_grid(const EriLaunch& a, int wpc) {
  int dev = 0, nsm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  return (int)std::max<long long>(1, std::min<long long>((a.nwork + wpc - 1) / wpc, (long long)nsm * 8));
}

// Access to a class's programs, staged in shared memory or read from the global tables.
struct ProgView {
  const short (*ins)[8];
  const short* idx;
  int ins0, idx0;
  __device__ __forceinline__ const short* I(int i) const { return ins[i - ins0]; }
  __device__ __forceinline__ int X(int j) const { return idx[j - idx0]; }
};

__device__ __forceinline__ double pick3(int d, double x, double y, double z) {
  return d == 0 ? x : (d == 1 ? y : z);
}

__device__ __forceinline__ const double* sph_mat(int l) { return kCoopSph + (l == 2 ? 0 : 30); }

__device__ __forceinline__ int n_int(const ShellDev& s) {
  return (s.sph && s.l >= 2) ? 2 * s.l + 1 : ncart(s.l);
}

// Lane m <= L writes pref * F_m(T) to X[m]: T < 40 by the 8-term Taylor expansion of F_m
// around the nearest grid point (orders m..m+7 of the table), T >= 40 by F_0 = sqrt(pi/T)/2
// and m upward steps F_{k+1} = ((2k+1) F_k - e^{-T})/(2T).
__device__ __forceinline__ double boys_lane_value(int m, double T, const double* __restrict__ tab) {
  double f;
  T = fmax(T, 0.0);  // T >= 0 by construction; the table is never indexed below its start
  if (T < kBoysTMax) {
    const int n = __double2int_rn(T * 10.0);
    const double x = fma(-T, 10.0, (double)n) * 0.1;
    const double* g = tab + n * (kBoysOrders + 1) + m;
    f = g[7] * (1.0 / 5040);
    f = fma(f, x, g[6] * (1.0 / 720));
    f = fma(f, x, g[5] * (1.0 / 120));
    f = fma(f, x, g[4] * (1.0 / 24));
    f = fma(f, x, g[3] * (1.0 / 6));
    f = fma(f, x, g[2] * 0.5);
    f = fma(f, x, g[1]);
    f = fma(f, x, g[0]);
  } else {
    const double r = rsqrt(T);
    f = 0.88622692545275801365 * r;
    if (m > 0) {
      const double emT = exp(-T), o2T = 0.5 * r * r;
      for (int k = 0; k < m; ++k) f = fma((double)(2 * k + 1), f, -emT) * o2T;
    }
  }
  return f;
}

// Lane m <= L writes pref * F_m(T) to X[m]; for the range-separated operators (potential 1:
// erf(omega r)/r, 2: erfc(omega r)/r; gbasis/integrals/boys_functions.py:145-223) the values
// s^{m+1/2} F_m(s T), s = omega^2 / (omega^2 + rho), or the Coulomb value minus those.
__device__ __forceinline__ void boys_lanes(int L, int lane, double T, double pref,
                                           const double* __restrict__ tab, double* X,
                                           int potential = 0, double omega = 0.0,
                                           double rho = 0.0) {
  if (lane > L) return;
  double f = boys_lane_value(lane, T, tab);
  if (potential) {
    const double w2 = omega * omega, sc = w2 / (w2 + rho);
    double s = sqrt(sc);
    for (int k = 0; k < lane; ++k) s *= sc;
    const double g = boys_lane_value(lane, sc * T, tab) * s;
    f = potential == 1 ? g : f - g;
  }
  X[lane] = f * pref;
}

// Threads that run one quartet's tail together: a warp (WarpGroup), or the NW warps of a CTA
// that holds one quartet (CtaGroup<NW>).  t: the thread's index in the group; kN: its size;
// sync(): the group's barrier.
struct WarpGroup {
  int t;
  static constexpr int kN = 32;
  __device__ __forceinline__ void sync() const { __syncwarp(); }
};
template <int NW>
struct CtaGroup {
  int t;
  static constexpr int kN = 32 * NW;
  __device__ __forceinline__ void sync() const { __syncthreads(); }
};

// Phases B-D of one quartet (bra pair pq.x, ket pair pq.y) from ACC = S[0 .. NE*NF), by the
// threads of group g.  A group larger than a warp runs modes 0 (store) and 2 (Coulomb) only.
template <class G>
__device__ __forceinline__ void coop_tail_g(const CoopArgs& A, const ProgView& pv, double* S,
                                            const int2 pq, const PairDev& P, const PairDev& Q,
                                            const G& g) {
  const EriLaunch& a = A.a;
  const CoopMeta& M = A.m;
  auto INS = [&](int i) -> const short* { return pv.I(i); };
  auto IDX = [&](int j) -> int { return pv.X(j); };
  const int NENF = M.NE * M.NF;
  const int NCA = ncart(M.la), NCB = ncart(M.lb), NCC = ncart(M.lc), NCDD = ncart(M.ld);
  const int NCD = NCC * NCDD, NAB = NCA * NCB;
  double* ACC = S;
  double* HF = S + NENF;
  double* KN = HF + M.NE * NCD;
  double* T1 = KN;
  double* BN = KN;
  double* OB = BN + A.Cc * M.nB;
  double* T2 = OB + A.Cc * NAB;
  double* VAB = T2 + A.Cc * NAB;  // Coulomb mode: sum_cd (ab|cd) D[c][d] per (a, b)
  double* DAB = VAB + NAB;        // Coulomb mode: D[a][b] of the bra block
    // ---------------------------------------------------------------- B
  // HF[e][cd] overlays X (dead); rows are processed R at a time in KN
  for (int r0 = 0; r0 < M.NE; r0 += A.R) {
    const int rr = min(A.R, M.NE - r0);
    for (int i = g.t; i < rr * M.NF; i += G::kN) {
      const int r = i / M.NF, f = i - r * M.NF;
      KN[r * M.nK + f] = ACC[(r0 + r) * M.NF + f];
    }
    g.sync();
    for (int l = 0; l < M.k_nlv; ++l) {
      const int b = kCoopLv[M.k_lv + l], e = kCoopLv[M.k_lv + l + 1], cnt = e - b;
      for (int i = g.t; i < rr * cnt; i += G::kN) {
        const int r = i / cnt;
        const short* I = INS(M.k_ins + b + (i - r * cnt));
        double* Kr = KN + r * M.nK;
        Kr[I[0]] = fma(pick3(I[5], Q.ABx, Q.ABy, Q.ABz), Kr[I[2]], Kr[I[1]]);
      }
      g.sync();
    }
    for (int i = g.t; i < rr * NCD; i += G::kN) {
      const int r = i / NCD, j = i - r * NCD;
      HF[(r0 + r) * NCD + j] = KN[r * M.nK + IDX(M.kfin + j)];
    }
    g.sync();
  }
  const ShellDev& sA = a.shells[P.shA];
  const ShellDev& sB = a.shells[P.shB];
  const ShellDev& sC = a.shells[Q.shA];
  const ShellDev& sD = a.shells[Q.shB];
  const bool schwarz = a.mode == 1;  // Cartesian block, max |(ab|ab)| with component norms
  const bool coulomb = a.mode == 2;  // accumulate J instead of storing the block
  const int nAi = schwarz ? NCA : n_int(sA), nBi = schwarz ? NCB : n_int(sB);
  const int nCi = schwarz ? NCC : n_int(sC), nDi = schwarz ? NCDD : n_int(sD);
  double mx = 0.0;
  if (coulomb) {
    for (int i = g.t; i < nAi * nBi; i += G::kN) {
      const int ua = i / nBi, ub = i - ua * nBi;
      VAB[i] = 0.0;
      DAB[i] = a.D[(sA.func_off + sA.pos[ua]) * a.nbf + sB.func_off + sB.pos[ub]] *
               sA.scl[ua] * sB.scl[ub];
    }
    g.sync();
  }
  // ---------------------------------------------------------------- C
  if (nCi != NCC || nDi != NCDD) {
    for (int e = 0; e < M.NE; ++e) {
      double* row = HF + e * NCD;
      // axis D: T1[c][ud]
      for (int i = g.t; i < NCC * nDi; i += G::kN) {
        const int c = i / nDi, ud = i - c * nDi;
        double v;
        if (nDi != NCDD) {
          const double* W = sph_mat(M.ld) + ud * NCDD;
          v = 0.0;
          for (int d = 0; d < NCDD; ++d) v = fma(W[d], row[c * NCDD + d], v);
        } else {
          v = row[c * NCDD + ud];
        }
        T1[i] = v;
      }
      g.sync();
      // axis C: row[uc * nDi + ud]
      for (int i = g.t; i < nCi * nDi; i += G::kN) {
        const int uc = i / nDi, ud = i - uc * nDi;
        double v;
        if (nCi != NCC) {
          const double* W = sph_mat(M.lc) + uc * NCC;
          v = 0.0;
          for (int c = 0; c < NCC; ++c) v = fma(W[c], T1[c * nDi + ud], v);
        } else {
          v = T1[uc * nDi + ud];
        }
        row[i] = v;
      }
      g.sync();
    }
  }
  // ---------------------------------------------------------------- D
  const int ncol = nCi * nDi;
  const long long nBo = sB.nout, nDo = sD.nout;
  long long bbase, bcols;
  block_dest(a, P, bbase, bcols);
  const bool tr = quartet_transposed(P, Q);  // values stored at [ket row][bra column]
  for (int c0 = 0; c0 < ncol; c0 += A.Cc) {
    const int cc = min(A.Cc, ncol - c0);
    for (int i = g.t; i < cc * M.NE; i += G::kN) {
      const int c = i / M.NE, e = i - c * M.NE;
      BN[c * M.nB + e] = HF[e * NCD + c0 + c];
    }
    g.sync();
    for (int l = 0; l < M.b_nlv; ++l) {
      const int b = kCoopLv[M.b_lv + l], e = kCoopLv[M.b_lv + l + 1], cnt = e - b;
      for (int i = g.t; i < cc * cnt; i += G::kN) {
        const int c = i / cnt;
        const short* I = INS(M.b_ins + b + (i - c * cnt));
        double* Bc = BN + c * M.nB;
        Bc[I[0]] = fma(pick3(I[5], P.ABx, P.ABy, P.ABz), Bc[I[2]], Bc[I[1]]);
      }
      g.sync();
    }
    for (int i = g.t; i < cc * NAB; i += G::kN) {
      const int c = i / NAB, j = i - c * NAB;
      OB[i] = BN[c * M.nB + IDX(M.bfin + j)];
    }
    g.sync();
    // axis B then A (per column), result in OB as [c][ua][ub] with row stride nBi
    if (nBi != NCB) {
      const double* W = sph_mat(M.lb);
      for (int i = g.t; i < cc * NCA * nBi; i += G::kN) {
        const int c = i / (NCA * nBi), rem = i - c * NCA * nBi, a_ = rem / nBi, ub = rem - a_ * nBi;
        double v = 0.0;
        for (int b = 0; b < NCB; ++b) v = fma(W[ub * NCB + b], OB[c * NAB + a_ * NCB + b], v);
        T2[c * NAB + a_ * nBi + ub] = v;
      }
    } else {
      for (int i = g.t; i < cc * NAB; i += G::kN) T2[i] = OB[i];
    }
    g.sync();
    if (nAi != NCA) {
      const double* W = sph_mat(M.la);
      for (int i = g.t; i < cc * nAi * nBi; i += G::kN) {
        const int c = i / (nAi * nBi), rem = i - c * nAi * nBi, ua = rem / nBi, ub = rem - ua * nBi;
        double v = 0.0;
        for (int a_ = 0; a_ < NCA; ++a_) v = fma(W[ua * NCA + a_], T2[c * NAB + a_ * nBi + ub], v);
        OB[c * NAB + ua * nBi + ub] = v;
      }
    } else {
      for (int i = g.t; i < cc * NAB; i += G::kN) OB[i] = T2[i];
    }
    g.sync();
    if (coulomb) {
      // J[a][b] partial sums over this chunk's columns; J[c][d] of each column
      const int nab = nAi * nBi;
      for (int i = g.t; i < nab; i += G::kN) {
        double s = VAB[i];
        for (int c = 0; c < cc; ++c) {
          const int col = c0 + c, uc = col / nDi, ud = col - uc * nDi;
          const double dcd = a.D[(sC.func_off + sC.pos[uc]) * a.nbf + sD.func_off + sD.pos[ud]] *
                             sC.scl[uc] * sD.scl[ud];
          s = fma(OB[c * NAB + i], dcd, s);
        }
        VAB[i] = s;
      }
      if (pq.x != pq.y) {
        for (int c = g.t; c < cc; c += G::kN) {
          const int col = c0 + c, uc = col / nDi, ud = col - uc * nDi;
          double s = 0.0;
          for (int i = 0; i < nab; ++i) s = fma(OB[c * NAB + i], DAB[i], s);
          s *= ((P.shA != P.shB) ? 2.0 : 1.0) * sC.scl[uc] * sD.scl[ud];
          const long long fc = sC.func_off + sC.pos[uc], fd = sD.func_off + sD.pos[ud];
          j_add(a, fc * a.nbf + fd, s);
          if (Q.shA != Q.shB) j_add(a, fd * a.nbf + fc, s);
        }
      }
      g.sync();
      continue;
    }
    for (int i = g.t; i < cc * nAi * nBi; i += G::kN) {
      const int c = i / (nAi * nBi), rem = i - c * nAi * nBi, ua = rem / nBi, ub = rem - ua * nBi;
      const int col = c0 + c, uc = col / nDi, ud = col - uc * nDi;
      if (schwarz) {
        mx = fmax(mx, fabs(OB[c * NAB + ua * nBi + ub]) * kCoopCn[M.la * 10 + ua] *
                          kCoopCn[M.lb * 10 + ub] * kCoopCn[M.lc * 10 + uc] *
                          kCoopCn[M.ld * 10 + ud]);
        continue;
      }
      const double v = OB[c * NAB + ua * nBi + ub] * sA.scl[ua] * sB.scl[ub] * sC.scl[uc] *
                       sD.scl[ud];
      const long long rab = (long long)P.fo + sA.pos[ua] * nBo + sB.pos[ub];
      const long long rcd = (long long)Q.fo + sC.pos[uc] * nDo + sD.pos[ud];
      out_store(a, bbase + (tr ? rcd * bcols + rab : rab * bcols + rcd), v);
    }
    g.sync();
  }
  if constexpr (G::kN == 32) {
    if (schwarz) {
      for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
      if (g.t == 0) a.qout[pq.x] = sqrt(mx);
    }
  }
  if (coulomb) {
    const double fk = (Q.shA != Q.shB) ? 2.0 : 1.0;
    for (int i = g.t; i < nAi * nBi; i += G::kN) {
      const int ua = i / nBi, ub = i - ua * nBi;
      const long long fa = sA.func_off + sA.pos[ua], fbn = sB.func_off + sB.pos[ub];
      const double s = VAB[i] * fk * sA.scl[ua] * sB.scl[ub];
      j_add(a, fa * a.nbf + fbn, s);
      if (P.shA != P.shB) j_add(a, fbn * a.nbf + fa, s);
    }
  }
  g.sync();
}

__device__ __forceinline__ void coop_tail(const CoopArgs& A, const ProgView& pv, double* S,
                                          const int2 pq, const PairDev& P, const PairDev& Q,
                                          const int lane) {
  coop_tail_g(A, pv, S, pq, P, Q, WarpGroup{lane});
}

}  // namespace gbx
