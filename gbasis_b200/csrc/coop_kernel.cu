// Cooperative ERI kernel: one warp per contracted shell quartet, for classes whose
// intermediates do not fit one thread's registers (high angular momentum).
//
// The warp interprets the class's generated programs (gen_coop.py) in shared memory:
//   A. per primitive quartet: Boys F_m(T) (lane 0), then the Obara-Saika VRR program
//        X[d] = PA_i X[s1] + WP_i X[s2] + k/(2 zeta) (X[s3] - rho/zeta X[s4])
//      and the electron-transfer program
//        X[d] = CE_i X[s1] - (zeta/eta) X[s2] + k1/(2 eta) X[s3] + k2/(2 eta) X[s4]
//      level by level (lanes over the instructions of a level), then ACC += X[targets];
//   B. ket HRR per row e:      K[d] = K[s1] + CD_i K[s2]   -> HF[e][cd]
//   C. ket Cartesian->spherical transform of HF rows (axis D, then C), in place;
//   D. per chunk of columns: bra HRR B[d] = B[s1] + AB_i B[s2] -> (ab), bra transform
//      (axis B, then A), permutation/scale to output functions, store.
// Same mathematics as the register kernel (eri_kernels.cuh) and as gbasis
// (gbasis/integrals/_two_elec_int.py:335-788, gbasis/base_four_symm.py:195-349).
#include <algorithm>
#include <cstring>

#include "coop.cuh"
#include "coop_programs.cuh"  // kCoopIns, kCoopLv, kCoopIdx, kCoopSph, kCoopCn, kCoopMeta
#include "errors.h"

namespace gbx {

struct CoopArgs {
  EriLaunch a;
  CoopMeta m;
  int R, Cc, smem_per_warp;  // rows / columns per HRR chunk, doubles of smem per warp
  int prog_doubles;          // shared memory taken by the staged programs (0: read globally)
};

__device__ __forceinline__ double pick3(int d, double x, double y, double z) {
  return d == 0 ? x : (d == 1 ? y : z);
}

__device__ __forceinline__ const double* sph_mat(int l) { return kCoopSph + (l == 2 ? 0 : 30); }

__device__ __forceinline__ int n_int(const ShellDev& s) {
  return (s.sph && s.l >= 2) ? 2 * s.l + 1 : ncart(s.l);
}

// F_0..F_L(T) into X[0..L] (scaled by pref); same method as boys_eval, runtime L.
__device__ void boys_to_smem(int L, double T, double pref, const double* __restrict__ tab,
                             double* X) {
  if (T < kBoysTMax) {
    const int n = __double2int_rn(T * 10.0);
    const double x = fma(-T, 10.0, (double)n) * 0.1;
    const double* g = tab + n * (kBoysOrders + 1) + L;
    constexpr double inv_fact[8] = {1.0, 1.0, 0.5, 1.0 / 6, 1.0 / 24, 1.0 / 120, 1.0 / 720,
                                    1.0 / 5040};
    double f = g[7] * inv_fact[7];
    for (int k = 6; k >= 0; --k) f = fma(f, x, g[k] * inv_fact[k]);
    double e = 1.0 / 5040.0;
    e = fma(e, x, 1.0 / 720.0);
    e = fma(e, x, 1.0 / 120.0);
    e = fma(e, x, 1.0 / 24.0);
    e = fma(e, x, 1.0 / 6.0);
    e = fma(e, x, 0.5);
    e = fma(e, x, 1.0);
    e = fma(e, x, 1.0);
    const double emT = tab[n * (kBoysOrders + 1) + kBoysOrders] * e;
    const double t2 = 2.0 * T;
    X[L] = f * pref;
    for (int m = L - 1; m >= 0; --m) {
      f = fma(t2, f, emT) / (2 * m + 1);
      X[m] = f * pref;
    }
  } else {
    const double r = rsqrt(T);
    double f = 0.88622692545275801365 * r;
    X[0] = f * pref;
    const double emT = exp(-T), o2T = 0.5 * r * r;
    for (int m = 0; m < L; ++m) {
      f = fma((double)(2 * m + 1), f, -emT) * o2T;
      X[m + 1] = f * pref;
    }
  }
}

// Lane m <= L writes pref * F_m(T) to X[m]: T < 40 by the 8-term Taylor expansion of F_m
// around the nearest grid point (orders m..m+7 of the table), T >= 40 by F_0 = sqrt(pi/T)/2
// and m upward steps F_{k+1} = ((2k+1) F_k - e^{-T})/(2T).
__device__ __forceinline__ void boys_lanes(int L, int lane, double T, double pref,
                                           const double* __restrict__ tab, double* X) {
  if (lane > L) return;
  double f;
  if (T < kBoysTMax) {
    const int n = __double2int_rn(T * 10.0);
    const double x = fma(-T, 10.0, (double)n) * 0.1;
    const double* g = tab + n * (kBoysOrders + 1) + lane;
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
    if (lane > 0) {
      const double emT = exp(-T), o2T = 0.5 * r * r;
      for (int m = 0; m < lane; ++m) f = fma((double)(2 * m + 1), f, -emT) * o2T;
    }
  }
  X[lane] = f * pref;
}

__global__ void eri_coop(const CoopArgs A) {
  extern __shared__ double smem[];
  const EriLaunch& a = A.a;
  const CoopMeta& M = A.m;
  const int lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  // the class's programs, staged once per CTA when they fit (A.prog_doubles > 0)
  short(*s_ins)[8] = reinterpret_cast<short(*)[8]>(smem);
  short* s_idx = reinterpret_cast<short*>(smem) + 8 * M.n_ins;
  const bool staged = A.prog_doubles > 0;
  if (staged) {
    const int4* src = reinterpret_cast<const int4*>(&kCoopIns[M.v_ins][0]);
    int4* dst4 = reinterpret_cast<int4*>(smem);
    for (int i = threadIdx.x; i < M.n_ins; i += blockDim.x) dst4[i] = src[i];
    for (int i = threadIdx.x; i < M.n_idx; i += blockDim.x) s_idx[i] = kCoopIdx[M.targets + i];
    __syncthreads();
  }
  auto INS = [&](int i) -> const short* {
    return staged ? s_ins[i - M.v_ins] : kCoopIns[i];
  };
  auto IDX = [&](int j) -> int { return staged ? s_idx[j - M.targets] : kCoopIdx[j]; };
  double* S = smem + A.prog_doubles + (size_t)wib * A.smem_per_warp;
  const int NENF = M.NE * M.NF;
  const int NCA = ncart(M.la), NCB = ncart(M.lb), NCC = ncart(M.lc), NCDD = ncart(M.ld);
  const int NCD = NCC * NCDD, NAB = NCA * NCB;
  double* ACC = S;
  double* X = S + NENF;
  double* HF = S + NENF;
  double* KN = HF + M.NE * NCD;
  double* T1 = KN;
  double* BN = KN;
  double* OB = BN + A.Cc * M.nB;
  double* T2 = OB + A.Cc * NAB;
  double* VAB = T2 + A.Cc * NAB;  // Coulomb mode: sum_cd (ab|cd) D[c][d] per (a, b)
  double* DAB = VAB + NAB;        // Coulomb mode: D[a][b] of the bra block

  const long long count = a.work_count ? (long long)(*a.work_count) : a.nwork;
  const long long nwarps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long w = (long long)blockIdx.x * (blockDim.x >> 5) + wib; w < count; w += nwarps) {
    const int2 pq = a.work[a.reverse ? a.work_off + a.nwork - 1 - w : a.work_off + w];
    const PairDev P = a.pairs[pq.x];
    const PairDev Q = a.pairs[pq.y];
    for (int i = lane; i < NENF; i += 32) ACC[i] = 0.0;
    // ---------------------------------------------------------------- A
    for (int ip = 0; ip < P.nprim; ++ip) {
      const PrimPair bp = a.prims[P.prim_off + ip];
      for (int jq = 0; jq < Q.nprim; ++jq) {
        const PrimPair kp = a.prims[Q.prim_off + jq];
        const double r = rsqrt(bp.zeta + kp.zeta);
        const double inv = r * r;
        const double PQx = bp.Px - kp.Px, PQy = bp.Py - kp.Py, PQz = bp.Pz - kp.Pz;
        const double rz = kp.zeta * inv;
        const double T = bp.zeta * rz * fma(PQx, PQx, fma(PQy, PQy, PQz * PQz));
        const double o2z = 0.5 * bp.izeta, ze = bp.zeta * kp.izeta, o2e = 0.5 * kp.izeta;
        const double WPx = -rz * PQx, WPy = -rz * PQy, WPz = -rz * PQz;
        const double CEx = fma(ze, bp.Xx, kp.Xx), CEy = fma(ze, bp.Xy, kp.Xy),
                     CEz = fma(ze, bp.Xz, kp.Xz);
        __syncwarp();
        boys_lanes(M.L, lane, T, bp.C * kp.C * r, a.boys_tab, X);
        __syncwarp();
        for (int l = 0; l < M.v_nlv; ++l) {
          const int b = kCoopLv[M.v_lv + l], e = kCoopLv[M.v_lv + l + 1];
          for (int i = b + lane; i < e; i += 32) {
            const short* I = INS(M.v_ins + i);
            const int dir = I[5];
            double v = fma(pick3(dir, bp.Xx, bp.Xy, bp.Xz), X[I[1]],
                           pick3(dir, WPx, WPy, WPz) * X[I[2]]);
            if (I[6]) v = fma(I[6] * o2z, fma(-rz, X[I[4]], X[I[3]]), v);
            X[I[0]] = v;
          }
          __syncwarp();
        }
        for (int l = 0; l < M.t_nlv; ++l) {
          const int b = kCoopLv[M.t_lv + l], e = kCoopLv[M.t_lv + l + 1];
          for (int i = b + lane; i < e; i += 32) {
            const short* I = INS(M.t_ins + i);
            const int dir = I[5];
            double v = fma(pick3(dir, CEx, CEy, CEz), X[I[1]], -ze * X[I[2]]);
            if (I[6]) v = fma(I[6] * o2e, X[I[3]], v);
            if (I[7]) v = fma(I[7] * o2e, X[I[4]], v);
            X[I[0]] = v;
          }
          __syncwarp();
        }
        for (int i = lane; i < NENF; i += 32) ACC[i] += X[IDX(M.targets + i)];
      }
    }
    __syncwarp();
    // ---------------------------------------------------------------- B
    // HF[e][cd] overlays X (dead); rows are processed R at a time in KN
    for (int r0 = 0; r0 < M.NE; r0 += A.R) {
      const int rr = min(A.R, M.NE - r0);
      for (int i = lane; i < rr * M.NF; i += 32) {
        const int r = i / M.NF, f = i - r * M.NF;
        KN[r * M.nK + f] = ACC[(r0 + r) * M.NF + f];
      }
      __syncwarp();
      for (int l = 0; l < M.k_nlv; ++l) {
        const int b = kCoopLv[M.k_lv + l], e = kCoopLv[M.k_lv + l + 1], cnt = e - b;
        for (int i = lane; i < rr * cnt; i += 32) {
          const int r = i / cnt;
          const short* I = INS(M.k_ins + b + (i - r * cnt));
          double* Kr = KN + r * M.nK;
          Kr[I[0]] = fma(pick3(I[5], Q.ABx, Q.ABy, Q.ABz), Kr[I[2]], Kr[I[1]]);
        }
        __syncwarp();
      }
      for (int i = lane; i < rr * NCD; i += 32) {
        const int r = i / NCD, j = i - r * NCD;
        HF[(r0 + r) * NCD + j] = KN[r * M.nK + IDX(M.kfin + j)];
      }
      __syncwarp();
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
      for (int i = lane; i < nAi * nBi; i += 32) {
        const int ua = i / nBi, ub = i - ua * nBi;
        VAB[i] = 0.0;
        DAB[i] = a.D[(sA.func_off + sA.pos[ua]) * a.nbf + sB.func_off + sB.pos[ub]] *
                 sA.scl[ua] * sB.scl[ub];
      }
      __syncwarp();
    }
    // ---------------------------------------------------------------- C
    if (nCi != NCC || nDi != NCDD) {
      for (int e = 0; e < M.NE; ++e) {
        double* row = HF + e * NCD;
        // axis D: T1[c][ud]
        for (int i = lane; i < NCC * nDi; i += 32) {
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
        __syncwarp();
        // axis C: row[uc * nDi + ud]
        for (int i = lane; i < nCi * nDi; i += 32) {
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
        __syncwarp();
      }
    }
    // ---------------------------------------------------------------- D
    const int ncol = nCi * nDi;
    const long long nBo = sB.nout, nDo = sD.nout;
    long long bbase, bcols;
    block_dest(a, P, bbase, bcols);
    double* __restrict__ dst = a.out + bbase + Q.fo;
    for (int c0 = 0; c0 < ncol; c0 += A.Cc) {
      const int cc = min(A.Cc, ncol - c0);
      for (int i = lane; i < cc * M.NE; i += 32) {
        const int c = i / M.NE, e = i - c * M.NE;
        BN[c * M.nB + e] = HF[e * NCD + c0 + c];
      }
      __syncwarp();
      for (int l = 0; l < M.b_nlv; ++l) {
        const int b = kCoopLv[M.b_lv + l], e = kCoopLv[M.b_lv + l + 1], cnt = e - b;
        for (int i = lane; i < cc * cnt; i += 32) {
          const int c = i / cnt;
          const short* I = INS(M.b_ins + b + (i - c * cnt));
          double* Bc = BN + c * M.nB;
          Bc[I[0]] = fma(pick3(I[5], P.ABx, P.ABy, P.ABz), Bc[I[2]], Bc[I[1]]);
        }
        __syncwarp();
      }
      for (int i = lane; i < cc * NAB; i += 32) {
        const int c = i / NAB, j = i - c * NAB;
        OB[i] = BN[c * M.nB + IDX(M.bfin + j)];
      }
      __syncwarp();
      // axis B then A (per column), result in OB as [c][ua][ub] with row stride nBi
      if (nBi != NCB) {
        const double* W = sph_mat(M.lb);
        for (int i = lane; i < cc * NCA * nBi; i += 32) {
          const int c = i / (NCA * nBi), rem = i - c * NCA * nBi, a_ = rem / nBi, ub = rem - a_ * nBi;
          double v = 0.0;
          for (int b = 0; b < NCB; ++b) v = fma(W[ub * NCB + b], OB[c * NAB + a_ * NCB + b], v);
          T2[c * NAB + a_ * nBi + ub] = v;
        }
      } else {
        for (int i = lane; i < cc * NAB; i += 32) T2[i] = OB[i];
      }
      __syncwarp();
      if (nAi != NCA) {
        const double* W = sph_mat(M.la);
        for (int i = lane; i < cc * nAi * nBi; i += 32) {
          const int c = i / (nAi * nBi), rem = i - c * nAi * nBi, ua = rem / nBi, ub = rem - ua * nBi;
          double v = 0.0;
          for (int a_ = 0; a_ < NCA; ++a_) v = fma(W[ua * NCA + a_], T2[c * NAB + a_ * nBi + ub], v);
          OB[c * NAB + ua * nBi + ub] = v;
        }
      } else {
        for (int i = lane; i < cc * NAB; i += 32) OB[i] = T2[i];
      }
      __syncwarp();
      if (coulomb) {
        // J[a][b] partial sums over this chunk's columns; J[c][d] of each column
        const int nab = nAi * nBi;
        for (int i = lane; i < nab; i += 32) {
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
          for (int c = lane; c < cc; c += 32) {
            const int col = c0 + c, uc = col / nDi, ud = col - uc * nDi;
            double s = 0.0;
            for (int i = 0; i < nab; ++i) s = fma(OB[c * NAB + i], DAB[i], s);
            s *= ((P.shA != P.shB) ? 2.0 : 1.0) * sC.scl[uc] * sD.scl[ud];
            const long long fc = sC.func_off + sC.pos[uc], fd = sD.func_off + sD.pos[ud];
            atomicAdd(a.J + fc * a.nbf + fd, s);
            if (Q.shA != Q.shB) atomicAdd(a.J + fd * a.nbf + fc, s);
          }
        }
        __syncwarp();
        continue;
      }
      for (int i = lane; i < cc * nAi * nBi; i += 32) {
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
        dst[((long long)P.fo + sA.pos[ua] * nBo + sB.pos[ub]) * bcols + sC.pos[uc] * nDo +
            sD.pos[ud]] = v;
      }
      __syncwarp();
    }
    if (schwarz) {
      for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
      if (lane == 0) a.qout[pq.x] = sqrt(mx);
    }
    if (coulomb) {
      const double fk = (Q.shA != Q.shB) ? 2.0 : 1.0;
      for (int i = lane; i < nAi * nBi; i += 32) {
        const int ua = i / nBi, ub = i - ua * nBi;
        const long long fa = sA.func_off + sA.pos[ua], fbn = sB.func_off + sB.pos[ub];
        const double s = VAB[i] * fk * sA.scl[ua] * sB.scl[ub];
        atomicAdd(a.J + fa * a.nbf + fbn, s);
        if (P.shA != P.shB) atomicAdd(a.J + fbn * a.nbf + fa, s);
      }
    }
    __syncwarp();
  }
}

int coop_class(int la, int lb, int lc, int ld) {
  for (int c = 0; c < kCoopNumClasses; ++c) {
    const CoopMeta& m = kCoopMeta[c];
    if (m.la == la && m.lb == lb && m.lc == lc && m.ld == ld) return c;
  }
  return -1;
}

int launch_coop(int prog, const EriLaunch& a, cudaStream_t st) {
  CoopArgs A;
  A.a = a;
  A.m = kCoopMeta[prog];
  const CoopMeta& M = A.m;
  const int NCD = ncart(M.lc) * ncart(M.ld), NAB = ncart(M.la) * ncart(M.lb);
  const int NENF = M.NE * M.NF;
  const long long budget = 48 * 1024 / 8;  // doubles per warp before reducing warps per CTA
  auto size_for = [&](int R, int Cc) {
    long long s = NENF + M.nX;
    s = std::max<long long>(s, NENF + (long long)M.NE * NCD + (long long)R * M.nK);
    s = std::max<long long>(s, NENF + (long long)M.NE * NCD + NCD);
    s = std::max<long long>(s, NENF + (long long)M.NE * NCD + (long long)Cc * (M.nB + 2 * NAB) +
                                   2 * NAB);
    return s;
  };
  int R = 8, Cc = 8;
  while ((R > 1 || Cc > 1) && size_for(R, Cc) > budget) {
    if (R > 1) R /= 2;
    if (Cc > 1) Cc /= 2;
  }
  A.R = R;
  A.Cc = Cc;
  const long long per_warp = size_for(R, Cc);
  A.smem_per_warp = (int)per_warp;
  const long long max_smem = 227 * 1024;
  const long long prog_bytes = (long long)M.n_ins * 16 + (long long)M.n_idx * 2;
  A.prog_doubles = 0;
  if (prog_bytes <= 32 * 1024 && prog_bytes + per_warp * 8 <= max_smem)
    A.prog_doubles = (int)((prog_bytes + 15) / 16 * 2);
  const long long avail = max_smem - (long long)A.prog_doubles * 8;
  int wpc = (int)std::max<long long>(1, std::min<long long>(4, avail / (per_warp * 8)));
  const size_t smem = (size_t)A.prog_doubles * 8 + (size_t)wpc * per_warp * 8;
  if ((long long)smem > max_smem)
    return set_error(GBX_ERR_UNSUPPORTED, "class (%d%d|%d%d) needs %zu bytes of shared memory",
                     M.la, M.lb, M.lc, M.ld, smem);
  int s = cuda_status(cudaFuncSetAttribute(eri_coop, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)max_smem), "eri_coop shared memory attribute");
  if (s) return s;
  int dev = 0, nsm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const long long nq = a.nwork;
  const int grid = (int)std::max<long long>(1, std::min<long long>((nq + wpc - 1) / wpc, (long long)nsm * 8));
  eri_coop<<<grid, 32 * wpc, smem, st>>>(A);
  return cuda_status(cudaGetLastError(), "eri_coop launch");
}

}  // namespace gbx
