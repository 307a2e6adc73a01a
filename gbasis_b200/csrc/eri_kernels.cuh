// Class-templated ERI kernels (FP64 form).
//
// One thread owns one contracted shell quartet (bra pair p, ket pair q) of a class block:
// it loops over the primitive quartets, evaluates F_m(T) from a shared-memory Taylor table,
// runs the generated VRR+ETR into register accumulators [e0|f0], then the generated HRR,
// the Cartesian->spherical transform (constant code) and the per-function permutation /
// scale, and stores the block into the compact store.
//
// Reference mathematics: gbasis/integrals/_two_elec_int.py:293-812 (prefactor, VRR, ETR,
// contraction, HRR, component norm) and gbasis/base_four_symm.py:195-349 (norm_cont,
// spherical transform).
#pragma once
#include <type_traits>
#include "gbx_common.cuh"
#include "eri_gen.cuh"

namespace gbx {

constexpr int kEriThreads = 128;

__device__ __forceinline__ constexpr double inv_odd(int m) { return 1.0 / (2 * m + 1); }

// Boys function F_0..F_L(T).  T < 40: Taylor expansion of F_L around the nearest grid point
// T_n = n/10 (8 terms, |T - T_n| <= 0.05, remainder < 1e-15 relative) from the staged table
// g[k][n] = F_{L+k}(T_n)/k!, e^{-T} = e^{-T_n} e^{T_n - T} by the same Taylor series, then
// the downward recursion F_m = (2T F_{m+1} + e^{-T})/(2m+1).  T >= 40: F_0 = sqrt(pi/T)/2
// (erfc(sqrt(40)) < 1e-18) and the upward recursion F_{m+1} = ((2m+1) F_m - e^{-T})/(2T).
// Reference: gbasis/integrals/boys_functions.py:26-63 (definition), :102-142 (recursion).
template <int L>
__device__ __forceinline__ void boys_eval(double T, const double* __restrict__ s_tab,
                                          const double* __restrict__ s_exp, double* F) {
  T = fmax(T, 0.0);  // T >= 0 by construction; the table is never indexed below its start
  if (T < kBoysTMax) {
    const int n = __double2int_rn(T * 10.0);
    const double x = fma(-T, 10.0, (double)n) * 0.1;  // T_n - T
    const double* g = s_tab + n;
    double f = g[(kBoysTaylor - 1) * kBoysNGrid];
#pragma unroll
    for (int k = kBoysTaylor - 2; k >= 0; --k) f = fma(f, x, g[k * kBoysNGrid]);
    F[L] = f;
    if (L > 0) {
      double e = 1.0 / 5040.0;
      e = fma(e, x, 1.0 / 720.0);
      e = fma(e, x, 1.0 / 120.0);
      e = fma(e, x, 1.0 / 24.0);
      e = fma(e, x, 1.0 / 6.0);
      e = fma(e, x, 0.5);
      e = fma(e, x, 1.0);
      e = fma(e, x, 1.0);
      const double emT = s_exp[n] * e;
      const double t2 = 2.0 * T;
#pragma unroll
      for (int m = L - 1; m >= 0; --m) F[m] = fma(t2, F[m + 1], emT) * inv_odd(m);
    }
  } else {
    const double r = rsqrt(T);
    F[0] = 0.88622692545275801365 * r;  // sqrt(pi)/2
    if (L > 0) {
      const double emT = exp(-T);
      const double o2T = 0.5 * r * r;
#pragma unroll
      for (int m = 0; m < L; ++m) F[m + 1] = fma((double)(2 * m + 1), F[m], -emT) * o2T;
    }
  }
}

// F[m] += c0 sc^m F_m(T) for m = 0..L: the Boys values of one argument folded into F as the
// recursion produces them (one value live at a time).
template <int L>
__device__ __forceinline__ void boys_accumulate(double T, const double* __restrict__ s_tab,
                                                const double* __restrict__ s_exp, double c0,
                                                double sc, double* F) {
  T = fmax(T, 0.0);
  if (T < kBoysTMax) {
    const int n = __double2int_rn(T * 10.0);
    const double x = fma(-T, 10.0, (double)n) * 0.1;
    const double* g = s_tab + n;
    double f = g[(kBoysTaylor - 1) * kBoysNGrid];
#pragma unroll
    for (int k = kBoysTaylor - 2; k >= 0; --k) f = fma(f, x, g[k * kBoysNGrid]);
    double c = c0;
#pragma unroll
    for (int m = 0; m < L; ++m) c *= sc;
    F[L] = fma(c, f, F[L]);
    if (L > 0) {
      double e = 1.0 / 5040.0;
      e = fma(e, x, 1.0 / 720.0);
      e = fma(e, x, 1.0 / 120.0);
      e = fma(e, x, 1.0 / 24.0);
      e = fma(e, x, 1.0 / 6.0);
      e = fma(e, x, 0.5);
      e = fma(e, x, 1.0);
      e = fma(e, x, 1.0);
      const double emT = s_exp[n] * e, t2 = 2.0 * T, isc = 1.0 / sc;
#pragma unroll
      for (int m = L - 1; m >= 0; --m) {
        f = fma(t2, f, emT) * inv_odd(m);
        c *= isc;
        F[m] = fma(c, f, F[m]);
      }
    }
  } else {
    const double r = rsqrt(T);
    double f = 0.88622692545275801365 * r, c = c0;
    F[0] = fma(c, f, F[0]);
    if (L > 0) {
      const double emT = exp(-T), o2T = 0.5 * r * r;
#pragma unroll
      for (int m = 0; m < L; ++m) {
        f = fma((double)(2 * m + 1), f, -emT) * o2T;
        c *= sc;
        F[m + 1] = fma(c, f, F[m + 1]);
      }
    }
  }
}

// Range-separated operators (gbasis/integrals/boys_functions.py:145-223): for erf(omega r)/r
// the Boys values become s^{m+1/2} F_m(s T), s = omega^2 / (omega^2 + rho); erfc(omega r)/r
// takes the Coulomb values minus those.  F holds F_m(T) on entry.
template <int L>
__device__ __forceinline__ void boys_attenuate(int potential, double omega, double rho, double T,
                                               const double* __restrict__ s_tab,
                                               const double* __restrict__ s_exp, double* F) {
  const double w2 = omega * omega, sc = w2 / (w2 + rho);
  if (potential == 1) {
#pragma unroll
    for (int m = 0; m <= L; ++m) F[m] = 0.0;
  }
  boys_accumulate<L>(sc * T, s_tab, s_exp, potential == 1 ? sqrt(sc) : -sqrt(sc), sc, F);
}

// In-place Cartesian->spherical transform of one axis of a [OUTER][ncart(L)][INNER] array.
template <int L, int OUTER, int INNER>
__device__ __forceinline__ void sph_axis(double* v) {
  if constexpr (L >= 2) {
#pragma unroll
    for (int o = 0; o < OUTER; ++o) {
#pragma unroll
      for (int i = 0; i < INNER; ++i) {
        double x[ncart(L)], y[2 * L + 1];
#pragma unroll
        for (int c = 0; c < ncart(L); ++c) x[c] = v[(o * ncart(L) + c) * INNER + i];
        gen::Sph<L>::apply(x, y);
#pragma unroll
        for (int u = 0; u < 2 * L + 1; ++u) v[(o * ncart(L) + u) * INNER + i] = y[u];
      }
    }
  }
}

__device__ __forceinline__ int internal_count(const ShellDev& s) {
  return (s.sph && s.l >= 2) ? 2 * s.l + 1 : ncart(s.l);
}

// Stage F_{L+k}(T_n)/k! (k < kBoysTaylor) and e^{-T_n} into shared memory, k-major: the
// lanes of a warp look up one k at a time at their own grid points n, and consecutive n sit in
// different banks (an n-major row of 8 doubles would put every n in one of two bank pairs).
template <int L>
__device__ __forceinline__ void stage_boys(const double* __restrict__ tab, double* s_tab,
                                           double* s_exp) {
  double inv_fact = 1.0;  // 1/k!
#pragma unroll
  for (int k = 0; k < kBoysTaylor; ++k) {
    if (k > 1) inv_fact /= k;
    for (int n = threadIdx.x; n < kBoysNGrid; n += blockDim.x)
      s_tab[k * kBoysNGrid + n] = tab[n * (kBoysOrders + 1) + L + k] * inv_fact;
  }
  for (int n = threadIdx.x; n < kBoysNGrid; n += blockDim.x)
    s_exp[n] = tab[n * (kBoysOrders + 1) + kBoysOrders];
}

// Coulomb-matrix epilogue of one unique quartet (bra pair shells A, B; ket C, D), block `v`
// in internal order [NA][NB][NC][ND] after the spherical transforms.  Every ordered shell
// quartet mapping to this unique one contributes:
//   J[a][b] += (1 + [C != D]) sum_cd (ab|cd) D[c][d]      (and J[b][a] when A != B)
//   J[c][d] += (1 + [A != B]) sum_ab (ab|cd) D[a][b]      (when bra pair != ket pair;
//                                                           and J[d][c] when C != D)
template <int NA, int NB, int NC, int ND>
__device__ __forceinline__ void coulomb_epilogue(const EriLaunch& a, int2 pq, const PairDev& P,
                                                 const PairDev& Q, const ShellDev& sA,
                                                 const ShellDev& sB, const ShellDev& sC,
                                                 const ShellDev& sD, int nAi, int nBi, int nCi,
                                                 int nDi, const double* v) {
  const long long n = a.nbf;
  const double fk = (Q.shA != Q.shB) ? 2.0 : 1.0;
  const double fb = (P.shA != P.shB) ? 2.0 : 1.0;
  const bool swap = pq.x != pq.y;
  double dcd[NC * ND];
  double w[NC * ND];
#pragma unroll
  for (int ic = 0; ic < NC; ++ic)
#pragma unroll
    for (int id = 0; id < ND; ++id) {
      w[ic * ND + id] = 0.0;
      dcd[ic * ND + id] = (ic < nCi && id < nDi)
                              ? a.D[(sC.func_off + sC.pos[ic]) * n + sD.func_off + sD.pos[id]] *
                                    sC.scl[ic] * sD.scl[id]
                              : 0.0;
    }
#pragma unroll
  for (int ia = 0; ia < NA; ++ia) {
    if (ia >= nAi) break;
#pragma unroll
    for (int ib = 0; ib < NB; ++ib) {
      if (ib >= nBi) break;
      const long long fa = sA.func_off + sA.pos[ia], fbn = sB.func_off + sB.pos[ib];
      const double sab = sA.scl[ia] * sB.scl[ib];
      const double dab = a.D[fa * n + fbn] * sab;
      double s = 0.0;
#pragma unroll
      for (int c = 0; c < NC * ND; ++c) {
        const double x = v[(ia * NB + ib) * NC * ND + c];
        s = fma(x, dcd[c], s);
        w[c] = fma(x, dab, w[c]);
      }
      s *= fk * sab;
      j_add(a, fa * n + fbn, s);
      if (P.shA != P.shB) j_add(a, fbn * n + fa, s);
    }
  }
  if (!swap) return;
#pragma unroll
  for (int ic = 0; ic < NC; ++ic) {
    if (ic >= nCi) break;
#pragma unroll
    for (int id = 0; id < ND; ++id) {
      if (id >= nDi) break;
      const long long fc = sC.func_off + sC.pos[ic], fd = sD.func_off + sD.pos[id];
      const double s = w[ic * ND + id] * fb * sC.scl[ic] * sD.scl[id];
      j_add(a, fc * n + fd, s);
      if (Q.shA != Q.shB) j_add(a, fd * n + fc, s);
    }
  }
}

// R = double: the FP64 form.  R = float: the mixed form's FP32 path — Boys values and the
// geometric factors are formed in FP64 and rounded, the vertical and transfer recursions run
// in FP32 and [e0|f0] accumulates in FP32 over the lane's primitive quartets; the team
// reduction, horizontal recursion, transforms and stores are FP64.
// Resident CTAs per SM a class's register kernel is compiled for.  Classes whose unconstrained
// register use is 171-200 per thread would fit 2 CTAs of 128 threads per SM; for these the cap
// of 168 registers that a third CTA needs costs at most a few spilled values, and the extra warps
// hide more of the primitive-loop latency (measured per class on medium8 and chain20: 8-13 %
// shorter blocks; classes further above the cap spill heavily and lose).
// (ss|ss) keeps the 64 registers that let 8 CTAs (the shared-memory limit) share an SM.
__host__ __device__ constexpr int eri_min_blocks(int la, int lb, int lc, int ld) {
  return (la + lb + lc + ld == 0) ? 8
         : ((la == 0 && lb == 2 && lc == 0 && ld == 1) ||
            (la == 1 && lb == 1 && lc == 0 && ld == 1) || (la == 1 && lb == 3 && lc == 0 && ld == 0))
             ? 3
             : 1;
}

// ATT: the instantiation for the range-separated operators (a.potential != 0); the 1/r kernels
// carry no attenuation code.
template <int LA, int LB, int LC, int LD, typename R, bool ATT = false>
__global__ void __launch_bounds__(kEriThreads, eri_min_blocks(LA, LB, LC, LD))
    eri_block(const EriLaunch a) {
  using C = gen::Cls<LA, LB, LC, LD>;
  constexpr int L = C::L;
  constexpr int NCA = ncart(LA), NCB = ncart(LB), NCC = ncart(LC), NCD = ncart(LD);
  __shared__ double s_tab[kBoysNGrid * kBoysTaylor];
  __shared__ double s_exp[kBoysNGrid];

  // A team of `team` consecutive lanes (1..32, power of two) shares one quartet: its lanes
  // take interleaved primitive quartets and the accumulators are summed with shuffles.  The
  // loop is warp-uniform (each warp takes 32/team quartets per step) so that the shuffles
  // always see the whole warp.
  const long long count = a.work_count ? (long long)(*a.work_count) : a.nwork;
  const int team = a.team > 0 ? a.team : 1;
  const int lane = threadIdx.x & 31;
  const int tl = lane & (team - 1);
  const int per_warp = 32 / team;
  // a CTA without a quartet (a screened or mixed-form list shorter than the grid) leaves
  // before staging the Boys table; the test is the same for all its threads
  if ((long long)blockIdx.x * (blockDim.x >> 5) * per_warp >= count) return;
  stage_boys<L>(a.boys_tab, s_tab, s_exp);
  __syncthreads();
  const long long gwarp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  // static order (a.ticket is not used: a step here is short, and one draw per warp and step
  // from a shared counter measured 4 % slower on the 120-function full tensor)
  for (long long wb = gwarp * per_warp; wb < count; wb += nwarps * per_warp) {
    const long long w = wb + lane / team;
    const bool valid = w < count;
    const int2 pq = valid ? a.work[a.reverse ? a.work_off + a.nwork - 1 - w : a.work_off + w]
                          : make_int2(0, 0);
    const PairDev P = a.pairs[pq.x];
    const PairDev Q = a.pairs[pq.y];
    R accr[C::NE * C::NF];  // FP32 form: accumulated in FP32 over the primitive quartets
#pragma unroll
    for (int i = 0; i < C::NE * C::NF; ++i) accr[i] = R(0);

    const int nprim = valid ? P.nprim * Q.nprim : 0;
    int ip = tl / Q.nprim, jq = tl - ip * Q.nprim;
    // one primitive quartet (bra primitive pair ipx, ket jqx) into accr
    auto prim_quartet = [&](int ipx, int jqx) {
      const PrimPair bp = a.prims[P.prim_off + ipx];
      const double o2z = 0.5 * bp.izeta;
      const PrimPair kp = a.prims[Q.prim_off + jqx];
      const double r = rsqrt(bp.zeta + kp.zeta);
      const double inv = r * r;
      const double PQx = bp.Px - kp.Px, PQy = bp.Py - kp.Py, PQz = bp.Pz - kp.Pz;
      const double rz = kp.zeta * inv;  // rho / zeta
      const double T = bp.zeta * rz * fma(PQx, PQx, fma(PQy, PQy, PQz * PQz));
      double F[L + 1];
      boys_eval<L>(T, s_tab, s_exp, F);
      if constexpr (ATT)
        boys_attenuate<L>(a.potential, a.omega, bp.zeta * rz, T, s_tab, s_exp, F);
      const double pref = bp.C * kp.C * r;
#pragma unroll
      for (int m = 0; m <= L; ++m) F[m] *= pref;
      const double ze = bp.zeta * kp.izeta;
      const double o2e = 0.5 * kp.izeta;
      if constexpr (sizeof(R) == sizeof(double)) {
        C::template prim<double>(F, bp.Xx, bp.Xy, bp.Xz, -rz * PQx, -rz * PQy, -rz * PQz, o2z,
                                 rz, fma(ze, bp.Xx, kp.Xx), fma(ze, bp.Xy, kp.Xy),
                                 fma(ze, bp.Xz, kp.Xz), ze, o2e, accr);
      } else {
        float F32[L + 1];
#pragma unroll
        for (int m = 0; m <= L; ++m) F32[m] = (float)F[m];
        C::template prim<float>(F32, (float)bp.Xx, (float)bp.Xy, (float)bp.Xz,
                                (float)(-rz * PQx), (float)(-rz * PQy), (float)(-rz * PQz),
                                (float)o2z, (float)rz, (float)fma(ze, bp.Xx, kp.Xx),
                                (float)fma(ze, bp.Xy, kp.Xy), (float)fma(ze, bp.Xz, kp.Xz),
                                (float)ze, (float)o2e, accr);
      }
    };
    auto advance = [&]() {
      jq += team;
      while (jq >= Q.nprim) {
        jq -= Q.nprim;
        ++ip;
      }
    };
    for (int idx = tl; idx < nprim; idx += team) {
      prim_quartet(ip, jq);
      advance();
    }
    double acc[C::NE * C::NF];
#pragma unroll
    for (int i = 0; i < C::NE * C::NF; ++i) acc[i] = (double)accr[i];
    for (int o = team >> 1; o > 0; o >>= 1) {
#pragma unroll
      for (int i = 0; i < C::NE * C::NF; ++i) acc[i] += __shfl_xor_sync(0xffffffffu, acc[i], o);
    }
    if (!valid || tl != 0) continue;

    double out[C::NAB * C::NCD];
    C::hrr(acc, P.ABx, P.ABy, P.ABz, Q.ABx, Q.ABy, Q.ABz, out);

    if (a.mode == 1) {
      // Schwarz diagonal quartet (p, p): max |(ab|ab)| with Cartesian component norms
      double mx = 0.0;
#pragma unroll
      for (int ia = 0; ia < NCA; ++ia)
#pragma unroll
        for (int ib = 0; ib < NCB; ++ib)
#pragma unroll
          for (int ic = 0; ic < NCC; ++ic)
#pragma unroll
            for (int id = 0; id < NCD; ++id)
              mx = fmax(mx, fabs(out[((ia * NCB + ib) * NCC + ic) * NCD + id]) *
                                (gen::cnorm<LA>(ia) * gen::cnorm<LB>(ib) * gen::cnorm<LC>(ic) *
                                 gen::cnorm<LD>(id)));
      a.qout[pq.x] = sqrt(mx);
      continue;
    }

    const ShellDev& sA = a.shells[P.shA];
    const ShellDev& sB = a.shells[P.shB];
    const ShellDev& sC = a.shells[Q.shA];
    const ShellDev& sD = a.shells[Q.shB];
    if (LD >= 2 && sD.sph) sph_axis<LD, NCA * NCB * NCC, 1>(out);
    if (LC >= 2 && sC.sph) sph_axis<LC, NCA * NCB, NCD>(out);
    if (LB >= 2 && sB.sph) sph_axis<LB, NCA, NCC * NCD>(out);
    if (LA >= 2 && sA.sph) sph_axis<LA, 1, NCB * NCC * NCD>(out);
    const int nAi = internal_count(sA), nBi = internal_count(sB);
    const int nCi = internal_count(sC), nDi = internal_count(sD);
    if (a.mode == 2) {
      coulomb_epilogue<NCA, NCB, NCC, NCD>(a, pq, P, Q, sA, sB, sC, sD, nAi, nBi, nCi, nDi, out);
      continue;
    }
    const long long nBo = sB.nout, nDo = sD.nout;
    long long bbase, bcols;
    block_dest(a, P, bbase, bcols);
    // element (ab|cd) at [bra pair function][ket pair function], or transposed
    // (quartet_transposed: a diagonal-block quartet run from its lower pair)
    auto store = [&](auto transposed) {
      constexpr bool TR = decltype(transposed)::value;
#pragma unroll
      for (int ia = 0; ia < NCA; ++ia) {
        if (ia >= nAi) break;
        const double fa = sA.scl[ia];
        const long long ra = (long long)P.fo + sA.pos[ia] * nBo;
#pragma unroll
        for (int ib = 0; ib < NCB; ++ib) {
          if (ib >= nBi) break;
          const double fab = fa * sB.scl[ib];
          const long long rab = ra + sB.pos[ib];
#pragma unroll
          for (int ic = 0; ic < NCC; ++ic) {
            if (ic >= nCi) break;
            const double fabc = fab * sC.scl[ic];
            const long long rc = (long long)Q.fo + sC.pos[ic] * nDo;
#pragma unroll
            for (int id = 0; id < NCD; ++id) {
              if (id >= nDi) break;
              const long long rcd = rc + sD.pos[id];
              out_store(a, bbase + (TR ? rcd * bcols + rab : rab * bcols + rcd),
                        out[((ia * NCB + ib) * NCC + ic) * NCD + id] * fabc * sD.scl[id]);
            }
          }
        }
      }
    };
    if (quartet_transposed(P, Q)) store(std::true_type{});
    else store(std::false_type{});
  }
}

}  // namespace gbx
