// Device pipeline of a full-tensor call:
//   K1 pair_precompute   — primitive-pair data (zeta, P, P-A, K_AB x coefficients) in HBM
//   K2 build_work        — Schwarz test + warp-ballot compaction into per-class-block
//                          work lists (bra pair, ket pair), enumerated in sorted pair order
//   K4/K5 eri_block_fp64 — class-templated quartet kernels (eri_kernels.cuh)
//   K6 expand_full       — the 8-fold symmetric N^4 tensor from the compact store,
//                          coalesced writes in chemist or physicist order
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "gbx_eri.h"
#include "gbx_common.cuh"
#include "pipeline_kernels.cuh"
#include "coop.cuh"
#include "runtime.h"

namespace gbx {

#define GBX_CUDA(call, what)              \
  do {                                    \
    int _s = cuda_status((call), (what)); \
    if (_s != GBX_OK) return _s;          \
  } while (0)

// ------------------------------------------------------------------- K1
// Reference: gbasis/integrals/_two_elec_int.py:306-322 (exponent sums, product centres,
// relative coordinates) and :335-348, :528-547 (prefactor and primitive normalisation).
//
// Primitive pairs whose Gaussian-product factor exp(-ab/zeta |AB|^2) is below e^{-69}
// (1e-30, kPrimPairCut) are left out: a normalised primitive pair's charge distribution is
// bounded by that factor times powers of the distances that stay far below 1e10 here, so every
// integral they would add is below 1e-20.  On a pair of tight primitives on different atoms the
// factor is e^{-500} and less.  The kept ones are stored first, in their original order, and the
// pair's primitive count on the device becomes theirs (at least one is kept).

__global__ void pair_precompute(PairDev* __restrict__ pairs, int npairs,
                                const ShellDev* __restrict__ shells,
                                const double* __restrict__ exps, const double* __restrict__ coefs,
                                PrimPair* __restrict__ prims) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npairs) return;
  const PairDev P = pairs[p];
  const ShellDev& A = shells[P.shA];
  const ShellDev& B = shells[P.shB];
  const double ab2 = P.ABx * P.ABx + P.ABy * P.ABy + P.ABz * P.ABz;
  const double kpi = 5.914967172795613;  // sqrt(2) pi^{5/4}
  // the primitive pair of smallest exponent argument is always kept (found with the same
  // expression as below, so the pair's list is never empty)
  const int keep0 = kept_primitive_pair(exps + A.prim_off, A.nprim, exps + B.prim_off, B.nprim, ab2);
  int kept = 0;
  for (int ia = 0; ia < A.nprim; ++ia) {
    const double a = exps[A.prim_off + ia];
    const double na = coefs[A.prim_off + ia] * pow(2.0 * a / 3.14159265358979323846, 0.75) *
                      pow(4.0 * a, 0.5 * A.l);
    for (int ib = 0; ib < B.nprim; ++ib) {
      const double b = exps[B.prim_off + ib];
      const double nb = coefs[B.prim_off + ib] * pow(2.0 * b / 3.14159265358979323846, 0.75) *
                        pow(4.0 * b, 0.5 * B.l);
      const double z = a + b, iz = 1.0 / z;
      const double x = prim_pair_arg(a, b, ab2);
      if (x > kPrimPairCut && ia * B.nprim + ib != keep0) continue;
      PrimPair r;
      r.zeta = z;
      r.izeta = iz;
      r.Px = (a * A.x + b * B.x) * iz;
      r.Py = (a * A.y + b * B.y) * iz;
      r.Pz = (a * A.z + b * B.z) * iz;
      r.Xx = r.Px - A.x;
      r.Xy = r.Py - A.y;
      r.Xz = r.Pz - A.z;
      r.C = kpi * na * nb * exp(-x) * iz;
      r.pad = 0.0;
      prims[P.prim_off + kept++] = r;
    }
  }
  pairs[p].nprim = kept;
}

// ------------------------------------------------------------------- K2
// Candidates [start, start + len) of one class block: Schwarz test, warp-ballot compaction
// into work[0..count) (the direct Coulomb path processes the quartet space in chunks).
__global__ void build_work_range(const BuildBlock B, long long start, long long len,
                                 const double* __restrict__ qs, double tau,
                                 int2* __restrict__ work, int* __restrict__ count) {
  const long long t = start + (long long)blockIdx.x * blockDim.x + threadIdx.x;
  bool pass = false;
  int p = 0, q = 0;
  if (t < start + len && t < B.ncand) {
    long long pl, ql;
    if (B.tri) {
      pl = (long long)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
      while (pl * (pl + 1) / 2 > t) --pl;
      while ((pl + 1) * (pl + 2) / 2 <= t) ++pl;
      ql = t - pl * (pl + 1) / 2;
    } else {
      pl = t / B.nk;
      ql = t - pl * B.nk;
    }
    p = B.pb0 + (int)pl;
    q = B.pk0 + (int)ql;
    pass = (tau <= 0.0) || (qs[p] * qs[q] >= tau);
  }
  const unsigned mask = __ballot_sync(0xffffffffu, pass);
  const int lane = threadIdx.x & 31;
  int base = 0;
  if (lane == 0 && mask) base = atomicAdd(count, __popc(mask));
  base = __shfl_sync(0xffffffffu, base, 0);
  if (pass) work[base + __popc(mask & ((1u << lane) - 1u))] = make_int2(p, q);
}

__global__ void build_work(const int2* __restrict__ cta_map, const BuildBlock* __restrict__ bb,
                           const double* __restrict__ qs, double tau, int2* __restrict__ work,
                           int* __restrict__ counts, const MixedParams mp,
                           const PairDev* __restrict__ pairs) {
  const int2 cm = cta_map[blockIdx.x];
  const BuildBlock B = bb[cm.x];
  const long long t = (long long)cm.y + threadIdx.x;
  bool pass = false, fp32 = false, zero = false;
  int p = 0, q = 0;
  if (t < B.ncand) {
    long long pl, ql;
    if (B.tri) {
      pl = (long long)((sqrt(8.0 * (double)t + 1.0) - 1.0) * 0.5);
      while (pl * (pl + 1) / 2 > t) --pl;
      while ((pl + 1) * (pl + 2) / 2 <= t) ++pl;
      ql = t - pl * (pl + 1) / 2;
    } else {
      pl = t / B.nk;
      ql = t - pl * B.nk;
    }
    p = B.pb0 + (int)pl;
    q = B.pk0 + (int)ql;
    pass = (tau <= 0.0) || (qs[p] * qs[q] >= tau);
    if (mp.counts32) {
      // mixed form: bound of the final values (Schwarz bound times the largest output scale
      // of each shell) decides skip (< skip), FP32 (< fp32) or FP64
      const double bnd = mp.qm[p] * mp.qm[q];
      if (bnd < mp.skip) {
        zero = pass && mp.zero_work != nullptr;  // listed for zero_quartets
        pass = false;
      }
      fp32 = pass && B.fp32_ok && (!mp.fp32_on || mp.fp32_on[B.blk]) && bnd < mp.fp32;
    }
  }
  // diagonal blocks: the better-conditioned pair is the bra (quartet_transposed)
  if (B.orient && pairs && pass && pairs[q].orient < pairs[p].orient) {
    const int t2 = p;
    p = q;
    q = t2;
  }
  const bool p64 = pass && !fp32;
  const unsigned mask = __ballot_sync(0xffffffffu, p64);
  const unsigned mask32 = __ballot_sync(0xffffffffu, fp32);
  const int lane = threadIdx.x & 31;
  int base = 0, base32 = 0;
  if (lane == 0 && mask) base = atomicAdd(&counts[B.blk], __popc(mask));
  if (lane == 0 && mask32) base32 = atomicAdd(&mp.counts32[B.blk], __popc(mask32));
  base = __shfl_sync(0xffffffffu, base, 0);
  base32 = __shfl_sync(0xffffffffu, base32, 0);
  const unsigned below = (1u << lane) - 1u;
  if (p64) {
    const long long i = base + __popc(mask & below);
    if (gbx_in_bounds(mp.fault, kSiteWorkList, i, B.ncand)) work[B.work_off + i] = make_int2(p, q);
  }
  if (fp32) {  // FP32 quartets fill the block's slots from the end
    const long long i = B.ncand - 1 - (base32 + __popc(mask32 & below));
    if (gbx_in_bounds(mp.fault, kSiteWorkList, i, B.ncand)) work[B.work_off + i] = make_int2(p, q);
  }
  if (mp.zero_work) {
    // left-out quartets in their listed orientation (bra pair p of the block's bra class)
    const unsigned maskz = __ballot_sync(0xffffffffu, zero);
    int basez = 0;
    if (lane == 0 && maskz) basez = atomicAdd(mp.zero_count, __popc(maskz));
    basez = __shfl_sync(0xffffffffu, basez, 0);
    const long long iz = (long long)basez + __popc(maskz & below);
    if (zero && iz < mp.zero_cap) mp.zero_work[iz] = make_int2(p, q);
    else if (zero) gbx_in_bounds(mp.fault, kSiteWorkList, iz, mp.zero_cap);  // recorded
  }
}

// Mixed form: zeros in the compact store for the left-out quartets of a call (those whose
// final-value bound is below the skip threshold), in place of clearing the whole store.  A
// warp per quartet clears its entries of the block matrix: rows P.fo .. P.fo + nout(A) nout(B)
// - 1 (the bra pair's functions) by the ket pair's columns, where a computed quartet of the
// same orientation would have stored them.
__global__ void zero_quartets(const int2* __restrict__ list, const int* __restrict__ count,
                              long long cap, const PairDev* __restrict__ pairs,
                              const ShellDev* __restrict__ shells,
                              const BlockDev* __restrict__ blocks, double* __restrict__ out,
                              long long out_len, unsigned long long* fault) {
  const long long n = min((long long)*count, cap);
  const int lane = threadIdx.x & 31;
  const long long nw = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < n; w += nw) {
    const int2 pq = list[w];
    const PairDev P = pairs[pq.x];
    const PairDev Q = pairs[pq.y];
    const BlockDev b = blocks[P.cls * kNumPairClasses + Q.cls];
    const int nr = shells[P.shA].nout * P.nB, nc = shells[Q.shA].nout * Q.nB;
    const long long first = b.base + (long long)P.fo * b.ncols + Q.fo;
    for (int i = lane; i < nr * nc; i += 32) {
      const int r = i / nc, c = i - r * nc;
      const long long at = first + (long long)r * b.ncols + c;
      if (gbx_in_bounds(fault, kSiteZeroFill, at, out_len)) out[at] = 0.0;
    }
  }
}

// ------------------------------------------------------------------- K6
__device__ __forceinline__ long long pair_row(const ExpandArgs& e, int s1, int c1, int s2, int c2,
                                              int4& info) {
  const int pe = e.pair_of[s1 * e.nsh + s2];
  info = e.pinfo[pe >> 1];
  return (long long)info.z + ((pe & 1) ? (long long)c2 * info.w + c1 : (long long)c1 * info.w + c2);
}

// Function-pair key: class (bits 56..63), index of the shell pair within its class
// (bits 32..55) and row of the ordered function pair in that class's block matrix
// (bits 0..31).  One key per ordered pair of basis functions, built on the host.
__device__ __forceinline__ int fk_cls(long long k) { return (int)(k >> 56); }
__device__ __forceinline__ int fk_loc(long long k) { return (int)((k >> 32) & 0xffffff); }
__device__ __forceinline__ long long fk_row(long long k) { return k & 0xffffffffLL; }

// Debug builds: the expansion's destination p within the launch's output range, and a
// compact-store read index within the store.
__device__ __forceinline__ bool dst_ok(const ExpandArgs& e, const double* p) {
  return gbx_in_bounds(e.fault, kSiteExpand, (long long)(p - e.out_lo), e.out_len);
}
__device__ __forceinline__ bool compact_ok(const ExpandArgs& e, long long i) {
  return gbx_in_bounds(e.fault, kSiteCompactRead, i, e.compact_len);
}

__global__ void __launch_bounds__(256) expand_full(const ExpandArgs e) {
  __shared__ long long s_base[kNumPairClasses * kNumPairClasses];
  __shared__ long long s_ncols[kNumPairClasses * kNumPairClasses];
  for (int i = threadIdx.x; i < kNumPairClasses * kNumPairClasses; i += blockDim.x) {
    s_base[i] = e.blocks[i].base;
    s_ncols[i] = e.blocks[i].ncols;
  }
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const int warp = (int)(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int nwarps = (int)(((long long)gridDim.x * blockDim.x) >> 5);
  const int n = (int)e.n;
  const bool phys = e.notation == GBX_PHYSICIST;
  // a warp takes whole planes out[i0, i1, :, :]; chemist rows are (a,b,c) = (i0,i1,i2),
  // physicist out[i,j,k,l] = (ik|jl) rows are (a,b,c) = (i0,i2,i1)
  for (int pl = warp; pl < n * n; pl += nwarps) {
    const int i0 = pl / n, i1 = pl - i0 * n;
    double* __restrict__ oplane = e.out + (long long)pl * n * n;
    long long kp = phys ? 0 : e.ftab[(long long)i0 * n + i1];
    const long long* __restrict__ qrow = e.ftab + (long long)(phys ? i1 : 0) * n;
    for (int i2 = 0; i2 < n; ++i2) {
      if (phys) kp = e.ftab[(long long)i0 * n + i2];
      else qrow = e.ftab + (long long)i2 * n;
      const unsigned hp = (unsigned)(kp >> 32);
      const int cp = (int)(hp >> 24), lp = (int)(hp & 0xffffffu);
      const unsigned rowp = (unsigned)kp;
      double* __restrict__ orow = oplane + (long long)i2 * n;
      for (int d = lane; d < n; d += 32) {
        const long long kq = __ldg(qrow + d);
        const unsigned hq = (unsigned)(kq >> 32);
        const int cq = (int)(hq >> 24), lq = (int)(hq & 0xffffffu);
        const unsigned rowq = (unsigned)kq;
        long long off;
        if (cp > cq || (cp == cq && lp >= lq)) {
          const int t = cp * kNumPairClasses + cq;
          off = s_base[t] + (long long)rowp * s_ncols[t] + rowq;
        } else {
          const int t = cq * kNumPairClasses + cp;
          off = s_base[t] + (long long)rowq * s_ncols[t] + rowp;
        }
        if (compact_ok(e, off) && dst_ok(e, orow + d)) orow[d] = __ldg(e.compact + off);
      }
    }
  }
}

// Row-staged expansion.  The unique integrals form a symmetric matrix M over pair functions
// (class-major numbering); the compact store holds its class blocks (X, Y), X >= Y, and in a
// diagonal block (X, X) the entries whose bra pair has the larger local index.  A CTA takes
// pair functions r = blockIdx.x, blockIdx.x + gridDim.x, ...: it gathers row r of M into
// shared memory (a contiguous row of each block (X, Y), a column of each block (Y, X)), then
// writes the one or two N^2 planes of the output that row r fills — out[x, y, :, :] (chemist)
// or out[x, :, y, :] (physicist) for the ordered function pairs (x, y) of r — with streaming
// stores, each element gathered from shared memory through gtab.  CTAs in flight hold
// consecutive rows, so the strided column reads of one block hit the same L2 sectors and the
// compact store crosses HBM about once; the output is written once.
// Row r of M (class X, row rho within the class, local pair index lr) into shared memory.
__device__ __forceinline__ void stage_row(const ExpandArgs& e, long long r, int lr,
                                          double* __restrict__ s_row) {
  const int tid = threadIdx.x, nt = blockDim.x;
  int X = 0;
  while (r >= e.pf_first[X + 1]) ++X;
  const long long rho = r - e.pf_first[X];
  for (int Y = 0; Y < kNumPairClasses; ++Y) {
    const long long y0 = e.pf_first[Y], ny = e.pf_first[Y + 1] - y0;
    if (ny == 0) continue;
    if (X != Y) {
      // a row of block (X, Y) (unit stride) or a column of block (Y, X) (stride = columns);
      // four loads in flight per thread
      const BlockDev b = X > Y ? e.blocks[X * kNumPairClasses + Y] : e.blocks[Y * kNumPairClasses + X];
      const long long s0 = b.base + (X > Y ? rho * b.ncols : rho);
      const double* __restrict__ src = e.compact + s0;
      const long long stride = X > Y ? 1 : b.ncols;
      for (long long j0 = tid; j0 < ny; j0 += 4LL * nt) {
        double v[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const long long j = j0 + (long long)k * nt;
          v[k] = (j < ny && compact_ok(e, s0 + j * stride)) ? __ldg(src + j * stride) : 0.0;
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const long long j = j0 + (long long)k * nt;
          if (j < ny) s_row[y0 + j] = v[k];
        }
      }
    } else {
      const BlockDev b = e.blocks[X * kNumPairClasses + X];
      const double* __restrict__ blk = e.compact + b.base;
      for (long long j = tid; j < ny; j += nt) {
        const int lj = __ldg(&e.rowinfo[y0 + j].w);
        const long long at = lj <= lr ? rho * b.ncols + j : j * b.ncols + rho;
        s_row[y0 + j] = compact_ok(e, b.base + at) ? __ldg(blk + at) : 0.0;
      }
    }
  }
}

// One N^2 plane from the staged row: dst[c*cs + d] = M[r, gtab[c, d]], cs = N (chemist plane
// out[x, y, :, :], contiguous) or N^2 (physicist out[x, :, y, :]); when `mir` is not null the
// same values also go to the mirror plane there (one table and row read for both stores).
//   chemist: thread t takes plane elements t, t + T, t + 2T, t + 3T per pass (T threads; table
//     loads in flight together, each store coalesced across the warp);
//   physicist: warp w takes the plane rows c = w, w + warps, ...; lane l the columns d = l + 32k,
//     four per pass, so no element index is divided by N.
template <bool PHYS>
__device__ __forceinline__ void write_plane(const ExpandArgs& e, const double* __restrict__ s_row,
                                            double* __restrict__ dst, double* __restrict__ mir) {
  const int* __restrict__ gtab = e.gtab;
  const int n = (int)e.n;
  if constexpr (!PHYS) {
    const unsigned nt = blockDim.x, n2 = (unsigned)n * (unsigned)n;
    for (unsigned t0 = threadIdx.x; t0 < n2; t0 += 4u * nt) {
      int g[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const unsigned t = t0 + k * nt;
        g[k] = t < n2 ? __ldg(gtab + t) : 0;
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const unsigned t = t0 + k * nt;
        if (t < n2) {
          const double v = s_row[g[k]];
          if (dst_ok(e, dst + t)) __stcs(dst + t, v);
          if (mir && dst_ok(e, mir + t)) __stcs(mir + t, v);
        }
      }
    }
  } else {
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const long long cs = (long long)n * n;
    for (int c = threadIdx.x >> 5; c < n; c += nw) {
      const int* __restrict__ grow = gtab + (long long)c * n;
      double* __restrict__ drow = dst + (long long)c * cs;
      double* __restrict__ mrow = mir ? mir + (long long)c * cs : nullptr;
      for (int d0 = lane; d0 < n; d0 += 128) {
        int g[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int d = d0 + 32 * k;
          g[k] = d < n ? __ldg(grow + d) : 0;
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          const int d = d0 + 32 * k;
          if (d < n) {
            const double v = s_row[g[k]];
            if (dst_ok(e, drow + d)) __stcs(drow + d, v);
            if (mrow && dst_ok(e, mrow + d)) __stcs(mrow + d, v);
          }
        }
      }
    }
  }
}

__device__ __forceinline__ double* plane_ptr(const ExpandArgs& e, double* base, long long x,
                                             long long y, bool phys) {
  const long long n = e.n, n2 = n * n;
  return phys ? base + x * n * n2 + y * n : base + (x * n + y) * n2;
}

// Plane (x, y) of a staged row and, when the row's pair has x != y, the mirror plane (y, x).
__device__ __forceinline__ void write_row_planes(const ExpandArgs& e, const double* s_row,
                                                 double* base, long long x, long long y,
                                                 bool mirror, bool phys) {
  if (phys)
    write_plane<true>(e, s_row, plane_ptr(e, base, x, y, true),
                      mirror ? plane_ptr(e, base, y, x, true) : nullptr);
  else
    write_plane<false>(e, s_row, plane_ptr(e, base, x, y, false),
                       mirror ? plane_ptr(e, base, y, x, false) : nullptr);
}

__global__ void __launch_bounds__(512) expand_rows(const ExpandArgs e) {
  extern __shared__ double s_row[];
  const bool phys = e.notation == GBX_PHYSICIST;
  for (long long r = blockIdx.x; r < e.npf; r += gridDim.x) {
    const int4 ri = __ldg(e.rowinfo + r);
    if (ri.x < 0) continue;  // no ordered pair maps here (cannot happen for a built basis)
    __syncthreads();  // the previous row's planes are written
    stage_row(e, r, ri.w, s_row);
    __syncthreads();
    write_row_planes(e, s_row, e.out, ri.x, ri.y, ri.z != 0, phys);
  }
}

// Element (p, q) of the compact matrix M of unique integrals (p, q pair functions; p of class X,
// rp its row within the class, lp its local pair index), read from global memory: the block
// (X, Y) with X > Y, or with X == Y and lp >= q's local pair index, holds it at row p, column q;
// otherwise it sits transposed in block (Y, X).
__device__ __forceinline__ double compact_at(const ExpandArgs& e, int X, long long rp, int lp,
                                             long long q) {
  int Y = 0;
  while (q >= e.pf_first[Y + 1]) ++Y;
  const long long rq = q - e.pf_first[Y];
  const int lq = __ldg(&e.rowinfo[q].w);
  if (X > Y || (X == Y && lp >= lq)) {
    const BlockDev bd = e.blocks[X * kNumPairClasses + Y];
    const long long at = bd.base + rp * bd.ncols + rq;
    return compact_ok(e, at) ? __ldg(e.compact + at) : 0.0;
  }
  const BlockDev bd = e.blocks[Y * kNumPairClasses + X];
  const long long at = bd.base + rq * bd.ncols + rp;
  return compact_ok(e, at) ? __ldg(e.compact + at) : 0.0;
}

// Coulomb and exchange matrices from the compact store.  Row r of M (the pair function of the
// ordered function pairs (x, y) and, when x != y, (y, x)) holds (xy|cd) for every (c, d)
// through gtab, so
//   J[x][y] = J[y][x] = sum_cd (xy|cd) D[c][d],
//   K[x][c] += sum_d (xy|cd) D[y][d],   K[y][c] += sum_d (xy|cd) D[x][d]  (x != y).
// Every ordered pair belongs to exactly one row: J is stored, K (cleared by the caller) summed
// with atomics, 2N per row.  Warp w takes the plane rows c = w, w + warps, ...; lanes take d.
// STAGED: the row is gathered into shared memory first (as expand_rows does); otherwise each
// element is read from the compact store (rows larger than shared memory).
template <bool STAGED>
__global__ void __launch_bounds__(512) jk_rows(const ExpandArgs e, const double* __restrict__ D,
                                               double* __restrict__ J, double* __restrict__ K) {
  extern __shared__ double s_row[];
  __shared__ double s_j[16];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  const int n = (int)e.n;
  for (long long r = blockIdx.x; r < e.npf; r += gridDim.x) {
    const int4 ri = __ldg(e.rowinfo + r);
    if (ri.x < 0) continue;
    int X = 0;
    while (r >= e.pf_first[X + 1]) ++X;
    const long long rp = r - e.pf_first[X];
    __syncthreads();  // the previous row's shared values are read
    if constexpr (STAGED) stage_row(e, r, ri.w, s_row);
    __syncthreads();
    const double* __restrict__ Dx = D + (long long)ri.x * n;
    const double* __restrict__ Dy = D + (long long)ri.y * n;
    double jp = 0.0;
    for (int c = warp; c < n; c += nw) {
      const int* __restrict__ grow = e.gtab + (long long)c * n;
      const double* __restrict__ Dc = D + (long long)c * n;
      double kx = 0.0, ky = 0.0;
      for (int d = lane; d < n; d += 32) {
        const int g = __ldg(grow + d);
        double v;
        if constexpr (STAGED) v = s_row[g];
        else v = compact_at(e, X, rp, ri.w, g);
        jp = fma(v, __ldg(Dc + d), jp);
        kx = fma(v, __ldg(Dy + d), kx);
        ky = fma(v, __ldg(Dx + d), ky);
      }
      for (int o = 16; o > 0; o >>= 1) {
        kx += __shfl_xor_sync(0xffffffffu, kx, o);
        ky += __shfl_xor_sync(0xffffffffu, ky, o);
      }
      if (lane == 0) {
        const long long n2 = (long long)n * n;
        const long long kx_at = (long long)ri.x * n + c, ky_at = (long long)ri.y * n + c;
        if (gbx_in_bounds(e.fault, kSiteJK, kx_at, n2)) atomicAdd(K + kx_at, kx);
        if (ri.z && gbx_in_bounds(e.fault, kSiteJK, ky_at, n2)) atomicAdd(K + ky_at, ky);
      }
    }
    for (int o = 16; o > 0; o >>= 1) jp += __shfl_xor_sync(0xffffffffu, jp, o);
    if (lane == 0) s_j[warp] = jp;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < nw; ++w) t += s_j[w];
      const long long n2 = (long long)n * n;
      const long long j0 = (long long)ri.x * n + ri.y, j1 = (long long)ri.y * n + ri.x;
      if (gbx_in_bounds(e.fault, kSiteJK, j0, n2)) J[j0] = t;
      if (ri.z && gbx_in_bounds(e.fault, kSiteJK, j1, n2)) J[j1] = t;
    }
  }
}

// (ab|cd) of n function quadruples (a, b, c, d) from the compact store (indices checked by
// the host to be below N).
__global__ void gather_unique(const ExpandArgs e, const long long* __restrict__ idx4, long long n,
                              double* __restrict__ out) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const long long a = idx4[4 * i], b = idx4[4 * i + 1], c = idx4[4 * i + 2], d = idx4[4 * i + 3];
  const long long p = e.gtab[a * e.n + b], q = e.gtab[c * e.n + d];
  int X = 0, Y = 0;
  while (p >= e.pf_first[X + 1]) ++X;
  while (q >= e.pf_first[Y + 1]) ++Y;
  const long long rp = p - e.pf_first[X], rq = q - e.pf_first[Y];
  const int lp = e.rowinfo[p].w, lq = e.rowinfo[q].w;
  long long off;
  if (X > Y || (X == Y && lp >= lq)) {
    const BlockDev bd = e.blocks[X * kNumPairClasses + Y];
    off = bd.base + rp * bd.ncols + rq;
  } else {
    const BlockDev bd = e.blocks[Y * kNumPairClasses + X];
    off = bd.base + rq * bd.ncols + rp;
  }
  out[i] = compact_ok(e, off) ? e.compact[off] : 0.0;
}

// Batch form of the row-staged expansion: molecule m's pair-function rows are the global rows
// [row_first[m], row_first[m + 1]); each molecule has its own descriptor (tables, compact
// store, output).
__global__ void __launch_bounds__(512) expand_rows_batch(const ExpandArgs* __restrict__ mols,
                                                         const long long* __restrict__ row_first,
                                                         int nmol) {
  extern __shared__ double s_row[];
  const long long total = row_first[nmol];
  for (long long g = blockIdx.x; g < total; g += gridDim.x) {
    int lo = 0, hi = nmol - 1;  // last molecule whose first row is <= g
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (__ldg(row_first + mid) <= g) lo = mid;
      else hi = mid - 1;
    }
    const ExpandArgs& e = mols[lo];
    const bool phys = e.notation == GBX_PHYSICIST;
    const long long r = g - row_first[lo];
    const int4 ri = __ldg(e.rowinfo + r);
    if (ri.x < 0) continue;
    __syncthreads();
    stage_row(e, r, ri.w, s_row);
    __syncthreads();
    write_row_planes(e, s_row, e.out, ri.x, ri.y, ri.z != 0, phys);
  }
}

// Slab form of the row-staged expansion: the planes of x in [x0, x1) only — the contiguous
// range out[x0 * N^3, x1 * N^3) — into dst (which holds that range), one plane per ordered
// pair (x, y).  Used to stream the tensor to host memory slab by slab.
__global__ void __launch_bounds__(512) expand_slab(const ExpandArgs e, long long x0, long long x1,
                                                   double* __restrict__ dst) {
  extern __shared__ double s_row[];
  const bool phys = e.notation == GBX_PHYSICIST;
  const long long n = e.n;
  const long long np = (x1 - x0) * n;
  for (long long q = blockIdx.x; q < np; q += gridDim.x) {
    const long long x = x0 + q / n, y = q % n;
    const long long r = __ldg(e.gtab + x * n + y);
    const int lr = __ldg(&e.rowinfo[r].w);
    __syncthreads();
    stage_row(e, r, lr, s_row);
    __syncthreads();
    if (phys) write_plane<true>(e, s_row, plane_ptr(e, dst, x - x0, y, true), nullptr);
    else write_plane<false>(e, s_row, plane_ptr(e, dst, x - x0, y, false), nullptr);
  }
}

// ------------------------------------------------------------------- host side
static int num_sms(int device) {
  int v = 0;
  cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device);
  return v > 0 ? v : 1;
}

int upload_basis(Basis& B) {
  NvtxRange range("gbx upload basis");
  const int n = (int)B.shells.size();
  const int np = (int)B.pairs.size();
  int s;
  if ((s = B.alloc((void**)&B.d_shells, n * sizeof(ShellDev), "cudaMalloc(shells)"))) return s;
  if ((s = B.alloc((void**)&B.d_pairs, np * sizeof(PairDev), "cudaMalloc(pairs)"))) return s;
  if ((s = B.alloc((void**)&B.d_prims, B.n_prim_pairs * sizeof(PrimPair), "cudaMalloc(prims)")))
    return s;
  if ((s = B.alloc((void**)&B.d_exps, B.h_exps.size() * sizeof(double), "cudaMalloc(exps)")))
    return s;
  if ((s = B.alloc((void**)&B.d_coefs, B.h_coefs.size() * sizeof(double), "cudaMalloc(coefs)")))
    return s;
  if ((s = B.alloc((void**)&B.d_pair_of, (size_t)n * n * sizeof(int), "cudaMalloc(pair_of)")))
    return s;
  GBX_CUDA(cudaMemcpy(B.d_shells, B.shells.data(), n * sizeof(ShellDev), cudaMemcpyHostToDevice),
           "upload shells");
  GBX_CUDA(cudaMemcpy(B.d_pairs, B.pairs.data(), np * sizeof(PairDev), cudaMemcpyHostToDevice),
           "upload pairs");
  GBX_CUDA(cudaMemcpy(B.d_exps, B.h_exps.data(), B.h_exps.size() * sizeof(double),
                      cudaMemcpyHostToDevice), "upload exps");
  GBX_CUDA(cudaMemcpy(B.d_coefs, B.h_coefs.data(), B.h_coefs.size() * sizeof(double),
                      cudaMemcpyHostToDevice), "upload coefs");
  GBX_CUDA(cudaMemcpy(B.d_pair_of, B.pair_of.data(), (size_t)n * n * sizeof(int),
                      cudaMemcpyHostToDevice), "upload pair_of");
  pair_precompute<<<(np + 127) / 128, 128>>>(B.d_pairs, np, B.d_shells, B.d_exps, B.d_coefs,
                                             B.d_prims);
  GBX_CUDA(cudaGetLastError(), "pair_precompute launch");

  // function tables
  std::vector<int> fsh(B.nbf), fcomp(B.nbf);
  for (int sh = 0; sh < n; ++sh)
    for (int c = 0; c < B.shells[sh].nout; ++c) {
      fsh[B.shells[sh].func_off + c] = sh;
      fcomp[B.shells[sh].func_off + c] = c;
    }
  if ((s = B.alloc((void**)&B.d_func_shell, B.nbf * sizeof(int), "cudaMalloc(fsh)"))) return s;
  if ((s = B.alloc((void**)&B.d_func_comp, B.nbf * sizeof(int), "cudaMalloc(fcomp)"))) return s;
  GBX_CUDA(cudaMemcpy(B.d_func_shell, fsh.data(), B.nbf * sizeof(int), cudaMemcpyHostToDevice),
           "upload fsh");
  GBX_CUDA(cudaMemcpy(B.d_func_comp, fcomp.data(), B.nbf * sizeof(int), cudaMemcpyHostToDevice),
           "upload fcomp");
  if ((s = B.alloc((void**)&B.d_blocks, B.block_table.size() * sizeof(BlockDev),
                   "cudaMalloc(blocks)")))
    return s;
  GBX_CUDA(cudaMemcpy(B.d_blocks, B.block_table.data(), B.block_table.size() * sizeof(BlockDev),
                      cudaMemcpyHostToDevice), "upload blocks");

  const int nblk = (int)B.blocks.size();
  if ((s = B.alloc((void**)&B.d_counts, (nblk + 4) * sizeof(int), "cudaMalloc(counts)"))) return s;
  if ((s = B.alloc((void**)&B.d_pinfo, np * sizeof(int4), "cudaMalloc(pinfo)"))) return s;
  std::vector<int4> pinfo(np);
  for (int p = 0; p < np; ++p)
    pinfo[p] = make_int4(B.pairs[p].cls, B.pairs[p].local, B.pairs[p].fo, B.pairs[p].nB);
  GBX_CUDA(cudaMemcpy(B.d_pinfo, pinfo.data(), np * sizeof(int4), cudaMemcpyHostToDevice),
           "upload pinfo");
  if ((s = B.alloc((void**)&B.d_ftab, B.h_ftab.size() * sizeof(long long), "cudaMalloc(ftab)")))
    return s;
  GBX_CUDA(cudaMemcpy(B.d_ftab, B.h_ftab.data(), B.h_ftab.size() * sizeof(long long),
                      cudaMemcpyHostToDevice), "upload ftab");
  if ((s = B.alloc((void**)&B.d_gtab, B.h_gtab.size() * sizeof(int), "cudaMalloc(gtab)")))
    return s;
  GBX_CUDA(cudaMemcpy(B.d_gtab, B.h_gtab.data(), B.h_gtab.size() * sizeof(int),
                      cudaMemcpyHostToDevice), "upload gtab");
  if ((s = B.alloc((void**)&B.d_rowinfo, B.h_rowinfo.size() * sizeof(int4),
                   "cudaMalloc(rowinfo)")))
    return s;
  GBX_CUDA(cudaMemcpy(B.d_rowinfo, B.h_rowinfo.data(), B.h_rowinfo.size() * sizeof(int4),
                      cudaMemcpyHostToDevice), "upload rowinfo");
  if ((s = B.alloc((void**)&B.d_q, np * sizeof(double), "cudaMalloc(q)"))) return s;
  if ((s = B.alloc((void**)&B.d_qscreen, np * sizeof(double), "cudaMalloc(qscreen)"))) return s;
  if ((s = boys_table(B.device, &B.d_boys))) return s;
#if GBX_DEBUG_BOUNDS
  if ((s = B.alloc((void**)&B.d_fault, sizeof(unsigned long long), "cudaMalloc(fault word)")))
    return s;
  GBX_CUDA(cudaMemset(B.d_fault, 0, sizeof(unsigned long long)), "clear fault word");
#endif
  GBX_CUDA(cudaDeviceSynchronize(), "basis upload");
  return GBX_OK;
}

// Light classes run the register kernel, which has the FP32 path of the mixed form; the
// cooperative kernel of the heavy classes computes every quartet in FP64.
static bool block_has_fp32(const HostBlock& h) {
  return coop_class(kPairClassL[h.cb][0], kPairClassL[h.cb][1], kPairClassL[h.ck][0],
                    kPairClassL[h.ck][1]) < 0;
}

// Work list and build map of a full-tensor call (every unique quartet), made on first use.
static int ensure_full_work(Basis& B) {
  if (B.d_work) return GBX_OK;
  int s;
  const int nblk = (int)B.blocks.size();
  if ((s = B.alloc((void**)&B.d_work, (size_t)B.n_quartets * sizeof(int2), "cudaMalloc(work)")))
    return s;
  std::vector<BuildBlock> bb(nblk);
  std::vector<int2> cmap;
  for (int k = 0; k < nblk; ++k) {
    const HostBlock& h = B.blocks[k];
    bb[k] = BuildBlock{(int)B.class_first[h.cb], (int)h.nb, (int)B.class_first[h.ck], (int)h.nk,
                       h.tri ? 1 : 0, k, h.dev.work_off, h.ncand, block_has_fp32(h) ? 1 : 0,
                       block_orients(h.cb, h.ck) ? 1 : 0};
    for (long long c0 = 0; c0 < h.ncand; c0 += 256) cmap.push_back(make_int2(k, (int)c0));
    if (h.ncand > (1LL << 31) - 256)
      return set_error(GBX_ERR_UNSUPPORTED, "class block with %lld quartets exceeds the limit",
                       h.ncand);
  }
  B.n_cta_build = (int)cmap.size();
  void* dbb = nullptr;
  if ((s = B.alloc(&dbb, nblk * sizeof(BuildBlock), "cudaMalloc(build blocks)"))) return s;
  if ((s = B.alloc((void**)&B.d_cta_map, cmap.size() * sizeof(int2), "cudaMalloc(cta map)")))
    return s;
  GBX_CUDA(cudaMemcpy(dbb, bb.data(), nblk * sizeof(BuildBlock), cudaMemcpyHostToDevice),
           "upload build blocks");
  GBX_CUDA(cudaMemcpy(B.d_cta_map, cmap.data(), cmap.size() * sizeof(int2), cudaMemcpyHostToDevice),
           "upload cta map");
  B.d_build_blocks = dbb;
  return GBX_OK;
}

bool static_work_order() {
  static const bool v = [] {
    const char* e = std::getenv("GBX_WORK_ORDER");
    return e && std::strcmp(e, "static") == 0;
  }();
  return v;
}

// n work counters for one call's class launches, zeroed on stream st; *t = nullptr when the
// static order is chosen.
static int ensure_tickets(Basis& B, long long n, cudaStream_t st, unsigned long long** t) {
  *t = nullptr;
  if (static_work_order() || n <= 0) return GBX_OK;
  if (B.tickets_cap < n) {
    if (B.d_tickets) B.release(B.d_tickets);
    B.d_tickets = nullptr;
    B.tickets_cap = 0;
    int s = B.alloc((void**)&B.d_tickets, (size_t)n * sizeof(unsigned long long),
                    "cudaMalloc(work counters)");
    if (s) return s;
    B.tickets_cap = n;
  }
  GBX_CUDA(cudaMemsetAsync(B.d_tickets, 0, (size_t)n * sizeof(unsigned long long), st),
           "clear work counters");
  *t = B.d_tickets;
  return GBX_OK;
}

static EriLaunch base_launch(Basis& B) {
  EriLaunch a;
  memset(&a, 0, sizeof(a));
  a.pairs = B.d_pairs;
  a.prims = B.d_prims;
  a.shells = B.d_shells;
  a.boys_tab = B.d_boys;
  a.out = B.d_compact;
  return a;
}

static int class_dims(int cls, int& la, int& lb) {
  la = kPairClassL[cls][0];
  lb = kPairClassL[cls][1];
  return 0;
}

int ensure_schwarz(Basis& B, cudaStream_t st) {
  if (B.schwarz_ready) return GBX_OK;
  NvtxRange range("gbx Schwarz bounds");
  const int np = (int)B.pairs.size();
  std::vector<int2> diag(np);
  for (int p = 0; p < np; ++p) diag[p] = make_int2(p, p);
  int2* d_diag = nullptr;
  GBX_CUDA(cudaMalloc(&d_diag, np * sizeof(int2)), "cudaMalloc(schwarz work)");
  GBX_CUDA(cudaMemcpyAsync(d_diag, diag.data(), np * sizeof(int2), cudaMemcpyHostToDevice, st),
           "upload schwarz work");
  const int nsm = num_sms(B.device);
  for (int c = 0; c < kNumPairClasses; ++c) {
    if (B.class_count[c] == 0) continue;
    int la, lb;
    class_dims(c, la, lb);
    EriLaunch a = base_launch(B);
    a.work = d_diag;
    a.work_off = B.class_first[c];
    a.nwork = B.class_count[c];
    a.mode = 1;
    a.qout = B.d_q;
    const int grid = (int)std::min<long long>((a.nwork + 127) / 128, (long long)nsm * 8);
    int s = launch_class(la, lb, la, lb, a, grid, st);
    if (s) {
      cudaFree(d_diag);
      return s;
    }
  }
  std::vector<double> q(np);
  cudaError_t e1 = cudaMemcpyAsync(q.data(), B.d_q, np * sizeof(double), cudaMemcpyDeviceToHost, st);
  cudaError_t e2 = cudaStreamSynchronize(st);
  cudaFree(d_diag);
  GBX_CUDA(e1, "download schwarz bounds");
  GBX_CUDA(e2, "schwarz bounds");
  // bound of the original (generalized) shell pair: max over its segmented pairs
  const int n = (int)B.shells.size();
  std::vector<int> grp = B.group;
  if ((int)grp.size() != n) {
    grp.resize(n);
    for (int i = 0; i < n; ++i) grp[i] = i;
  }
  int ng = 0;
  for (int g : grp) ng = std::max(ng, g + 1);
  std::vector<double> gmax((size_t)ng * ng, 0.0);
  for (int p = 0; p < np; ++p) {
    int ga = grp[B.pairs[p].shA], gb = grp[B.pairs[p].shB];
    if (ga > gb) std::swap(ga, gb);
    double& m = gmax[(size_t)ga * ng + gb];
    m = std::max(m, q[p]);
  }
  B.h_q.resize(np);
  for (int p = 0; p < np; ++p) {
    int ga = grp[B.pairs[p].shA], gb = grp[B.pairs[p].shB];
    if (ga > gb) std::swap(ga, gb);
    B.h_q[p] = gmax[(size_t)ga * ng + gb];
  }
  GBX_CUDA(cudaMemcpy(B.d_qscreen, B.h_q.data(), np * sizeof(double), cudaMemcpyHostToDevice),
           "upload screening bounds");
  B.schwarz_ready = true;
  return GBX_OK;
}

// Q_p = sqrt(max |(ab|ab)|) over the output function pairs (a, b) of pair p, from the diagonal
// entries of block (p, p) in the compact store.
__global__ void diagonal_bounds(const PairDev* __restrict__ pairs, int npairs,
                                const ShellDev* __restrict__ shells,
                                const BlockDev* __restrict__ blocks,
                                const double* __restrict__ compact, double* __restrict__ q) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npairs) return;
  const PairDev P = pairs[p];
  const BlockDev b = blocks[P.cls * kNumPairClasses + P.cls];
  const int nf = shells[P.shA].nout * P.nB;
  double mx = 0.0;
  for (int i = 0; i < nf; ++i) {
    const long long r = (long long)P.fo + i;
    mx = fmax(mx, fabs(compact[b.base + r * b.ncols + r]));
  }
  q[p] = sqrt(mx);
}

// diagonal_bounds for one molecule of a batch (its pairs, block table and compact store).
int launch_diagonal_bounds(const PairDev* pairs, int npairs, const ShellDev* shells,
                           const BlockDev* blocks, const double* compact, double* q,
                           cudaStream_t st) {
  if (npairs <= 0) return GBX_OK;
  diagonal_bounds<<<(npairs + 127) / 128, 128, 0, st>>>(pairs, npairs, shells, blocks, compact, q);
  return cuda_status(cudaGetLastError(), "diagonal_bounds launch");
}

// Bounds of the final values for the mixed form: every output integral satisfies
// |(ab|cd)| <= sqrt((ab|ab) (cd|cd)) <= Q_p Q_q (Cauchy-Schwarz for the output functions
// themselves: norm_cont, component norms and spherical transforms included).  The diagonal
// quartets (p, p) are computed by the class kernels in their store mode, each into its own
// nf x nf block of a temporary buffer (a copy of the pair records with the pair-function
// offset 0 and the per-molecule destination index set to the pair), so no compact store is
// needed: the direct Coulomb path uses these bounds on systems whose store would not fit.
__global__ void diagonal_block_bounds(const PairDev* __restrict__ pairs, int npairs,
                                      const ShellDev* __restrict__ shells,
                                      const long long* __restrict__ off,
                                      const double* __restrict__ blk, double* __restrict__ q) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npairs) return;
  const PairDev P = pairs[p];
  const int nf = shells[P.shA].nout * P.nB;
  double mx = 0.0;
  for (int i = 0; i < nf; ++i) mx = fmax(mx, fabs(blk[off[p] + (long long)i * nf + i]));
  q[p] = sqrt(mx);
}

static int ensure_mixed_bounds(Basis& B, cudaStream_t st) {
  if (B.mixed_ready) return GBX_OK;
  NvtxRange range("gbx mixed-form bounds");
  int s;
  const int np = (int)B.pairs.size();
  if (!B.d_qmixed && (s = B.alloc((void**)&B.d_qmixed, np * sizeof(double), "cudaMalloc(qmixed)")))
    return s;
  // the device's pair records: their primitive counts are those pair_precompute kept
  std::vector<PairDev> tp(np);
  GBX_CUDA(cudaMemcpy(tp.data(), B.d_pairs, np * sizeof(PairDev), cudaMemcpyDeviceToHost),
           "download pairs");
  std::vector<int2> diag(np);
  std::vector<long long> off(np + 1, 0), ncols(np);
  for (int p = 0; p < np; ++p) {
    const long long nf = (long long)B.shells[tp[p].shA].nout * tp[p].nB;
    tp[p].fo = 0;
    tp[p].mol = p;
    diag[p] = make_int2(p, p);
    ncols[p] = nf;
    off[p + 1] = off[p] + nf * nf;
  }
  const size_t bytes = np * (sizeof(PairDev) + sizeof(int2) + 2 * sizeof(long long)) +
                       (size_t)off[np] * sizeof(double);
  unsigned char* tmp = nullptr;
  GBX_CUDA(cudaMalloc(&tmp, bytes), "cudaMalloc(diagonal quartets)");
  PairDev* d_tp = reinterpret_cast<PairDev*>(tmp);
  int2* d_diag = reinterpret_cast<int2*>(d_tp + np);
  long long* d_off = reinterpret_cast<long long*>(d_diag + np);
  long long* d_ncols = d_off + np;
  double* d_blk = reinterpret_cast<double*>(d_ncols + np);
  cudaError_t e = cudaMemcpyAsync(d_tp, tp.data(), np * sizeof(PairDev), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_diag, diag.data(), np * sizeof(int2), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_off, off.data(), np * sizeof(long long), cudaMemcpyHostToDevice, st);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(d_ncols, ncols.data(), np * sizeof(long long), cudaMemcpyHostToDevice, st);
  const int nsm = num_sms(B.device);
  s = GBX_OK;
  for (int c = 0; c < kNumPairClasses && e == cudaSuccess && !s; ++c) {
    if (B.class_count[c] == 0) continue;
    EriLaunch a = base_launch(B);
    a.pairs = d_tp;
    a.work = d_diag;
    a.work_off = B.class_first[c];
    a.nwork = B.class_count[c];
    a.out = d_blk;
    a.mol_base = d_off;
    a.mol_ncols = d_ncols;
    a.mode = 0;
    a.team = 1;
    const int grid = (int)std::min<long long>((a.nwork + 127) / 128, (long long)nsm * 8);
    s = launch_class(kPairClassL[c][0], kPairClassL[c][1], kPairClassL[c][0], kPairClassL[c][1],
                     a, std::max(grid, 1), st);
  }
  if (e == cudaSuccess && !s) {
    diagonal_block_bounds<<<(np + 127) / 128, 128, 0, st>>>(d_tp, np, B.d_shells, d_off, d_blk,
                                                            B.d_qmixed);
    e = cudaGetLastError();
  }
  const cudaError_t e2 = cudaStreamSynchronize(st);
  cudaFree(tmp);
  if (s) return s;
  GBX_CUDA(e, "mixed-form bounds");
  GBX_CUDA(e2, "mixed-form bounds");
  B.mixed_ready = true;
  return GBX_OK;
}

// The basis's auxiliary streams (kMaxAuxStreams, made on first use; calls use the first
// B.n_streams of them) with their join events and the fork event.
static int ensure_aux_streams(Basis& B) {
  if (!B.aux.empty()) return GBX_OK;
  B.aux.assign(kMaxAuxStreams, nullptr);
  B.join.assign(kMaxAuxStreams, nullptr);
  for (int j = 0; j < kMaxAuxStreams; ++j) {
    GBX_CUDA(cudaStreamCreateWithFlags(&B.aux[j], cudaStreamNonBlocking), "create stream");
    GBX_CUDA(cudaEventCreateWithFlags(&B.join[j], cudaEventDisableTiming), "create event");
  }
  GBX_CUDA(cudaEventCreateWithFlags(&B.fork, cudaEventDisableTiming), "create event");
  return GBX_OK;
}

namespace {
// number of entries of the descending array k[0..n) that are >= x
inline long long count_ge(const double* k, long long n, double x) {
  return std::upper_bound(k, k + n, x, [](double v, double e) { return v > e; }) - k;
}
}  // namespace

// Mixed form: per class block, upper bounds of its FP32 and left-out quartet counts, counted
// on the host from the final-value bounds ordered per class (a pair of pairs is below a
// threshold when the product of their bounds is; thresholds moved by 1e-9 relative in the
// direction that makes each count an upper bound of the device's classification).  Used to skip the FP32 launch of
// blocks without FP32 quartets, to size launch grids, and to clear the compact store only when
// quartets are left out.  Recomputed when the thresholds change.
static int ensure_mixed_counts(Basis& B, double skip, double fp32) {
  if (B.mix_key_skip == skip && B.mix_key_fp32 == fp32 && !B.mix_n32.empty()) return GBX_OK;
  const int np = (int)B.pairs.size();
  std::vector<double> q(np);
  GBX_CUDA(cudaMemcpy(q.data(), B.d_qmixed, np * sizeof(double), cudaMemcpyDeviceToHost),
           "download final-value bounds");
  std::vector<double> ks(np);
  for (int c = 0; c < kNumPairClasses; ++c) {
    const long long f = B.class_first[c], n = B.class_count[c];
    for (long long i = 0; i < n; ++i) ks[f + i] = q[f + i];
    std::sort(ks.begin() + f, ks.begin() + f + n, [](double x, double y) { return x > y; });
  }
  // pairs (i in bra class, j in ket class) with ks_i ks_j < t; for a triangular block the
  // unordered pairs, diagonal included
  auto below = [&](const HostBlock& h, double t) -> long long {
    if (t <= 0.0) return 0;
    const long long fb = B.class_first[h.cb], nb = B.class_count[h.cb];
    const long long fk = B.class_first[h.ck], nk = B.class_count[h.ck];
    long long ordered = 0, diag = 0;
    for (long long i = 0; i < nb; ++i) {
      const double v = ks[fb + i];
      const long long ge = v > 0.0 ? count_ge(ks.data() + fk, nk, t / v) : 0;
      ordered += nk - ge;
      if (h.tri && !(v * v >= t)) ++diag;
    }
    return h.tri ? (ordered + diag) / 2 : ordered;
  };
  const int nblk = (int)B.blocks.size();
  B.mix_n32.assign(nblk, 0);
  B.mix_nskip.assign(nblk, 0);
  std::vector<int> on(nblk, 0);
  for (int k = 0; k < nblk; ++k) {
    const HostBlock& h = B.blocks[k];
    B.mix_nskip[k] = below(h, skip * (1.0 + 1e-9));
    B.mix_n32[k] = block_has_fp32(h) ? std::max<long long>(
                                           0, below(h, fp32 * (1.0 + 1e-9)) - below(h, skip * (1.0 - 1e-9)))
                                      : 0;
    // an FP32 list pays for its own launch only when it holds a share of the block; the
    // quartets of a smaller one stay in the FP64 list
    on[k] = B.mix_n32[k] >= B.fp32_min && B.mix_n32[k] * B.fp32_share >= h.ncand;
    if (!on[k]) B.mix_n32[k] = 0;
  }
  if (!B.d_fp32_on && B.alloc((void**)&B.d_fp32_on, nblk * sizeof(int), "cudaMalloc(fp32 flags)"))
    return GBX_ERR_OOM;
  GBX_CUDA(cudaMemcpy(B.d_fp32_on, on.data(), nblk * sizeof(int), cudaMemcpyHostToDevice),
           "upload fp32 flags");
  B.mix_key_skip = skip;
  B.mix_key_fp32 = fp32;
  return GBX_OK;
}

int run_compact(Basis& B, double tau, cudaStream_t st, double skip, double fp32) {
  NvtxRange range("gbx work list and class kernels");
  int s;
  const bool mixed = skip > 0.0 || fp32 > 0.0;
  if (mixed && B.potential)
    return set_error(GBX_ERR_UNSUPPORTED, "the mixed-precision form computes 1/r integrals only");
  if (tau > 0.0 && (s = ensure_schwarz(B, st))) return s;
  if (mixed && (s = ensure_mixed_bounds(B, st))) return s;
  if (mixed && (s = ensure_mixed_counts(B, skip, fp32))) return s;
  if ((s = ensure_full_work(B))) return s;
  if ((s = B.ensure_scratch(B.compact_elems, 0))) return s;
  const int nblk = (int)B.blocks.size();
  if (mixed && !B.d_counts32) {
    if ((s = B.alloc((void**)&B.d_counts32, nblk * sizeof(int), "cudaMalloc(counts32)"))) return s;
  }
  B.counts_on_host = false;
  GBX_CUDA(cudaMemsetAsync(B.d_counts, 0, nblk * sizeof(int), st), "clear counts");
  if (mixed) GBX_CUDA(cudaMemsetAsync(B.d_counts32, 0, nblk * sizeof(int), st), "clear counts");
  long long left_out = 0;
  if (mixed)
    for (long long v : B.mix_nskip) left_out += v;
  // the mixed form's left-out quartets (at most left_out: the host counts bound the device's)
  // are listed by the work-list build and zeroed by zero_quartets, so that only their entries
  // of the store are written
  const bool zero_list = mixed && tau <= 0.0 && left_out > 0;
  if (zero_list) {
    if (B.zero_cap < left_out) {
      if (B.d_zero_work) B.release(B.d_zero_work);
      B.d_zero_work = nullptr;
      B.zero_cap = 0;
      if ((s = B.alloc((void**)&B.d_zero_work, (size_t)left_out * sizeof(int2),
                       "cudaMalloc(zero list)")))
        return s;
      B.zero_cap = left_out;
    }
    if (!B.d_zero_count &&
        (s = B.alloc((void**)&B.d_zero_count, sizeof(int), "cudaMalloc(zero count)")))
      return s;
    GBX_CUDA(cudaMemsetAsync(B.d_zero_count, 0, sizeof(int), st), "clear zero count");
  }
  if (tau > 0.0 || (left_out > 0 && !zero_list)) {
    // screened-out quartets are zero in the output: clear the store first
    GBX_CUDA(cudaMemsetAsync(B.d_compact, 0, B.compact_elems * sizeof(double), st),
             "clear compact store");
  }
  B.last_mixed = mixed;
  const MixedParams mp{B.d_qmixed, skip, fp32, mixed ? B.d_counts32 : nullptr,
                       mixed ? B.d_fp32_on : nullptr, zero_list ? B.d_zero_work : nullptr,
                       zero_list ? B.d_zero_count : nullptr, zero_list ? B.zero_cap : 0,
                       B.d_fault};
  if (B.profiling) cudaEventRecord(B.ev[0], st);
  build_work<<<B.n_cta_build, 256, 0, st>>>(B.d_cta_map, (const BuildBlock*)B.d_build_blocks,
                                            B.d_qscreen, tau, B.d_work, B.d_counts, mp,
                                            B.d_pairs);
  GBX_CUDA(cudaGetLastError(), "build_work launch");
  if (B.profiling) cudaEventRecord(B.ev[1], st);
  const int nsm = num_sms(B.device);
  // Class blocks are independent: spread them over the basis's auxiliary streams (largest
  // first) so that small and latency-bound classes overlap; per-block timing runs them in
  // order on the caller's stream instead.
  const bool per_block = B.profiling && B.profile_level >= 2;
  const int nstreams = per_block ? 0 : B.n_streams;
  unsigned long long* tickets = nullptr;  // [2 k]: block k's FP64 list, [2 k + 1]: its FP32 list
  if ((s = ensure_tickets(B, 2LL * nblk, st, &tickets))) return s;
  if (nstreams) {
    if ((s = ensure_aux_streams(B))) return s;
    GBX_CUDA(cudaEventRecord(B.fork, st), "fork");
    for (int j = 0; j < nstreams; ++j) GBX_CUDA(cudaStreamWaitEvent(B.aux[j], B.fork, 0), "fork wait");
  }
  if (zero_list) {
    // on the caller's stream, beside the class blocks (disjoint entries of the store)
    const int zgrid = (int)std::max<long long>(
        1, std::min<long long>((B.zero_cap + 7) / 8, (long long)nsm * 8));
    zero_quartets<<<zgrid, 256, 0, st>>>(B.d_zero_work, B.d_zero_count, B.zero_cap, B.d_pairs,
                                         B.d_shells, B.d_blocks, B.d_compact, B.compact_elems,
                                         B.d_fault);
    GBX_CUDA(cudaGetLastError(), "zero_quartets launch");
  }
  for (int i = 0; i < nblk; ++i) {
    const int k = B.launch_order.empty() ? i : B.launch_order[i];
    const cudaStream_t bs = nstreams ? B.aux[i % nstreams] : st;
    const HostBlock& h = B.blocks[k];
    int la, lb, lc, ld;
    class_dims(h.cb, la, lb);
    class_dims(h.ck, lc, ld);
    EriLaunch a = base_launch(B);
    a.work = B.d_work;
    a.work_count = B.d_counts + k;
    a.work_off = h.dev.work_off;
    a.nwork = h.ncand;
    a.base = h.dev.base;
    a.ncols = h.dev.ncols;
    a.mode = 0;
    a.fault = B.d_fault;
    a.out_len = B.compact_elems;
    a.team = h.team;
    a.variant = h.variant;
    a.potential = B.potential;
    a.omega = B.omega;
    a.ticket = tickets ? tickets + 2 * k : nullptr;
    // launch grids from the quartets each list can hold (FP64: all but those left out and
    // the FP32 ones; the kernels read the exact counts from the device)
    const long long n32 = mixed ? B.mix_n32[k] : 0;
    const long long n64 = mixed ? std::max<long long>(1, h.ncand - B.mix_nskip[k] - n32 + 1) : h.ncand;
    const int grid = (int)std::max<long long>(
        1, std::min<long long>((n64 * h.team + 127) / 128, (long long)nsm * h.ctas_per_sm));
    if (per_block) cudaEventRecord(B.blk_ev[i], st);
    if ((s = launch_class(la, lb, lc, ld, a, grid, bs))) return s;
    if (n32 > 0) {  // the block's FP32 list, on the next stream (beside its FP64 list)
      a.work_count = B.d_counts32 + k;
      a.reverse = 1;
      a.fp32 = 1;
      a.ticket = tickets ? tickets + 2 * k + 1 : nullptr;
      const int grid32 = (int)std::max<long long>(
          1, std::min<long long>((n32 * h.team + 127) / 128, (long long)nsm * h.ctas_per_sm));
      const cudaStream_t bs32 = nstreams ? B.aux[(i + 1) % nstreams] : st;
      if ((s = launch_class(la, lb, lc, ld, a, grid32, bs32))) return s;
    }
  }
  if (per_block) cudaEventRecord(B.blk_ev[nblk], st);
  if (nstreams) {
    for (int j = 0; j < nstreams; ++j) {
      GBX_CUDA(cudaEventRecord(B.join[j], B.aux[j]), "join");
      GBX_CUDA(cudaStreamWaitEvent(st, B.join[j], 0), "join wait");
    }
  }
  return GBX_OK;
}

// Direct Coulomb matrix.  Within each pair class the pairs are ordered by their bound,
// largest first, so that for a bra pair the ket pairs that pass the screening form a prefix of
// its class's order (and, in the mixed form, the FP64 quartets a prefix of that prefix).  The
// host counts every row's quartets by binary search; the device expands row ranges of those
// counts into work lists chunk by chunk (expand_jwork) and the class kernels contract each
// chunk with D as it is produced (mode 2, atomics into J).  Work is proportional to the
// quartets that survive, not to the N_pair^2 candidates; class blocks run concurrently on the
// basis's auxiliary streams, each stream with its own work buffer.  No integral is stored.
__global__ void expand_jwork(const long long* __restrict__ row_start, int nrows,
                             const int* __restrict__ first_col, const int* __restrict__ perm_b,
                             const int* __restrict__ perm_k, long long w0, long long len,
                             int2* __restrict__ work, const PairDev* __restrict__ pairs, int tri) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= len) return;
  const long long w = w0 + t;
  int lo = 0, hi = nrows - 1;  // the last row whose start is <= w (it is not empty)
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (row_start[mid] <= w) lo = mid;
    else hi = mid - 1;
  }
  int p = perm_b[lo], q = perm_k[first_col[lo] + (int)(w - row_start[lo])];
  if (tri && pairs[q].orient < pairs[p].orient) {  // the better-conditioned pair as the bra
    const int t2 = p;
    p = q;
    q = t2;
  }
  work[t] = make_int2(p, q);
}

int run_coulomb(Basis& B, const double* D, double tau, double* J, cudaStream_t st, double skip,
                double fp32) {
  NvtxRange range("gbx direct Coulomb matrix");
  int s;
  const bool mixed = skip > 0.0 || fp32 > 0.0;
  if (mixed && B.potential)
    return set_error(GBX_ERR_UNSUPPORTED, "the mixed-precision form computes 1/r integrals only");
  if ((s = ensure_schwarz(B, st))) return s;
  const int np = (int)B.pairs.size();
  std::vector<double> key(np);
  if (mixed) {
    if ((s = ensure_mixed_bounds(B, st))) return s;
    GBX_CUDA(cudaMemcpy(key.data(), B.d_qmixed, np * sizeof(double), cudaMemcpyDeviceToHost),
             "download final-value bounds");
  } else {
    key = B.h_q;
  }
  // per class: pairs by descending bound
  std::vector<int> perm(np);
  std::vector<double> ks(np);
  for (int c = 0; c < kNumPairClasses; ++c) {
    const long long f = B.class_first[c], n = B.class_count[c];
    for (long long i = 0; i < n; ++i) perm[f + i] = (int)(f + i);
    std::stable_sort(perm.begin() + f, perm.begin() + f + n,
                     [&](int x, int y) { return key[x] > key[y]; });
    for (long long i = 0; i < n; ++i) ks[f + i] = key[perm[f + i]];
  }
  // per class block and precision: row starts and first ket positions
  struct JList {
    int blk, fp32;
    long long total;
    size_t row_off, col_off;  // into rows / cols
    int nrows;
  };
  std::vector<JList> lists;
  std::vector<long long> rows;
  std::vector<int> cols;
  long long computed = 0, candidates = 0;
  for (HostBlock& hb : B.blocks) hb.j_computed = 0;
  const double lo64 = mixed ? std::max(fp32, skip) : tau;  // FP64 when the bound is >= lo64
  const double lo = mixed ? skip : tau;                     // computed when the bound is >= lo
  for (int k = 0; k < (int)B.blocks.size(); ++k) {
    const HostBlock& h = B.blocks[k];
    candidates += h.ncand;
    const long long fb = B.class_first[h.cb], nb = B.class_count[h.cb];
    const long long fk = B.class_first[h.ck], nk = B.class_count[h.ck];
    const bool has32 = mixed && block_has_fp32(h);
    for (int prec = 0; prec < (has32 ? 2 : 1); ++prec) {
      JList L{k, prec, 0, rows.size(), cols.size(), (int)nb};
      rows.push_back(0);
      for (long long i = 0; i < nb; ++i) {
        const double kb = ks[fb + i];
        auto upto = [&](double cut) -> long long {
          if (cut <= 0.0) return nk;
          if (!(kb > 0.0)) return 0;
          return count_ge(ks.data() + fk, nk, cut / kb);
        };
        long long n_all = upto(lo), n64 = has32 ? upto(lo64) : n_all;
        if (h.tri) {
          n_all = std::min(n_all, i + 1);
          n64 = std::min(n64, i + 1);
        }
        const long long first = prec == 0 ? 0 : n64;
        const long long cnt = prec == 0 ? n64 : n_all - n64;
        cols.push_back((int)first);
        rows.push_back(rows.back() + std::max<long long>(cnt, 0));
      }
      L.total = rows.back();
      computed += L.total;
      B.blocks[k].j_computed += L.total;
      if (L.total > 0) lists.push_back(L);
    }
  }
  B.last_computed = computed;
  B.last_screened = candidates - computed;
  B.counts_on_host = true;
  GBX_CUDA(cudaMemsetAsync(J, 0, (size_t)B.nbf * B.nbf * sizeof(double), st), "clear J");
  if (lists.empty()) return GBX_OK;
  // device copies (one block, kept by the basis until the next call)
  const size_t bytes = np * sizeof(int) + rows.size() * sizeof(long long) + cols.size() * sizeof(int);
  if (B.jplan_bytes < bytes) {
    if (B.d_jplan) B.release(B.d_jplan);
    B.d_jplan = nullptr;
    if ((s = B.alloc(&B.d_jplan, bytes, "cudaMalloc(J plan)"))) return s;
    B.jplan_bytes = bytes;
  }
  long long* d_rows = reinterpret_cast<long long*>(B.d_jplan);
  int* d_perm = reinterpret_cast<int*>(d_rows + rows.size());
  int* d_cols = d_perm + np;
  GBX_CUDA(cudaMemcpyAsync(d_rows, rows.data(), rows.size() * sizeof(long long),
                           cudaMemcpyHostToDevice, st), "upload J rows");
  GBX_CUDA(cudaMemcpyAsync(d_perm, perm.data(), np * sizeof(int), cudaMemcpyHostToDevice, st),
           "upload J order");
  GBX_CUDA(cudaMemcpyAsync(d_cols, cols.data(), cols.size() * sizeof(int), cudaMemcpyHostToDevice,
                           st), "upload J columns");
  // the host vectors are pageable: the copies above have completed on return
  const int nstreams = B.n_streams;
  if ((s = ensure_aux_streams(B))) return s;
  long long biggest = 0;
  for (const JList& L : lists) biggest = std::max(biggest, L.total);
  const long long chunk = std::min<long long>(kCoulombChunk, biggest);
  if (!B.d_jwork || B.jwork_cap < chunk * nstreams) {
    if (B.d_jwork) B.release(B.d_jwork);
    B.d_jwork = nullptr;
    if ((s = B.alloc((void**)&B.d_jwork, (size_t)chunk * nstreams * sizeof(int2), "cudaMalloc(J work)")))
      return s;
    B.jwork_cap = chunk * nstreams;
  }
  const int nsm = num_sms(B.device);
  // one work counter per chunk launch, in list order
  std::vector<long long> first_ticket(lists.size() + 1, 0);
  for (size_t li = 0; li < lists.size(); ++li)
    first_ticket[li + 1] = first_ticket[li] + (lists[li].total + chunk - 1) / chunk;
  unsigned long long* tickets = nullptr;
  if ((s = ensure_tickets(B, first_ticket.back(), st, &tickets))) return s;
  auto launch_list = [&](int li, cudaStream_t bs, int2* wk) -> int {
    const JList& L = lists[li];
    const HostBlock& h = B.blocks[L.blk];
    for (long long w0 = 0; w0 < L.total; w0 += chunk) {
      const long long len = std::min(chunk, L.total - w0);
      expand_jwork<<<(int)((len + 255) / 256), 256, 0, bs>>>(
          d_rows + L.row_off, L.nrows, d_cols + L.col_off, d_perm + B.class_first[h.cb],
          d_perm + B.class_first[h.ck], w0, len, wk, B.d_pairs,
          block_orients(h.cb, h.ck) ? 1 : 0);
      GBX_CUDA(cudaGetLastError(), "expand_jwork launch");
      EriLaunch a = base_launch(B);
      a.work = wk;
      a.work_count = nullptr;
      a.work_off = 0;
      a.nwork = len;
      a.mode = 2;
      a.fault = B.d_fault;
      a.team = h.team;
      a.variant = h.variant;
      a.fp32 = L.fp32;
      a.potential = B.potential;
      a.omega = B.omega;
      a.D = D;
      a.J = J;
      a.nbf = B.nbf;
      a.ticket = tickets ? tickets + first_ticket[li] + w0 / chunk : nullptr;
      const int grid = (int)std::max<long long>(
          1, std::min<long long>((len * h.team + 127) / 128, (long long)nsm * h.ctas_per_sm));
      int s2 = launch_class(kPairClassL[h.cb][0], kPairClassL[h.cb][1], kPairClassL[h.ck][0],
                            kPairClassL[h.ck][1], a, grid, bs);
      if (s2) return s2;
    }
    return GBX_OK;
  };
  const int nblk = (int)B.blocks.size();
  if (B.profiling && B.profile_level >= 2 && (int)B.blk_ev.size() == nblk + 1) {
    // per-block timing: the blocks one after another on the caller's stream, in launch order
    std::vector<std::vector<int>> of_block(nblk);
    for (size_t li = 0; li < lists.size(); ++li) of_block[lists[li].blk].push_back((int)li);
    for (int i = 0; i < nblk; ++i) {
      const int k = B.launch_order.empty() ? i : B.launch_order[i];
      cudaEventRecord(B.blk_ev[i], st);
      for (int li : of_block[k])
        if ((s = launch_list(li, st, B.d_jwork))) return s;
    }
    cudaEventRecord(B.blk_ev[nblk], st);
    return GBX_OK;
  }
  GBX_CUDA(cudaEventRecord(B.fork, st), "fork");
  for (int j = 0; j < nstreams; ++j) GBX_CUDA(cudaStreamWaitEvent(B.aux[j], B.fork, 0), "fork wait");
  // largest lists first, round robin over the streams
  std::vector<int> order(lists.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = (int)i;
  std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
    const HostBlock& hx = B.blocks[lists[x].blk];
    const HostBlock& hy = B.blocks[lists[y].blk];
    return lists[x].total * hx.avg_prims > lists[y].total * hy.avg_prims;
  });
  for (size_t oi = 0; oi < order.size(); ++oi) {
    const int j = (int)(oi % nstreams);
    if ((s = launch_list(order[oi], B.aux[j], B.d_jwork + (size_t)j * chunk))) return s;
  }
  for (int j = 0; j < nstreams; ++j) {
    GBX_CUDA(cudaEventRecord(B.join[j], B.aux[j]), "join");
    GBX_CUDA(cudaStreamWaitEvent(st, B.join[j], 0), "join wait");
  }
  return GBX_OK;
}

static ExpandArgs expand_args(const Basis& B, int notation, double* out) {
  ExpandArgs e;
  e.n = B.nbf;
  e.nsh = (int)B.shells.size();
  e.notation = notation;
  e.fsh = B.d_func_shell;
  e.fcomp = B.d_func_comp;
  e.pair_of = B.d_pair_of;
  e.pinfo = B.d_pinfo;
  e.blocks = B.d_blocks;
  e.compact = B.d_compact;
  e.out = out;
  e.ftab = B.d_ftab;
  e.gtab = B.d_gtab;
  e.rowinfo = B.d_rowinfo;
  e.npf = B.pf_first[kNumPairClasses];
  for (int c = 0; c <= kNumPairClasses; ++c) e.pf_first[c] = B.pf_first[c];
  e.fault = B.d_fault;
  e.out_lo = out;
  e.out_len = B.nbf * B.nbf * B.nbf * B.nbf;
  e.compact_len = B.compact_elems;
  return e;
}

// CTAs per SM of a row-staged expansion kernel with one M row in shared memory (0 when the
// row does not fit).
template <typename K>
static int row_kernel_fit(int device, K kernel, size_t row_bytes, int* per_sm) {
  *per_sm = 0;
  int optin = 0;
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
  if (row_bytes > (size_t)optin) return GBX_OK;
  if (row_bytes > 48 * 1024)
    GBX_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)row_bytes), "expansion smem attribute");
  GBX_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, kernel, 512, row_bytes),
           "expansion occupancy");
  return GBX_OK;
}

// Row-staged expansion of a batch of molecules (descriptors and row offsets on the device).
int launch_expand_batch(int device, const ExpandArgs* d_mols, const long long* d_row_first,
                        int nmol, long long total_rows, size_t max_row_bytes, cudaStream_t st) {
  int per_sm = 0, s;
  if ((s = row_kernel_fit(device, expand_rows_batch, max_row_bytes, &per_sm))) return s;
  if (per_sm == 0)
    return set_error(GBX_ERR_UNSUPPORTED, "a molecule's pair-function row (%zu bytes) exceeds "
                     "shared memory", max_row_bytes);
  const int grid = (int)std::max<long long>(
      1, std::min<long long>(total_rows, (long long)num_sms(device) * per_sm));
  expand_rows_batch<<<grid, 512, max_row_bytes, st>>>(d_mols, d_row_first, nmol);
  return cuda_status(cudaGetLastError(), "expand_rows_batch launch");
}

ExpandArgs make_expand_args(const Basis& B, int notation, double* out) {
  return expand_args(B, notation, out);
}

int num_sms_of(int device) { return num_sms(device); }

// Page-locked host staging ring of the pageable-output path, shared by the process (held
// under g_pin_mu for the whole call that uses it) and kept for later calls.
static std::mutex g_pin_mu;
static double* g_pin_ring = nullptr;
static size_t g_pin_elems = 0;

static int ensure_pinned_ring(size_t elems, double** ring) {
  if (g_pin_elems < elems) {
    if (g_pin_ring) cudaFreeHost(g_pin_ring);
    g_pin_ring = nullptr;
    g_pin_elems = 0;
    GBX_CUDA(cudaHostAlloc((void**)&g_pin_ring, elems * sizeof(double), cudaHostAllocPortable),
             "cudaHostAlloc(staging ring)");
    g_pin_elems = elems;
  }
  *ring = g_pin_ring;
  return GBX_OK;
}

// Full tensor into host memory without an N^4 device buffer: after the class kernels, the
// tensor is expanded slab by slab (x-ranges of out[x, ...], each a contiguous host range)
// into kStageBuffers device staging slabs; each slab is copied out on a copy stream while
// the next ones expand.  Host memory may be pageable or page-locked (page-locked copies run
// asynchronously and overlap fully).  Synchronous.
int run_full_host(Basis& B, int notation, double tau, double* out_host, cudaStream_t st) {
  NvtxRange range("gbx full tensor to host");
  const long long n = B.nbf;
  const size_t slab = (size_t)n * n * n;  // elements of one x
  const size_t row_bytes = (size_t)B.pf_first[kNumPairClasses] * sizeof(double);
  int per_sm = 0, s;
  if ((s = row_kernel_fit(B.device, expand_slab, row_bytes, &per_sm))) return s;
  if (per_sm == 0) {
    // a pair-function row larger than shared memory: whole tensor on the device, one copy
    if ((s = B.ensure_out((size_t)n * slab))) return s;
    if ((s = run_full(B, notation, tau, B.d_out, st))) return s;
    GBX_CUDA(cudaMemcpyAsync(out_host, B.d_out, (size_t)n * slab * sizeof(double),
                             cudaMemcpyDeviceToHost, st), "copy tensor to host");
    GBX_CUDA(cudaStreamSynchronize(st), "synchronize");
    return GBX_OK;
  }
  const long long xs = std::max<long long>(1, (long long)(kStageBytes / (slab * sizeof(double))));
  const size_t chunk = (size_t)std::min<long long>(xs, n) * slab;
  if (B.stage_elems < chunk) {
    if (B.d_stage) {
      B.release(B.d_stage);
      B.d_stage = nullptr;
      B.stage_elems = 0;
    }
    if ((s = B.alloc((void**)&B.d_stage, kStageBuffers * chunk * sizeof(double),
                     "cudaMalloc(staging slabs)")))
      return s;
    B.stage_elems = chunk;
  }
  if (!B.copy_stream) {
    GBX_CUDA(cudaStreamCreateWithFlags(&B.copy_stream, cudaStreamNonBlocking), "create stream");
    for (int k = 0; k < kStageBuffers; ++k) {
      GBX_CUDA(cudaEventCreateWithFlags(&B.stage_ready[k], cudaEventDisableTiming), "event");
      GBX_CUDA(cudaEventCreateWithFlags(&B.stage_free[k], cudaEventDisableTiming), "event");
    }
  }
  if ((s = run_compact(B, tau, st))) return s;
  const ExpandArgs e = expand_args(B, notation, nullptr);
  const int nsm = num_sms(B.device);
  const int nslab = (int)((n + xs - 1) / xs);
  // page-locked destination: slabs are copied straight into it; pageable: through a
  // page-locked staging ring, from which host threads copy each slab into place
  bool pinned = true;
  for (const double* p : {out_host, out_host + (size_t)n * slab - 1}) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess || at.type != cudaMemoryTypeHost)
      pinned = false;
  }
  cudaGetLastError();
  std::unique_lock<std::mutex> pin_lock;
  double* hring = nullptr;
  if (!pinned) {
    pin_lock = std::unique_lock<std::mutex>(g_pin_mu);
    if ((s = ensure_pinned_ring(kStageBuffers * chunk, &hring))) return s;
  }
  auto issue = [&](int i) -> int {
    const long long x0 = (long long)i * xs, x1 = std::min(n, x0 + xs);
    const int k = i % kStageBuffers;
    double* buf = B.d_stage + (size_t)k * B.stage_elems;
    if (i >= kStageBuffers) GBX_CUDA(cudaStreamWaitEvent(st, B.stage_free[k], 0), "wait slab");
    const long long planes = (x1 - x0) * n;
    const int grid = (int)std::max<long long>(1, std::min<long long>(planes, (long long)nsm * per_sm));
    ExpandArgs es = e;  // this launch's destination: the slab
    es.out_lo = buf;
    es.out_len = (x1 - x0) * slab;
    expand_slab<<<grid, 512, row_bytes, st>>>(es, x0, x1, buf);
    GBX_CUDA(cudaGetLastError(), "expand_slab launch");
    GBX_CUDA(cudaEventRecord(B.stage_ready[k], st), "record slab");
    GBX_CUDA(cudaStreamWaitEvent(B.copy_stream, B.stage_ready[k], 0), "wait slab");
    double* dst = pinned ? out_host + (size_t)x0 * slab : hring + (size_t)k * chunk;
    GBX_CUDA(cudaMemcpyAsync(dst, buf, (size_t)(x1 - x0) * slab * sizeof(double),
                             cudaMemcpyDeviceToHost, B.copy_stream),
             "copy slab to host");
    GBX_CUDA(cudaEventRecord(B.stage_free[k], B.copy_stream), "record slab copy");
    return GBX_OK;
  };
  if (pinned) {
    for (int i = 0; i < nslab; ++i)
      if ((s = issue(i))) return s;
  } else {
    // workers copy their share of each slab once its device-to-host copy has finished; slab
    // i + kStageBuffers reuses ring slot i % kStageBuffers only after every worker is done
    const int nthr = (int)std::max(1u, std::min(16u, std::thread::hardware_concurrency() / 2));
    std::atomic<int> issued{0}, failed{0};
    std::unique_ptr<std::atomic<int>[]> done(new std::atomic<int>[nslab]);
    for (int i = 0; i < nslab; ++i) done[i].store(0);
    auto worker = [&](int t) {
      for (int i = 0; i < nslab; ++i) {
        while (issued.load(std::memory_order_acquire) <= i) {
          if (failed.load()) return;
          std::this_thread::yield();
        }
        if (cudaEventSynchronize(B.stage_free[i % kStageBuffers]) != cudaSuccess) {
          failed.store(1);
        } else {
          const long long x0 = (long long)i * xs, x1 = std::min(n, x0 + xs);
          const size_t len = (size_t)(x1 - x0) * slab;
          const size_t a = len * t / nthr, b = len * (t + 1) / nthr;
          std::memcpy(out_host + (size_t)x0 * slab + a,
                      hring + (size_t)(i % kStageBuffers) * chunk + a, (b - a) * sizeof(double));
        }
        done[i].fetch_add(1, std::memory_order_release);
      }
    };
    std::vector<std::thread> pool;
    for (int t = 0; t < nthr; ++t) pool.emplace_back(worker, t);
    for (int i = 0; i < nslab && !s; ++i) {
      if (i >= kStageBuffers)
        while (done[i - kStageBuffers].load(std::memory_order_acquire) < nthr) {
          if (failed.load()) break;
          std::this_thread::yield();
        }
      if (failed.load()) break;
      s = issue(i);
      if (!s) issued.store(i + 1, std::memory_order_release);
    }
    if (s) failed.store(1);
    for (std::thread& th : pool) th.join();
    if (s) return s;
    if (failed.load()) return set_error(GBX_ERR_CUDA, "slab copy to host failed");
  }
  GBX_CUDA(cudaStreamSynchronize(B.copy_stream), "synchronize copies");
  GBX_CUDA(cudaStreamSynchronize(st), "synchronize");
  return GBX_OK;
}

int run_full(Basis& B, int notation, double tau, double* out, cudaStream_t st, double skip,
             double fp32) {
  int s = run_compact(B, tau, st, skip, fp32);
  if (s) return s;
  NvtxRange range("gbx expansion");
  const ExpandArgs e = expand_args(B, notation, out);
  if (B.profiling) cudaEventRecord(B.ev[2], st);
  const size_t row_bytes = (size_t)e.npf * sizeof(double);
  int per_sm = 0;
  if ((s = row_kernel_fit(B.device, expand_rows, row_bytes, &per_sm))) return s;
  if (per_sm > 0) {
    // one pair-function row of M in shared memory per CTA; persistent grid of the CTAs that
    // fit on the SMs together
    const int grid = (int)std::max<long long>(
        1, std::min<long long>(e.npf, (long long)num_sms(B.device) * per_sm));
    expand_rows<<<grid, 512, row_bytes, st>>>(e);
    GBX_CUDA(cudaGetLastError(), "expand_rows launch");
  } else {
    const long long rows = (long long)B.nbf * B.nbf * B.nbf;
    const int grid = (int)std::max<long long>(
        1, std::min<long long>((rows + 7) / 8, (long long)num_sms(B.device) * 16));
    expand_full<<<grid, 256, 0, st>>>(e);
    GBX_CUDA(cudaGetLastError(), "expand_full launch");
  }
  if (B.profiling) cudaEventRecord(B.ev[3], st);
  return GBX_OK;
}

// J and K of a density from the unique integrals (compact store; the N^4 tensor is never
// formed).  D, J, K: device N x N row-major.
int run_jk(Basis& B, const double* D, double tau, double* J, double* K, cudaStream_t st) {
  NvtxRange range("gbx J and K");
  int s = run_compact(B, tau, st, 0.0, 0.0);
  if (s) return s;
  const ExpandArgs e = expand_args(B, GBX_CHEMIST, nullptr);
  GBX_CUDA(cudaMemsetAsync(K, 0, (size_t)B.nbf * B.nbf * sizeof(double), st), "clear K");
  if (B.profiling) cudaEventRecord(B.ev[2], st);  // the contraction takes the expansion's slot
  const size_t row_bytes = (size_t)e.npf * sizeof(double);
  int per_sm = 0;
  if ((s = row_kernel_fit(B.device, jk_rows<true>, row_bytes, &per_sm))) return s;
  const int nsm = num_sms(B.device);
  if (per_sm > 0) {
    const int grid = (int)std::max<long long>(1, std::min<long long>(e.npf, (long long)nsm * per_sm));
    jk_rows<true><<<grid, 512, row_bytes, st>>>(e, D, J, K);
  } else {
    const int grid = (int)std::max<long long>(1, std::min<long long>(e.npf, (long long)nsm * 4));
    jk_rows<false><<<grid, 512, 0, st>>>(e, D, J, K);
  }
  if ((s = cuda_status(cudaGetLastError(), "jk_rows launch"))) return s;
  if (B.profiling) cudaEventRecord(B.ev[3], st);
  return GBX_OK;
}

int unique_values(Basis& B, long long n, const long long* idx4_host, double* out_host,
                  cudaStream_t st) {
  if (!B.d_compact) return set_error(GBX_ERR_INVALID, "no integrals computed on this basis yet");
  for (long long i = 0; i < 4 * n; ++i)
    if (idx4_host[i] < 0 || idx4_host[i] >= B.nbf)
      return set_error(GBX_ERR_INVALID, "function index %lld out of range [0, %lld)",
                       (long long)idx4_host[i], B.nbf);
  if (n == 0) return GBX_OK;
  long long* d_idx = nullptr;
  double* d_out = nullptr;
  GBX_CUDA(cudaMalloc(&d_idx, (size_t)n * 4 * sizeof(long long)), "cudaMalloc(indices)");
  cudaError_t err = cudaMalloc(&d_out, (size_t)n * sizeof(double));
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(d_idx, idx4_host, (size_t)n * 4 * sizeof(long long),
                          cudaMemcpyHostToDevice, st);
  if (err == cudaSuccess) {
    gather_unique<<<(int)((n + 255) / 256), 256, 0, st>>>(expand_args(B, GBX_CHEMIST, nullptr),
                                                        d_idx, n, d_out);
    err = cudaGetLastError();
  }
  if (err == cudaSuccess)
    err = cudaMemcpyAsync(out_host, d_out, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, st);
  if (err == cudaSuccess) err = cudaStreamSynchronize(st);
  cudaFree(d_idx);
  if (d_out) cudaFree(d_out);
  return cuda_status(err, "unique values");
}

}  // namespace gbx
