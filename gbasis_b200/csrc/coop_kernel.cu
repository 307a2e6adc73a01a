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
#include "coop_tail.cuh"
#include "errors.h"

namespace gbx {


// Phase A of one quartet: the contracted [e0|f0] over its primitive quartets into ACC (the
// first NE*NF doubles of the warp's buffer S).
__device__ __forceinline__ void coop_accumulate(const CoopArgs& A, const ProgView& pv, double* S,
                                                const PairDev& P, const PairDev& Q, int lane) {
  const EriLaunch& a = A.a;
  const CoopMeta& M = A.m;
  auto INS = [&](int i) -> const short* { return pv.I(i); };
  auto IDX = [&](int j) -> int { return pv.X(j); };
  const int NENF = M.NE * M.NF;
  double* ACC = S;
  double* X = S + NENF;
  for (int i = lane; i < NENF; i += 32) ACC[i] = 0.0;
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
      boys_lanes(M.L, lane, T, bp.C * kp.C * r, a.boys_tab, X, a.potential, a.omega,
                 bp.zeta * rz);
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
  const ProgView pv = staged ? ProgView{s_ins, s_idx, M.v_ins, M.targets}
                             : ProgView{kCoopIns, kCoopIdx, 0, 0};
  double* S = smem + A.prog_doubles + (size_t)wib * A.smem_per_warp;

  const long long count = a.work_count ? (long long)(*a.work_count) : a.nwork;
  const long long nwarps = (long long)gridDim.x * (blockDim.x >> 5);
  unsigned long long* const tk = a.ticket;  // one quartet per draw
  for (long long w = tk ? warp_ticket(tk, lane) : (long long)blockIdx.x * (blockDim.x >> 5) + wib;
       w < count; w = tk ? warp_ticket(tk, lane) : w + nwarps) {
    const int2 pq = a.work[a.reverse ? a.work_off + a.nwork - 1 - w : a.work_off + w];
    const PairDev P = a.pairs[pq.x];
    const PairDev Q = a.pairs[pq.y];
    coop_accumulate(A, pv, S, P, Q, lane);
    coop_tail(A, pv, S, pq, P, Q, lane);
  }
}

// Multi-class queue: a persistent grid whose warps draw quartets one at a time from a single
// counter over the queue of every segment (class block or batch block type, heaviest first),
// find the segment of the drawn position and run its class's programs (read from the global
// tables: the classes change from quartet to quartet) on the warp's shared buffer, sized for
// the largest class of the launch.
__global__ void eri_queue(const CoopArgs* __restrict__ args, const QueueSeg* __restrict__ segs,
                          int nseg, long long total, unsigned long long* cursor,
                          int smem_per_warp) {
  extern __shared__ double smem[];
  const int lane = threadIdx.x & 31;
  double* S = smem + (size_t)(threadIdx.x >> 5) * smem_per_warp;
  const ProgView pv{kCoopIns, kCoopIdx, 0, 0};
  for (long long t = warp_ticket(cursor, lane); t < total; t = warp_ticket(cursor, lane)) {
    int lo = 0, hi = nseg - 1;  // last segment whose first position is <= t
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (segs[mid].first <= t) lo = mid;
      else hi = mid - 1;
    }
    const CoopArgs& A = args[lo];
    const long long i = t - segs[lo].first;
    const int2 pq = A.a.work[A.a.work_off + i];
    const PairDev P = A.a.pairs[pq.x];
    const PairDev Q = A.a.pairs[pq.y];
    coop_accumulate(A, pv, S, P, Q, lane);
    coop_tail(A, pv, S, pq, P, Q, lane);
  }
}

int coop_class(int la, int lb, int lc, int ld) {
  for (int c = 0; c < kCoopNumHeavy; ++c) {
    const CoopMeta& m = kCoopMeta[c];
    if (m.la == la && m.lb == lb && m.lc == lc && m.ld == ld) return c;
  }
  return -1;
}

int launch_coop(int prog, const EriLaunch& a, cudaStream_t st) {
  CoopArgs A;
  A.a = a;
  A.m = kCoopMeta[prog];
  size_t smem = 0;
  int wpc = 1;
  int s = coop_plan(A.m, A.m.nX, A, smem, wpc);
  if (s) return s;
  s = cuda_status(cudaFuncSetAttribute(eri_coop, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)kCoopMaxSmem), "eri_coop shared memory attribute");
  if (s) return s;
  eri_coop<<<coop_grid(a, wpc), 32 * wpc, smem, st>>>(A);
  return cuda_status(cudaGetLastError(), "eri_coop launch");
}

int coop_program(int la, int lb, int lc, int ld) {
  for (int c = 0; c < kCoopNumClasses; ++c) {
    const CoopMeta& m = kCoopMeta[c];
    if (m.la == la && m.lb == lb && m.lc == lc && m.ld == ld) return c;
  }
  return -1;
}

int queue_plan(const EriLaunch* launches, const int* progs, const long long* counts, int nseg,
               std::vector<unsigned char>& args_blob, std::vector<QueueSeg>& segs,
               QueuePlan& plan) {
  std::vector<CoopArgs> args(nseg);
  segs.assign(nseg, QueueSeg{0, 0});
  plan = QueuePlan{};
  long long per_warp = 0;
  for (int k = 0; k < nseg; ++k) {
    if (progs[k] < 0 || progs[k] >= kCoopNumClasses)
      return set_error(GBX_ERR_UNSUPPORTED, "queue segment %d: no program for its class", k);
    CoopArgs& A = args[k];
    A.a = launches[k];
    A.a.ticket = nullptr;
    A.a.work_count = nullptr;
    A.a.reverse = 0;
    A.m = kCoopMeta[progs[k]];
    size_t sm = 0;
    int w = 1;
    // the tail's chunks of this class; programs are never staged (classes change per quartet)
    int s = coop_plan(A.m, A.m.nX, A, sm, w, 16, false);
    if (s) return s;
    per_warp = std::max<long long>(per_warp, A.smem_per_warp);
    segs[k] = QueueSeg{plan.total, counts[k]};
    plan.total += counts[k];
  }
  for (CoopArgs& A : args) {
    A.smem_per_warp = (int)per_warp;
    A.prog_doubles = 0;
  }
  plan.nseg = nseg;
  plan.smem_per_warp = (int)per_warp;
  plan.wpc = (int)std::max<long long>(1, std::min<long long>(4, kCoopMaxSmem / (per_warp * 8)));
  plan.smem = (size_t)plan.wpc * per_warp * 8;
  if (plan.smem > (size_t)kCoopMaxSmem)
    return set_error(GBX_ERR_UNSUPPORTED, "queue: a warp's buffer exceeds the shared memory");
  plan.args_bytes = (size_t)nseg * sizeof(CoopArgs);
  args_blob.resize(plan.args_bytes);
  if (nseg) memcpy(args_blob.data(), args.data(), plan.args_bytes);
  return GBX_OK;
}

int launch_queue(const void* d_args, const QueueSeg* d_segs, unsigned long long* cursor,
                 const QueuePlan& plan, int device, cudaStream_t st) {
  if (plan.total == 0) return GBX_OK;
  int s = cuda_status(cudaFuncSetAttribute(eri_queue, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)kCoopMaxSmem), "eri_queue shared memory attribute");
  if (s) return s;
  int nsm = 1, per_sm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  s = cuda_status(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, eri_queue, 32 * plan.wpc,
                                                                plan.smem),
                  "eri_queue occupancy");
  if (s) return s;
  // persistent: the CTAs that are resident together, no more than the queue needs
  const long long grid = std::max<long long>(
      1, std::min<long long>((long long)nsm * std::max(1, per_sm), (plan.total + plan.wpc - 1) / plan.wpc));
  eri_queue<<<(int)grid, 32 * plan.wpc, plan.smem, st>>>(
      static_cast<const CoopArgs*>(d_args), d_segs, plan.nseg, plan.total, cursor,
      plan.smem_per_warp);
  return cuda_status(cudaGetLastError(), "eri_queue launch");
}

}  // namespace gbx
