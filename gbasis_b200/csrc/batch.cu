// Batched full tensors of many molecules, replayed as one CUDA graph.
//
// A batch merges its molecules' shells, pairs and primitive pairs into single device arrays
// (each pair records its molecule), and for every block type (bra pair class, ket pair
// class) concatenates the unique quartets of all molecules into one work list: one class
// kernel launch per block type covers the whole batch, writing each quartet into its own
// molecule's compact store (per-molecule block base and column count, looked up by the bra
// pair's molecule).  One batched row-staged expansion then writes every molecule's N^4
// tensor.  The work lists are static (full tensors screen nothing), so the launches — class
// kernels spread over auxiliary streams, joined, then the expansion — are captured once into
// a CUDA graph and replayed; output pointers and notation live in a device table that each
// run updates before the replay.  No counterpart in gbasis (one molecule per call there).
#include <algorithm>
#include <cstring>
#include <memory>
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

struct BatchType {
  int cb, ck;
  long long n = 0, work_off = 0;
  double avg_prims = 1.0;
  int team = 1;
  int variant = 0;      // heavy classes with both kernels: 0 split, 1 line kernel
  int ctas_per_sm = 8;  // grid cap of the register kernel (resident-CTA multiples of the SMs)
  long long* d_base = nullptr;   // per molecule: block base in the batch compact store
  long long* d_ncols = nullptr;  // per molecule: pair functions of the ket class
};

struct Batch {
  int device = 0;
  int nmol = 0;
  std::vector<std::unique_ptr<Basis>> mols;  // host tables of each molecule
  std::vector<long long> compact_off;
  std::vector<BatchType> types;
  std::vector<int> order;  // block types, largest estimated cost first
  ShellDev* d_shells = nullptr;
  PairDev* d_pairs = nullptr;
  PrimPair* d_prims = nullptr;
  double* d_exps = nullptr;
  double* d_coefs = nullptr;
  const double* d_boys = nullptr;
  int2* d_work = nullptr;
  unsigned long long* d_tickets = nullptr;  // per type: its FP64 and FP32 lists' work counters
  double* d_compact = nullptr;
  int* d_gtab = nullptr;
  int4* d_rowinfo = nullptr;
  BlockDev* d_blocks = nullptr;
  ExpandArgs* d_exp = nullptr;
  long long* d_row_first = nullptr;
  std::vector<ExpandArgs> h_exp;
  long long total_rows = 0, n_quartets = 0, compact_elems = 0;
  size_t max_row_bytes = 0;
  cudaStream_t exec = nullptr;
  std::vector<cudaStream_t> aux;
  std::vector<cudaEvent_t> join;
  cudaEvent_t fork = nullptr, ev_in = nullptr, ev_out = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t graph_exec = nullptr;
  bool use_graph = true;
  bool exp_dirty = true;
  // per-type timing (autotuner): types run one after another on the exec stream, eagerly
  bool profile = false;
  std::vector<cudaEvent_t> type_ev;
  std::vector<void*> allocs;
  // mixed-precision form: the FP64 work list and first merged pair of each molecule kept on
  // the host; per pair the bound of its output functions; per type, in d_work_mixed, the
  // FP64 quartets followed by the FP32 ones (quartets below the skip bound left out)
  std::vector<int2> h_work;
  std::vector<long long> pair_off;
  std::vector<double> h_qmixed;
  int2* d_work_mixed = nullptr;
  std::vector<long long> mix_off, mix_n64, mix_n32;
  long long mix_count[3] = {0, 0, 0};  // FP64, FP32, skipped quartets
  double mix_skip = -1.0, mix_fp32 = -1.0;
  cudaGraph_t graph_m = nullptr;
  cudaGraphExec_t graph_exec_m = nullptr;
  // multi-class queue form (gbx_batch_set_queue): the FP64 run's class kernels replaced by one
  // persistent eri_queue launch that drains every block type's quartets from a single queue
  bool use_queue = false;
  void* d_qargs = nullptr;
  QueueSeg* d_qsegs = nullptr;
  unsigned long long* d_qcursor = nullptr;
  QueuePlan qplan;
  unsigned long long* d_fault = nullptr;  // debug builds: fault word of the bounds checks

  int alloc(void** p, size_t bytes, const char* what) {
    if (bytes == 0) bytes = 16;
    GBX_CUDA(cudaMalloc(p, bytes), what);
    allocs.push_back(*p);
    return GBX_OK;
  }
  template <typename T>
  int upload(T** d, const std::vector<T>& h, const char* what) {
    int s = alloc((void**)d, h.size() * sizeof(T), what);
    if (s) return s;
    GBX_CUDA(cudaMemcpy(*d, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice), what);
    return GBX_OK;
  }
  ~Batch() {
    int prev = -1;
    cudaGetDevice(&prev);
    cudaSetDevice(device);
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph) cudaGraphDestroy(graph);
    if (graph_exec_m) cudaGraphExecDestroy(graph_exec_m);
    if (graph_m) cudaGraphDestroy(graph_m);
    for (void* p : allocs) cudaFree(p);
    for (cudaStream_t s : aux) cudaStreamDestroy(s);
    for (cudaEvent_t e : join) cudaEventDestroy(e);
    for (cudaEvent_t e : type_ev) cudaEventDestroy(e);
    if (fork) cudaEventDestroy(fork);
    if (ev_in) cudaEventDestroy(ev_in);
    if (ev_out) cudaEventDestroy(ev_out);
    if (exec) cudaStreamDestroy(exec);
    if (prev >= 0) cudaSetDevice(prev);
  }
};

// Lanes per quartet of the register kernel: about four primitive quartets per lane, fewer
// lanes when the accumulator set (reduced by shuffles) is large.
static int default_team(int cb, int ck, double avg_prims) {
  const int la = kPairClassL[cb][0], lb = kPairClassL[cb][1];
  const int lc = kPairClassL[ck][0], ld = kPairClassL[ck][1];
  int ne = 0, nf = 0;
  for (int e = la; e <= la + lb; ++e) ne += ncart(e);
  for (int f = lc; f <= lc + ld; ++f) nf += ncart(f);
  const int cap = ne * nf > 100 ? 2 : (ne * nf > 40 ? 8 : 32);
  int t = 1;
  while (t < cap && avg_prims / (2 * t) >= 4.0) t *= 2;
  return t;
}

static int build_batch(Batch& Bt, int n_mol, const int* mol_nshells, const int* angmom,
                       const int* nprim, const double* center, const double* exps,
                       const double* coefs, const int* nout, const int* sph, const int8_t* pos,
                       const double* scl) {
  Bt.nmol = n_mol;
  std::vector<ShellDev> shells;
  std::vector<PairDev> pairs;
  std::vector<double> hexps, hcoefs;
  std::vector<long long> pair_off(n_mol + 1, 0);
  long long sh0 = 0, ex0 = 0, pp0 = 0, c0 = 0;
  for (int m = 0; m < n_mol; ++m) {
    const int ns = mol_nshells[m];
    if (ns <= 0) return set_error(GBX_ERR_INVALID, "molecule %d has no shells", m);
    long long nex = 0;
    for (int s = 0; s < ns; ++s) nex += nprim[sh0 + s];
    auto B = std::make_unique<Basis>();
    B->device = Bt.device;
    B->lmax_supported = compiled_lmax();
    int s = build_basis(*B, ns, angmom + sh0, nprim + sh0, center + 3 * sh0, exps + ex0,
                        coefs + ex0, nout + sh0, sph + sh0, pos + kMaxCart * sh0,
                        scl + kMaxCart * sh0);
    if (s) return set_error(s, "molecule %d: %s", m, gbx_last_error_str());
    for (ShellDev d : B->shells) {
      d.prim_off += (int)ex0;
      shells.push_back(d);
    }
    for (PairDev p : B->pairs) {
      p.shA += (int)sh0;
      p.shB += (int)sh0;
      p.prim_off += (int)pp0;
      p.mol = m;
      pairs.push_back(p);
    }
    hexps.insert(hexps.end(), exps + ex0, exps + ex0 + nex);
    hcoefs.insert(hcoefs.end(), coefs + ex0, coefs + ex0 + nex);
    pair_off[m + 1] = pair_off[m] + (long long)B->pairs.size();
    Bt.compact_off.push_back(c0);
    c0 += B->compact_elems;
    sh0 += ns;
    ex0 += nex;
    pp0 += B->n_prim_pairs;
    Bt.mols.push_back(std::move(B));
  }
  Bt.compact_elems = c0;
  if (pp0 > (1LL << 31) - 1 || (long long)pairs.size() > (1LL << 31) - 1)
    return set_error(GBX_ERR_UNSUPPORTED, "batch too large for 32-bit pair indices");

  // block types: every molecule's quartets of (cb, ck), concatenated
  std::vector<int2> work;
  std::vector<std::vector<long long>> tbase, tcols;
  for (int cb = 0; cb < kNumPairClasses; ++cb)
    for (int ck = 0; ck <= cb; ++ck) {
      BatchType T;
      T.cb = cb;
      T.ck = ck;
      T.work_off = (long long)work.size();
      std::vector<long long> base(n_mol, 0), cols(n_mol, 0);
      double prim_sum = 0.0;
      for (int m = 0; m < n_mol; ++m) {
        const Basis& B = *Bt.mols[m];
        const BlockDev& bd = B.block_table[(size_t)cb * kNumPairClasses + ck];
        if (bd.base < 0) continue;
        base[m] = Bt.compact_off[m] + bd.base;
        cols[m] = bd.ncols;
        const long long fb = B.class_first[cb], nb = B.class_count[cb];
        const long long fk = B.class_first[ck], nk = B.class_count[ck];
        for (long long pl = 0; pl < nb; ++pl) {
          const long long qn = (cb == ck) ? pl + 1 : nk;
          const int p = (int)(pair_off[m] + fb + pl);
          for (long long ql = 0; ql < qn; ++ql) {
            const int q = (int)(pair_off[m] + fk + ql);
            // diagonal block types: the better-conditioned pair is the bra
            if (block_orients(cb, ck) && pairs[q].orient < pairs[p].orient)
              work.push_back(make_int2(q, p));
            else work.push_back(make_int2(p, q));
            prim_sum += (double)pairs[p].nprim * pairs[q].nprim;
          }
        }
      }
      T.n = (long long)work.size() - T.work_off;
      if (T.n == 0) continue;
      T.avg_prims = prim_sum / (double)T.n;
      T.team = default_team(cb, ck, T.avg_prims);
      Bt.types.push_back(T);
      tbase.push_back(std::move(base));
      tcols.push_back(std::move(cols));
    }
  Bt.n_quartets = (long long)work.size();
  std::vector<double> cost(Bt.types.size());
  for (size_t k = 0; k < Bt.types.size(); ++k) {
    const BatchType& T = Bt.types[k];
    cost[k] = (double)T.n * (T.avg_prims + 4.0) * ncart(kPairClassL[T.cb][0]) *
              ncart(kPairClassL[T.cb][1]) * ncart(kPairClassL[T.ck][0]) * ncart(kPairClassL[T.ck][1]);
  }
  Bt.order.resize(Bt.types.size());
  for (size_t k = 0; k < Bt.order.size(); ++k) Bt.order[k] = (int)k;
  std::stable_sort(Bt.order.begin(), Bt.order.end(), [&](int x, int y) { return cost[x] > cost[y]; });

  // device arrays
  DeviceGuardLite g(Bt.device);
  int s;
  if ((s = Bt.upload(&Bt.d_shells, shells, "upload batch shells"))) return s;
  if ((s = Bt.upload(&Bt.d_pairs, pairs, "upload batch pairs"))) return s;
  if ((s = Bt.upload(&Bt.d_exps, hexps, "upload batch exponents"))) return s;
  if ((s = Bt.upload(&Bt.d_coefs, hcoefs, "upload batch coefficients"))) return s;
  if ((s = Bt.upload(&Bt.d_work, work, "upload batch work list"))) return s;
  Bt.h_work = std::move(work);
  Bt.pair_off = pair_off;
  if ((s = Bt.alloc((void**)&Bt.d_prims, (size_t)std::max<long long>(pp0, 1) * sizeof(PrimPair),
                    "cudaMalloc(batch primitive pairs)")))
    return s;
  const int np = (int)pairs.size();
  pair_precompute<<<(np + 127) / 128, 128>>>(Bt.d_pairs, np, Bt.d_shells, Bt.d_exps, Bt.d_coefs,
                                             Bt.d_prims);
  GBX_CUDA(cudaGetLastError(), "pair_precompute launch");
  if ((s = boys_table(Bt.device, &Bt.d_boys))) return s;
  for (size_t k = 0; k < Bt.types.size(); ++k) {
    if ((s = Bt.upload(&Bt.types[k].d_base, tbase[k], "upload batch block bases"))) return s;
    if ((s = Bt.upload(&Bt.types[k].d_ncols, tcols[k], "upload batch block columns"))) return s;
  }
  if ((s = Bt.alloc((void**)&Bt.d_compact, (size_t)Bt.compact_elems * sizeof(double),
                    "cudaMalloc(batch compact store)")))
    return s;

  // expansion tables and descriptors
  std::vector<int> gtab;
  std::vector<int4> rowinfo;
  std::vector<BlockDev> blocks;
  std::vector<long long> goff, roff, boff;
  std::vector<long long> row_first(n_mol + 1, 0);
  for (int m = 0; m < n_mol; ++m) {
    const Basis& B = *Bt.mols[m];
    goff.push_back((long long)gtab.size());
    roff.push_back((long long)rowinfo.size());
    boff.push_back((long long)blocks.size());
    gtab.insert(gtab.end(), B.h_gtab.begin(), B.h_gtab.end());
    rowinfo.insert(rowinfo.end(), B.h_rowinfo.begin(), B.h_rowinfo.end());
    blocks.insert(blocks.end(), B.block_table.begin(), B.block_table.end());
    const long long npf = B.pf_first[kNumPairClasses];
    row_first[m + 1] = row_first[m] + npf;
    Bt.max_row_bytes = std::max(Bt.max_row_bytes, (size_t)npf * sizeof(double));
  }
  Bt.total_rows = row_first[n_mol];
  if ((s = Bt.upload(&Bt.d_gtab, gtab, "upload batch gtab"))) return s;
  if ((s = Bt.upload(&Bt.d_rowinfo, rowinfo, "upload batch rowinfo"))) return s;
  if ((s = Bt.upload(&Bt.d_blocks, blocks, "upload batch block tables"))) return s;
  if ((s = Bt.upload(&Bt.d_row_first, row_first, "upload batch row offsets"))) return s;
  if ((s = alloc_fault_word(&Bt.d_fault))) return s;
  if (Bt.d_fault) Bt.allocs.push_back(Bt.d_fault);
  Bt.h_exp.resize(n_mol);
  for (int m = 0; m < n_mol; ++m) {
    const Basis& B = *Bt.mols[m];
    ExpandArgs e;
    memset(&e, 0, sizeof(e));
    e.fault = Bt.d_fault;
    e.out_len = B.nbf * B.nbf * B.nbf * B.nbf;
    e.compact_len = (m + 1 < n_mol ? Bt.compact_off[m + 1] : Bt.compact_elems) - Bt.compact_off[m];
    e.n = B.nbf;
    e.nsh = (int)B.shells.size();
    e.notation = GBX_CHEMIST;
    e.blocks = Bt.d_blocks + boff[m];
    e.compact = Bt.d_compact + Bt.compact_off[m];
    e.out = nullptr;
    e.gtab = Bt.d_gtab + goff[m];
    e.rowinfo = Bt.d_rowinfo + roff[m];
    e.npf = B.pf_first[kNumPairClasses];
    for (int c = 0; c <= kNumPairClasses; ++c) e.pf_first[c] = B.pf_first[c];
    Bt.h_exp[m] = e;
  }
  if ((s = Bt.alloc((void**)&Bt.d_exp, n_mol * sizeof(ExpandArgs), "cudaMalloc(batch descriptors)")))
    return s;
  if ((s = Bt.alloc((void**)&Bt.d_tickets, 2 * Bt.types.size() * sizeof(unsigned long long),
                    "cudaMalloc(batch work counters)")))
    return s;
  GBX_CUDA(cudaStreamCreateWithFlags(&Bt.exec, cudaStreamNonBlocking), "create stream");
  Bt.aux.resize(kAuxStreams);
  Bt.join.resize(kAuxStreams);
  for (int j = 0; j < kAuxStreams; ++j) {
    GBX_CUDA(cudaStreamCreateWithFlags(&Bt.aux[j], cudaStreamNonBlocking), "create stream");
    GBX_CUDA(cudaEventCreateWithFlags(&Bt.join[j], cudaEventDisableTiming), "create event");
  }
  GBX_CUDA(cudaEventCreateWithFlags(&Bt.fork, cudaEventDisableTiming), "create event");
  GBX_CUDA(cudaEventCreateWithFlags(&Bt.ev_in, cudaEventDisableTiming), "create event");
  GBX_CUDA(cudaEventCreateWithFlags(&Bt.ev_out, cudaEventDisableTiming), "create event");
  GBX_CUDA(cudaDeviceSynchronize(), "batch upload");
  return GBX_OK;
}

// Mixed form, bounds: Q_p = sqrt(max |(ab|ab)|) over the output functions of every merged
// pair, as a single basis computes them (Cauchy-Schwarz for the final values, so
// |(ab|cd)| <= Q_p Q_q).  The diagonal quartets (p, p) of all molecules run through the class
// kernels into the batch compact store (scratch here: every run overwrites it), then
// diagonal_bounds reads each molecule's diagonals.  Once per batch, on Bt.exec, synchronous.
static int batch_mixed_bounds(Batch& Bt) {
  if (!Bt.h_qmixed.empty()) return GBX_OK;
  const long long np = Bt.pair_off[Bt.nmol];
  std::vector<int2> diag;
  diag.reserve((size_t)np);
  std::vector<long long> first(kNumPairClasses + 1, 0);
  for (int c = 0; c < kNumPairClasses; ++c) {
    first[c] = (long long)diag.size();
    for (int m = 0; m < Bt.nmol; ++m) {
      const Basis& B = *Bt.mols[m];
      for (long long pl = 0; pl < B.class_count[c]; ++pl) {
        const int p = (int)(Bt.pair_off[m] + B.class_first[c] + pl);
        diag.push_back(make_int2(p, p));
      }
    }
  }
  first[kNumPairClasses] = (long long)diag.size();
  if ((long long)diag.size() != np)
    return set_error(GBX_ERR_INVALID, "batch pair classes cover %lld of %lld pairs",
                     (long long)diag.size(), np);
  int2* d_diag = nullptr;
  double* d_q = nullptr;
  GBX_CUDA(cudaMalloc(&d_diag, std::max<size_t>(diag.size(), 1) * sizeof(int2)),
           "cudaMalloc(batch diagonal quartets)");
  cudaError_t e = cudaMalloc(&d_q, std::max<long long>(np, 1) * sizeof(double));
  if (e == cudaSuccess)
    e = cudaMemcpy(d_diag, diag.data(), diag.size() * sizeof(int2), cudaMemcpyHostToDevice);
  int s = cuda_status(e, "batch mixed-form bounds setup");
  const int nsm = num_sms_of(Bt.device);
  for (int c = 0; c < kNumPairClasses && !s; ++c) {
    const long long n = first[c + 1] - first[c];
    if (n == 0) continue;
    const BatchType* T = nullptr;
    for (const BatchType& t : Bt.types)
      if (t.cb == c && t.ck == c) T = &t;
    if (!T) {
      s = set_error(GBX_ERR_INVALID, "batch has pairs of class %d but no diagonal block type", c);
      break;
    }
    EriLaunch a;
    memset(&a, 0, sizeof(a));
    a.pairs = Bt.d_pairs;
    a.prims = Bt.d_prims;
    a.shells = Bt.d_shells;
    a.boys_tab = Bt.d_boys;
    a.out = Bt.d_compact;
    a.work = d_diag;
    a.work_off = first[c];
    a.nwork = n;
    a.mode = 0;
    a.team = 1;
    a.mol_base = T->d_base;
    a.mol_ncols = T->d_ncols;
    const int grid = (int)std::max<long long>(1, std::min<long long>((n + 127) / 128,
                                                                     (long long)nsm * 8));
    s = launch_class(kPairClassL[c][0], kPairClassL[c][1], kPairClassL[c][0], kPairClassL[c][1],
                     a, grid, Bt.exec);
  }
  for (int m = 0; m < Bt.nmol && !s; ++m)
    s = launch_diagonal_bounds(Bt.d_pairs + Bt.pair_off[m],
                               (int)(Bt.pair_off[m + 1] - Bt.pair_off[m]), Bt.d_shells,
                               Bt.h_exp[m].blocks, Bt.h_exp[m].compact, d_q + Bt.pair_off[m],
                               Bt.exec);
  e = cudaStreamSynchronize(Bt.exec);
  if (!s) s = cuda_status(e, "batch mixed-form bounds");
  if (!s) {
    Bt.h_qmixed.resize((size_t)np);
    s = cuda_status(cudaMemcpy(Bt.h_qmixed.data(), d_q, np * sizeof(double),
                               cudaMemcpyDeviceToHost), "download batch bounds");
    if (s) Bt.h_qmixed.clear();
  }
  cudaFree(d_diag);
  if (d_q) cudaFree(d_q);
  return s;
}

// Drops the captured graph of the mixed form (thresholds or teams changed).
static void batch_drop_mixed_graph(Batch& B) {
  if (B.graph_exec_m) cudaGraphExecDestroy(B.graph_exec_m);
  if (B.graph_m) cudaGraphDestroy(B.graph_m);
  B.graph_exec_m = nullptr;
  B.graph_m = nullptr;
}

// Mixed form, work lists: per block type the FP64 quartets, then those whose bound is below
// `fp32` (light classes only: the register kernel has the FP32 recursions), leaving out those
// below `skip`.  The thresholds decide exactly as the single-basis work-list build does.
static int batch_mixed_lists(Batch& Bt, double skip, double fp32) {
  if (Bt.d_work_mixed && skip == Bt.mix_skip && fp32 == Bt.mix_fp32) return GBX_OK;
  int s;
  if ((s = batch_mixed_bounds(Bt))) return s;
  const size_t nt = Bt.types.size();
  std::vector<int2> w, w32;
  w.reserve(Bt.h_work.size());
  Bt.mix_off.assign(nt, 0);
  Bt.mix_n64.assign(nt, 0);
  Bt.mix_n32.assign(nt, 0);
  long long nskip = 0;
  for (size_t k = 0; k < nt; ++k) {
    const BatchType& T = Bt.types[k];
    const bool light = coop_class(kPairClassL[T.cb][0], kPairClassL[T.cb][1],
                                  kPairClassL[T.ck][0], kPairClassL[T.ck][1]) < 0;
    Bt.mix_off[k] = (long long)w.size();
    w32.clear();
    for (long long i = 0; i < T.n; ++i) {
      const int2 pq = Bt.h_work[(size_t)(T.work_off + i)];
      const double bnd = Bt.h_qmixed[pq.x] * Bt.h_qmixed[pq.y];
      if (bnd < skip) {
        ++nskip;
        continue;
      }
      if (light && bnd < fp32)
        w32.push_back(pq);
      else
        w.push_back(pq);
    }
    Bt.mix_n64[k] = (long long)w.size() - Bt.mix_off[k];
    Bt.mix_n32[k] = (long long)w32.size();
    w.insert(w.end(), w32.begin(), w32.end());
  }
  if (!Bt.d_work_mixed &&
      (s = Bt.alloc((void**)&Bt.d_work_mixed, std::max<size_t>(Bt.h_work.size(), 1) * sizeof(int2),
                    "cudaMalloc(batch mixed work list)")))
    return s;
  GBX_CUDA(cudaMemcpy(Bt.d_work_mixed, w.data(), w.size() * sizeof(int2), cudaMemcpyHostToDevice),
           "upload batch mixed work list");
  long long n32 = 0;
  for (long long v : Bt.mix_n32) n32 += v;
  Bt.mix_count[0] = (long long)w.size() - n32;
  Bt.mix_count[1] = n32;
  Bt.mix_count[2] = nskip;
  Bt.mix_skip = skip;
  Bt.mix_fp32 = fp32;
  batch_drop_mixed_graph(Bt);
  return GBX_OK;
}

// Arguments of block type k's class-kernel launches (FP64 work list, per-molecule stores).
static EriLaunch type_launch(const Batch& Bt, int k) {
  const BatchType& T = Bt.types[k];
  EriLaunch a;
  memset(&a, 0, sizeof(a));
  a.pairs = Bt.d_pairs;
  a.prims = Bt.d_prims;
  a.shells = Bt.d_shells;
  a.boys_tab = Bt.d_boys;
  a.out = Bt.d_compact;
  a.work = Bt.d_work;
  a.work_off = T.work_off;
  a.nwork = T.n;
  a.mode = 0;
  a.team = T.team;
  a.variant = T.variant;
  a.mol_base = T.d_base;
  a.mol_ncols = T.d_ncols;
  a.fault = Bt.d_fault;
  a.out_len = Bt.compact_elems;
  return a;
}

// The queue of the multi-class form, made on first use: the block types in launch order
// (largest estimated cost first, so that the long quartets are drawn early), each a segment
// with its class's programs.
static int ensure_queue(Batch& Bt) {
  if (Bt.d_qargs) return GBX_OK;
  const int nseg = (int)Bt.order.size();
  std::vector<EriLaunch> launches(nseg);
  std::vector<int> progs(nseg);
  std::vector<long long> counts(nseg);
  for (int i = 0; i < nseg; ++i) {
    const int k = Bt.order[i];
    const BatchType& T = Bt.types[k];
    launches[i] = type_launch(Bt, k);
    progs[i] = coop_program(kPairClassL[T.cb][0], kPairClassL[T.cb][1], kPairClassL[T.ck][0],
                            kPairClassL[T.ck][1]);
    counts[i] = T.n;
  }
  std::vector<unsigned char> blob;
  std::vector<QueueSeg> segs;
  int s = queue_plan(launches.data(), progs.data(), counts.data(), nseg, blob, segs, Bt.qplan);
  if (s) return s;
  void* dargs = nullptr;
  if ((s = Bt.alloc(&dargs, blob.size(), "cudaMalloc(queue arguments)"))) return s;
  GBX_CUDA(cudaMemcpy(dargs, blob.data(), blob.size(), cudaMemcpyHostToDevice),
           "upload queue arguments");
  if ((s = Bt.upload(&Bt.d_qsegs, segs, "upload queue segments"))) return s;
  if ((s = Bt.alloc((void**)&Bt.d_qcursor, sizeof(unsigned long long), "cudaMalloc(queue cursor)")))
    return s;
  Bt.d_qargs = dargs;
  return GBX_OK;
}

// The launches of one batch run on stream `st` (class kernels on the auxiliary streams).
// mixed: the lists of batch_mixed_lists, FP32 lists on the register kernel's FP32 path, and
// the compact store cleared first when quartets were left out (their values are zero).
static int enqueue_batch(Batch& Bt, cudaStream_t st, bool mixed = false) {
  const int nsm = num_sms_of(Bt.device);
  if (Bt.use_queue && !mixed && !Bt.profile) {
    // multi-class form: one persistent launch drains every block type, then the expansion
    int s = ensure_queue(Bt);
    if (s) return s;
    GBX_CUDA(cudaMemsetAsync(Bt.d_qcursor, 0, sizeof(unsigned long long), st), "clear queue cursor");
    if ((s = launch_queue(Bt.d_qargs, Bt.d_qsegs, Bt.d_qcursor, Bt.qplan, Bt.device, st))) return s;
    return launch_expand_batch(Bt.device, Bt.d_exp, Bt.d_row_first, Bt.nmol, Bt.total_rows,
                               Bt.max_row_bytes, st);
  }
  if (mixed && Bt.mix_count[2] > 0)
    GBX_CUDA(cudaMemsetAsync(Bt.d_compact, 0, (size_t)Bt.compact_elems * sizeof(double), st),
             "clear batch compact store");
  const bool tickets = !static_work_order();
  if (tickets)
    GBX_CUDA(cudaMemsetAsync(Bt.d_tickets, 0, 2 * Bt.types.size() * sizeof(unsigned long long), st),
             "clear batch work counters");
  GBX_CUDA(cudaEventRecord(Bt.fork, st), "fork");
  for (cudaStream_t a : Bt.aux) GBX_CUDA(cudaStreamWaitEvent(a, Bt.fork, 0), "fork wait");
  for (size_t i = 0; i < Bt.order.size(); ++i) {
    const int k = Bt.order[i];
    const BatchType& T = Bt.types[k];
    if (Bt.profile) GBX_CUDA(cudaEventRecord(Bt.type_ev[i], st), "type event");
    EriLaunch a = type_launch(Bt, k);
    a.ticket = tickets ? Bt.d_tickets + 2 * k : nullptr;
    cudaStream_t ts = Bt.profile ? st : Bt.aux[i % Bt.aux.size()];
    if (mixed) {
      a.work = Bt.d_work_mixed;
      a.work_off = Bt.mix_off[k];
      a.nwork = Bt.mix_n64[k];
    }
    if (a.nwork > 0) {
      const int grid = (int)std::max<long long>(
          1, std::min<long long>((a.nwork * T.team + 127) / 128, (long long)nsm * T.ctas_per_sm));
      int s = launch_class(kPairClassL[T.cb][0], kPairClassL[T.cb][1], kPairClassL[T.ck][0],
                           kPairClassL[T.ck][1], a, grid, ts);
      if (s) return s;
    }
    if (mixed && Bt.mix_n32[k] > 0) {  // the type's FP32 list
      a.work_off = Bt.mix_off[k] + Bt.mix_n64[k];
      a.nwork = Bt.mix_n32[k];
      a.fp32 = 1;
      a.ticket = tickets ? Bt.d_tickets + 2 * k + 1 : nullptr;
      const int grid = (int)std::max<long long>(
          1, std::min<long long>((a.nwork * T.team + 127) / 128, (long long)nsm * T.ctas_per_sm));
      int s = launch_class(kPairClassL[T.cb][0], kPairClassL[T.cb][1], kPairClassL[T.ck][0],
                           kPairClassL[T.ck][1], a, grid, ts);
      if (s) return s;
    }
  }
  if (Bt.profile) GBX_CUDA(cudaEventRecord(Bt.type_ev[Bt.order.size()], st), "type event");
  for (size_t j = 0; j < Bt.aux.size(); ++j) {
    GBX_CUDA(cudaEventRecord(Bt.join[j], Bt.aux[j]), "join");
    GBX_CUDA(cudaStreamWaitEvent(st, Bt.join[j], 0), "join wait");
  }
  return launch_expand_batch(Bt.device, Bt.d_exp, Bt.d_row_first, Bt.nmol, Bt.total_rows,
                             Bt.max_row_bytes, st);
}

// mixed: thresholds (skip, fp32) of the mixed form, nullptr for the FP64 form.
static int run_batch(Batch& Bt, int notation, double* const* outs, cudaStream_t caller,
                     const double* mixed = nullptr) {
  NvtxRange range("gbx batch run");
  for (int m = 0; m < Bt.nmol; ++m)
    if (!outs[m]) return set_error(GBX_ERR_INVALID, "output of molecule %d is null", m);
  bool changed = Bt.exp_dirty;
  for (int m = 0; m < Bt.nmol; ++m) {
    if (Bt.h_exp[m].out != outs[m] || Bt.h_exp[m].notation != notation) changed = true;
    Bt.h_exp[m].out = outs[m];
    Bt.h_exp[m].out_lo = outs[m];
    Bt.h_exp[m].notation = notation;
  }
  GBX_CUDA(cudaEventRecord(Bt.ev_in, caller), "record caller");
  GBX_CUDA(cudaStreamWaitEvent(Bt.exec, Bt.ev_in, 0), "wait caller");
  if (changed) {
    Bt.exp_dirty = true;  // until the device table holds these outputs
    GBX_CUDA(cudaMemcpyAsync(Bt.d_exp, Bt.h_exp.data(), Bt.nmol * sizeof(ExpandArgs),
                             cudaMemcpyHostToDevice, Bt.exec), "upload batch descriptors");
    GBX_CUDA(cudaStreamSynchronize(Bt.exec), "upload batch descriptors");
    Bt.exp_dirty = false;
  }
  const bool mx = mixed != nullptr;
  if (mx) {
    const int s = batch_mixed_lists(Bt, mixed[0], mixed[1]);
    if (s) return s;
  }
  cudaGraph_t& graph_ref = mx ? Bt.graph_m : Bt.graph;
  cudaGraphExec_t& exec_ref = mx ? Bt.graph_exec_m : Bt.graph_exec;
  const bool graph = Bt.use_graph && !Bt.profile;
  if (graph && !exec_ref) {
    GBX_CUDA(cudaStreamBeginCapture(Bt.exec, cudaStreamCaptureModeRelaxed), "begin capture");
    const int s = enqueue_batch(Bt, Bt.exec, mx);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(Bt.exec, &g);
    if (s) {
      if (g) cudaGraphDestroy(g);
      return s;
    }
    GBX_CUDA(e, "end capture");
    graph_ref = g;
    GBX_CUDA(cudaGraphInstantiate(&exec_ref, g, 0), "instantiate batch graph");
  }
  if (graph) {
    GBX_CUDA(cudaGraphLaunch(exec_ref, Bt.exec), "launch batch graph");
  } else {
    const int s = enqueue_batch(Bt, Bt.exec, mx);
    if (s) return s;
  }
  GBX_CUDA(cudaEventRecord(Bt.ev_out, Bt.exec), "record batch");
  GBX_CUDA(cudaStreamWaitEvent(caller, Bt.ev_out, 0), "caller wait");
  return GBX_OK;
}

}  // namespace gbx

using namespace gbx;

struct gbx_batch {
  std::unique_ptr<Batch> impl;
};

int gbx_batch_create(gbx_batch** out, int n_mol, const int* mol_nshells, const int* angmom,
                     const int* nprim, const double* center, const double* exps,
                     const double* coefs, const int* nout, const int* sph, const int8_t* pos,
                     const double* scl, int device) {
  if (!out || n_mol <= 0 || !mol_nshells || !angmom || !nprim || !center || !exps || !coefs ||
      !nout || !sph || !pos || !scl)
    return set_error(GBX_ERR_INVALID, "gbx_batch_create: null argument or empty batch");
  *out = nullptr;
  int ndev = 0;
  GBX_CUDA(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
  if (device < 0 || device >= ndev)
    return set_error(GBX_ERR_INVALID, "device %d not present (%d devices)", device, ndev);
  auto B = std::make_unique<Batch>();
  B->device = device;
  DeviceGuardLite g(device);
  const int s = build_batch(*B, n_mol, mol_nshells, angmom, nprim, center, exps, coefs, nout,
                            sph, pos, scl);
  if (s) return s;
  *out = new gbx_batch{std::move(B)};
  return GBX_OK;
}

int gbx_batch_destroy(gbx_batch* b) {
  delete b;
  return GBX_OK;
}

int gbx_batch_info(const gbx_batch* b, int64_t* nbf, int64_t* n_quartets, int64_t* compact_bytes) {
  if (!b) return set_error(GBX_ERR_INVALID, "gbx_batch_info: null batch");
  const Batch& B = *b->impl;
  if (nbf)
    for (int m = 0; m < B.nmol; ++m) nbf[m] = B.mols[m]->nbf;
  if (n_quartets) *n_quartets = B.n_quartets;
  if (compact_bytes) *compact_bytes = B.compact_elems * (int64_t)sizeof(double);
  return GBX_OK;
}

int gbx_batch_set_graph(gbx_batch* b, int on) {
  if (!b) return set_error(GBX_ERR_INVALID, "gbx_batch_set_graph: null batch");
  b->impl->use_graph = on != 0;
  return GBX_OK;
}

// Drops the captured graph so that the next run captures the current launch parameters.
static void batch_drop_graph(Batch& B) {
  if (B.graph_exec) cudaGraphExecDestroy(B.graph_exec);
  if (B.graph) cudaGraphDestroy(B.graph);
  B.graph_exec = nullptr;
  B.graph = nullptr;
  batch_drop_mixed_graph(B);
}

int gbx_batch_set_queue(gbx_batch* b, int on) {
  if (!b) return set_error(GBX_ERR_INVALID, "gbx_batch_set_queue: null batch");
  Batch& B = *b->impl;
  if (B.use_queue != (on != 0)) {
    B.use_queue = on != 0;
    batch_drop_graph(B);
  }
  return GBX_OK;
}

int gbx_batch_num_types(const gbx_batch* b, int* n) {
  if (!b || !n) return set_error(GBX_ERR_INVALID, "gbx_batch_num_types: null argument");
  *n = (int)b->impl->types.size();
  return GBX_OK;
}

int gbx_batch_type_info(const gbx_batch* b, int k, int* cls4, int* team, double* avg_prims,
                        int64_t* n_quartets) {
  if (!b) return set_error(GBX_ERR_INVALID, "gbx_batch_type_info: null batch");
  const Batch& B = *b->impl;
  if (k < 0 || k >= (int)B.types.size()) return set_error(GBX_ERR_INVALID, "type %d out of range", k);
  const BatchType& T = B.types[k];
  if (cls4) {
    cls4[0] = kPairClassL[T.cb][0];
    cls4[1] = kPairClassL[T.cb][1];
    cls4[2] = kPairClassL[T.ck][0];
    cls4[3] = kPairClassL[T.ck][1];
  }
  if (team) *team = T.team;
  if (avg_prims) *avg_prims = T.avg_prims;
  if (n_quartets) *n_quartets = T.n;
  return GBX_OK;
}

int gbx_batch_set_type_config(gbx_batch* b, int k, int variant, int ctas_per_sm) {
  if (!b) return set_error(GBX_ERR_INVALID, "gbx_batch_set_type_config: null batch");
  Batch& B = *b->impl;
  if (k < 0 || k >= (int)B.types.size()) return set_error(GBX_ERR_INVALID, "type %d out of range", k);
  if (variant < 0 || variant > 2) return set_error(GBX_ERR_INVALID, "variant must be 0, 1 or 2");
  if (ctas_per_sm < 1 || ctas_per_sm > 32)
    return set_error(GBX_ERR_INVALID, "ctas_per_sm must be in [1, 32]");
  BatchType& T = B.types[k];
  if (T.variant != variant || T.ctas_per_sm != ctas_per_sm) {
    T.variant = variant;
    T.ctas_per_sm = ctas_per_sm;
    batch_drop_graph(B);
  }
  return GBX_OK;
}

int gbx_batch_set_team(gbx_batch* b, int k, int team) {
  if (!b) return set_error(GBX_ERR_INVALID, "gbx_batch_set_team: null batch");
  Batch& B = *b->impl;
  if (k < 0 || k >= (int)B.types.size()) return set_error(GBX_ERR_INVALID, "type %d out of range", k);
  if (team < 1 || team > 32 || (team & (team - 1)))
    return set_error(GBX_ERR_INVALID, "team must be a power of two in [1, 32]");
  if (B.types[k].team != team) {
    B.types[k].team = team;
    batch_drop_graph(B);
  }
  return GBX_OK;
}

int gbx_batch_set_profiling(gbx_batch* b, int on) {
  if (!b) return set_error(GBX_ERR_INVALID, "gbx_batch_set_profiling: null batch");
  Batch& B = *b->impl;
  DeviceGuardLite g(B.device);
  if (on && B.type_ev.empty()) {
    B.type_ev.resize(B.types.size() + 1);
    for (cudaEvent_t& e : B.type_ev) GBX_CUDA(cudaEventCreate(&e), "cudaEventCreate");
  }
  B.profile = on != 0;
  return GBX_OK;
}

int gbx_batch_type_times(gbx_batch* b, double* ms, int n) {
  if (!b || !ms) return set_error(GBX_ERR_INVALID, "gbx_batch_type_times: null argument");
  Batch& B = *b->impl;
  if (!B.profile) return set_error(GBX_ERR_INVALID, "profiling is off");
  if (n < (int)B.types.size()) return set_error(GBX_ERR_INVALID, "ms holds %d < %d types", n, (int)B.types.size());
  DeviceGuardLite g(B.device);
  GBX_CUDA(cudaEventSynchronize(B.type_ev[B.order.size()]), "type events");
  for (size_t i = 0; i < B.order.size(); ++i) {
    float t = 0.f;
    GBX_CUDA(cudaEventElapsedTime(&t, B.type_ev[i], B.type_ev[i + 1]), "type elapsed time");
    ms[B.order[i]] = t;
  }
  return GBX_OK;
}

int gbx_batch_run(gbx_batch* b, int notation, double* const* outs, void* stream) {
  if (!b || !outs) return set_error(GBX_ERR_INVALID, "gbx_batch_run: null argument");
  if (notation != GBX_CHEMIST && notation != GBX_PHYSICIST)
    return set_error(GBX_ERR_INVALID, "notation must be GBX_CHEMIST or GBX_PHYSICIST");
  Batch& B = *b->impl;
  DeviceGuardLite g(B.device);
  const int s = run_batch(B, notation, outs, (cudaStream_t)stream);
  return s ? s : check_bounds_fault(B.d_fault, (cudaStream_t)stream, "gbx_batch_run");
}

int gbx_batch_run_mixed(gbx_batch* b, int notation, double skip, double fp32,
                        double* const* outs, void* stream) {
  if (!b || !outs) return set_error(GBX_ERR_INVALID, "gbx_batch_run_mixed: null argument");
  if (notation != GBX_CHEMIST && notation != GBX_PHYSICIST)
    return set_error(GBX_ERR_INVALID, "notation must be GBX_CHEMIST or GBX_PHYSICIST");
  if (!(skip >= 0.0) || !(fp32 >= 0.0))
    return set_error(GBX_ERR_INVALID, "thresholds must be >= 0");
  Batch& B = *b->impl;
  DeviceGuardLite g(B.device);
  const double th[2] = {skip, fp32};
  const int s = run_batch(B, notation, outs, (cudaStream_t)stream, th);
  return s ? s : check_bounds_fault(B.d_fault, (cudaStream_t)stream, "gbx_batch_run_mixed");
}

int gbx_batch_mixed_counts(const gbx_batch* b, int64_t* n_fp64, int64_t* n_fp32,
                           int64_t* n_skipped) {
  if (!b) return set_error(GBX_ERR_INVALID, "gbx_batch_mixed_counts: null batch");
  const Batch& B = *b->impl;
  if (n_fp64) *n_fp64 = B.mix_count[0];
  if (n_fp32) *n_fp32 = B.mix_count[1];
  if (n_skipped) *n_skipped = B.mix_count[2];
  return GBX_OK;
}
