// Host-side state of a basis handle (internal to libgbx_eri).
#pragma once
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <utility>
#include <vector>

#include "errors.h"
#include "gbx_common.cuh"
#include "gbx_eri.h"

namespace gbx {

// Named host-phase range for timeline profilers (NVTX push/pop; without an attached tool the
// calls return at once).  Entry points and their phases (basis upload, Schwarz bounds, work
// list and class kernels, expansion, host copies) open one for their scope.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

constexpr int kAuxStreams = 6;      // default concurrent class-block streams of a basis
constexpr int kMaxAuxStreams = 16;  // the most a basis may be given
// mixed form: smallest FP32 list given its own launch, and its least share of the block (1 in
// kFp32ListShare).  A list below either stays in the FP64 list: measured on the 120-function
// full tensor, lists of 2,048 quartets and a twentieth of a block (20,524 quartets in all)
// made the call 4 % slower than FP64 (their launches, Boys-table staging and tails cost more
// than FP32 recursions save on classes whose time goes to the Boys function)
constexpr long long kMinFp32List = 65536;
constexpr long long kFp32ListShare = 4;
constexpr long long kCoulombChunk = 1LL << 23;  // quartets per direct-Coulomb work chunk
constexpr int kStageBuffers = 3;                // host-output staging slabs in flight
constexpr size_t kStageBytes = 64ull << 20;     // target bytes of one staging slab

int boys_table(int device, const double** out);
int compiled_lmax();

// Diagonal blocks whose quartets run from the better-conditioned pair (quartet_transposed):
// those of pairs with lA + lB >= 3, where a contracted recursion run from a poorly placed
// centre loses digits; the lighter ones keep one orientation (no divergent stores).
inline bool block_orients(int cb, int ck) {
  return cb == ck && kPairClassL[cb][0] + kPairClassL[cb][1] >= 3;
}

struct HostBlock {
  int cb, ck;
  long long nb, nk, ncand;
  bool tri;
  BlockDev dev;
  double avg_prims = 1.0;  // mean primitive quartets per shell quartet
  int team = 1;            // lanes per quartet (register kernel), set by heuristic or autotuner
  int variant = 0;         // heavy classes with both kernels: 0 split, 1 line kernel
  int ctas_per_sm = 8;     // grid cap of the register kernel: resident-CTA multiples of the SMs
  long long j_computed = 0;  // quartets the last direct-J call computed in this block
};

struct Basis {
  int device = 0;
  int lmax_supported = 0;
  long long nbf = 0;
  std::vector<ShellDev> shells;
  std::vector<double> h_exps, h_coefs;
  std::vector<PairDev> pairs;
  std::vector<int> pair_of;  // n*n: (pair << 1) | (first index on B shell)
  std::vector<int> group;    // original (generalized) shell of each segmented shell
  std::vector<long long> h_ftab;  // nbf*nbf function-pair keys of the expansion
  long long* d_ftab = nullptr;
  // row-staged expansion: pair functions numbered class-major (pf_first[c] = first of class
  // c), gtab[x*nbf+y] = pair function of the ordered function pair (x, y), rowinfo[g] =
  // (x, y, 1 if (y, x) is the same pair function, local pair index in its class)
  std::vector<long long> pf_first;
  std::vector<int> h_gtab;
  std::vector<int4> h_rowinfo;
  int* d_gtab = nullptr;
  int4* d_rowinfo = nullptr;
  int2* d_jwork = nullptr;  // direct Coulomb: one work-chunk buffer per auxiliary stream
  long long jwork_cap = 0;
  void* d_jplan = nullptr;   // direct Coulomb: row starts, pair order, first ket positions
  size_t jplan_bytes = 0;
  unsigned long long* d_tickets = nullptr;  // work counters of one call's class launches
  long long tickets_cap = 0;
  int* d_counts32 = nullptr;   // mixed form: FP32 quartets per block
  double* d_qmixed = nullptr;  // mixed form: per-pair bound of the final values
  std::vector<long long> class_first, class_count, class_funcs;
  std::vector<HostBlock> blocks;
  std::vector<BlockDev> block_table;  // kNumPairClasses^2, base = -1 when empty
  long long compact_elems = 0, n_quartets = 0, n_prim_pairs = 0;

  // device copies
  ShellDev* d_shells = nullptr;
  PairDev* d_pairs = nullptr;
  PrimPair* d_prims = nullptr;
  double* d_exps = nullptr;
  double* d_coefs = nullptr;
  int* d_pair_of = nullptr;
  int* d_func_shell = nullptr;
  int* d_func_comp = nullptr;
  BlockDev* d_blocks = nullptr;
  int2* d_work = nullptr;
  int* d_counts = nullptr;  // per block screened count + status words
  double* d_q = nullptr;    // per-pair Schwarz bound (segmented)
  double* d_qscreen = nullptr;  // per-pair bound of the original shell pair
  int2* d_cta_map = nullptr;    // work-list build: (block, first candidate) per CTA
  void* d_build_blocks = nullptr;
  int4* d_pinfo = nullptr;      // per pair (cls, local, fo, nB) for the expansion
  int n_cta_build = 0;
  const double* d_boys = nullptr;
  double* d_compact = nullptr;
  size_t compact_cap = 0;
  double* d_out = nullptr;
  size_t out_cap = 0;
  bool schwarz_ready = false;
  bool mixed_ready = false;  // d_qmixed holds the final-value bounds
  std::vector<double> h_q;  // per pair, original-shell-pair bound
  long long last_computed = 0, last_screened = 0;
  bool counts_on_host = false;
  // mixed form: per block, upper bounds of the FP32 and left-out quartets at (skip, fp32)
  std::vector<long long> mix_n32, mix_nskip;
  double mix_key_skip = -1.0, mix_key_fp32 = -1.0;
  int* d_fp32_on = nullptr;  // per block: FP32 list in use
  int2* d_zero_work = nullptr;  // mixed form: left-out quartets of a call (zero_quartets)
  int* d_zero_count = nullptr;
  long long zero_cap = 0;
  bool last_mixed = false;  // the last compact-store call ran the mixed form
  long long fp32_min = kMinFp32List, fp32_share = kFp32ListShare;  // FP32 list rule
  unsigned long long* d_fault = nullptr;  // debug builds: fault word of the bounds checks
  // optional phase timing with events on the launching stream:
  // [0] work-list build, [1] class kernels, [2] expansion
  bool profiling = false;
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  std::vector<cudaEvent_t> blk_ev;  // per class-block launch (profiling level 2), launch order
  int profile_level = 0;
  std::vector<int> launch_order;    // class blocks, largest estimated cost first
  std::vector<cudaStream_t> aux;    // concurrent class-block streams
  int n_streams = kAuxStreams;      // how many of them the class blocks are spread over
  std::vector<cudaEvent_t> join;
  cudaEvent_t fork = nullptr;
  // host-output streaming: staging slabs on the device, copied out on their own stream
  double* d_stage = nullptr;
  size_t stage_elems = 0;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t stage_ready[kStageBuffers] = {};
  cudaEvent_t stage_free[kStageBuffers] = {};
  std::vector<std::pair<void*, size_t>> dev_allocs;  // every device block the basis holds
  // two-electron operator of the integral runs (0 = 1/r, 1 = erf(omega r)/r, 2 = erfc); the
  // Schwarz and mixed-form bounds stay Coulomb bounds, which bound both attenuated operators
  int potential = 0;
  double omega = 0.0;

  ~Basis();
  int alloc(void** p, size_t bytes, const char* what);
  void release(void* p);  // give one block back (to the process's block cache)
  int ensure_scratch(size_t compact_elems, size_t work_elems);
  int ensure_out(size_t elems);
};

int build_basis(Basis& B, int n, const int* angmom, const int* nprim, const double* center,
                const double* exps, const double* coefs, const int* nout, const int* sph,
                const int8_t* pos, const double* scl);
void boys_host_table(double* h);
int upload_basis(Basis& B);
int run_full(Basis& B, int notation, double tau, double* out, cudaStream_t st, double skip = 0.0,
             double fp32 = 0.0);
int run_full_host(Basis& B, int notation, double tau, double* out_host, cudaStream_t st);
int run_compact(Basis& B, double tau, cudaStream_t st, double skip = 0.0, double fp32 = 0.0);
int run_coulomb(Basis& B, const double* D, double tau, double* J, cudaStream_t st,
                double skip = 0.0, double fp32 = 0.0);
int run_jk(Basis& B, const double* D, double tau, double* J, double* K, cudaStream_t st);
int run_point_charge(Basis& B, int npoints, const double* coords, const double* charges,
                     int sum, double* out, cudaStream_t st);
int ensure_schwarz(Basis& B, cudaStream_t st);
// Debug builds (GBX_DEBUG_BOUNDS): waits for the call's work on `st` and returns
// GBX_ERR_INVALID naming the site and index of the first out-of-range access recorded in
// *d_fault (then cleared); release builds return GBX_OK at once.
int check_bounds_fault(unsigned long long* d_fault, cudaStream_t st, const char* what);
// Debug builds: a cleared fault word on the device (nullptr in release builds).
int alloc_fault_word(unsigned long long** d_fault);
int unique_values(Basis& B, long long n, const long long* idx4_host, double* out_host,
                  cudaStream_t st);
struct ExpandArgs;
int launch_expand_batch(int device, const ExpandArgs* d_mols, const long long* d_row_first,
                        int nmol, long long total_rows, size_t max_row_bytes, cudaStream_t st);
ExpandArgs make_expand_args(const Basis& B, int notation, double* out);
int num_sms_of(int device);
int launch_diagonal_bounds(const PairDev* pairs, int npairs, const ShellDev* shells,
                           const BlockDev* blocks, const double* compact, double* q,
                           cudaStream_t st);
int launch_class(int la, int lb, int lc, int ld, const EriLaunch& a, int grid, cudaStream_t st);
// GBX_WORK_ORDER=static: class kernels take their quartets in the static grid-stride order
// instead of from per-launch work counters (read once per process; a diagnostic)
bool static_work_order();

}  // namespace gbx
