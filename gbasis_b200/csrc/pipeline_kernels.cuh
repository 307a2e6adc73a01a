// Argument structs and declarations of the pipeline kernels defined in pipeline.cu.
#pragma once
#include "gbx_common.cuh"

namespace gbx {

// One class block of the work-list build (K2).
struct BuildBlock {
  int pb0, nb, pk0, nk;
  int tri, blk;
  long long work_off, ncand;
  int fp32_ok;  // the block's class kernel has an FP32 path (mixed form); 0: FP64 only
  int orient;   // diagonal block whose quartets run from the better-conditioned pair
};

// Full-tensor expansion (K6).
struct ExpandArgs {
  long long n;
  int nsh, notation;
  const int* fsh;
  const int* fcomp;
  const int* pair_of;
  const int4* pinfo;  // (cls, local, fo, nB)
  const BlockDev* blocks;
  const double* compact;
  double* out;
  // debug builds: fault word, the valid destination range [out_lo, out_lo + out_len) of the
  // launch (the tensor or a host-copy slab) and the compact store's length
  unsigned long long* fault;
  const double* out_lo;
  long long out_len, compact_len;
  const long long* ftab;  // n*n function-pair keys (class, pair index in class, block row)
  // row-staged form (expand_rows)
  const int* gtab;        // n*n: pair function (class-major index) of each ordered pair
  const int4* rowinfo;    // per pair function: (x, y, mirror, local pair index in class)
  long long npf;
  long long pf_first[kNumPairClasses + 1];
};

__global__ void pair_precompute(PairDev* __restrict__ pairs, int npairs,
                                const ShellDev* __restrict__ shells,
                                const double* __restrict__ exps, const double* __restrict__ coefs,
                                PrimPair* __restrict__ prims);
// Mixed form of the work-list build (counts32 == nullptr: FP64 only, nothing skipped).
struct MixedParams {
  const double* qm;  // per pair: Schwarz bound x largest output scale of its two shells
  double skip, fp32;
  int* counts32;
  const int* fp32_on;  // per block: 1 = FP32 list in use (nullptr: every block with an FP32 path)
  // left-out quartets (bound below skip) listed for zero_quartets, which clears only their
  // entries of the compact store; nullptr: they are dropped (the caller clears the store)
  int2* zero_work;
  int* zero_count;
  long long zero_cap;
  unsigned long long* fault;  // debug builds: the call's fault word (work-list indices)
};

__global__ void build_work(const int2* __restrict__ cta_map, const BuildBlock* __restrict__ bb,
                           const double* __restrict__ qs, double tau, int2* __restrict__ work,
                           int* __restrict__ counts, const MixedParams mp,
                           const PairDev* __restrict__ pairs);
__global__ void expand_full(const ExpandArgs e);
__global__ void expand_rows(const ExpandArgs e);
__global__ void build_work_range(const BuildBlock B, long long start, long long len,
                                 const double* __restrict__ qs, double tau,
                                 int2* __restrict__ work, int* __restrict__ count);

}  // namespace gbx
