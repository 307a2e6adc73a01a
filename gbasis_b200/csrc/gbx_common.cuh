// Device data layout of the ERI engine (shared by all kernels and the C-ABI runtime).
//
// Terms: a "shell" here is a segmented contraction (one column m of a gbasis
// GeneralizedContractionShell's coefficient matrix); a "pair" is an unordered pair of
// shells stored with its higher-l shell first (A, then B); a "pair class" is (lA, lB);
// a "class block" is the set of quartets (bra pair p, ket pair q) with
// class(p) >= class(q), stored as a dense matrix of pair functions
// rows = sum over pairs p of class(p) of nout(A_p)*nout(B_p), cols likewise for class(q).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace gbx {

constexpr int kLMax = 3;          // highest shell angular momentum the engine handles
constexpr int kMaxCart = 10;      // (kLMax+1)(kLMax+2)/2
constexpr int kBoysNGrid = 401;   // T_n = n / 10, n = 0..400
constexpr double kBoysStep = 0.1;
constexpr double kBoysTMax = 40.0;  // F_m(T) for T >= kBoysTMax by the asymptotic form
constexpr int kBoysTaylor = 8;      // Taylor terms around the nearest grid point (|dT| <= 0.05)
constexpr int kBoysMMax = 4 * kLMax + 1;  // highest Boys order any class needs (+1 spare)
constexpr int kBoysOrders = kBoysMMax + kBoysTaylor;  // orders stored in the global table

__host__ __device__ constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }

// Pair classes are ordered pair types (lA, lB), A being the shell the vertical recursion runs
// on (the one with the larger exponent, for numerical stability), sorted by
// (lA + lB, max(lA, lB), lA).  A quartet's bra is the pair with the larger class index.
constexpr int kNumPairClasses = (kLMax + 1) * (kLMax + 1);
constexpr int kPairClassL[kNumPairClasses][2] = {
    {0, 0}, {0, 1}, {1, 0}, {1, 1}, {0, 2}, {2, 0}, {1, 2}, {2, 1},
    {0, 3}, {3, 0}, {2, 2}, {1, 3}, {3, 1}, {2, 3}, {3, 2}, {3, 3}};
constexpr int pair_class_index(int la, int lb) {
  for (int c = 0; c < kNumPairClasses; ++c)
    if (kPairClassL[c][0] == la && kPairClassL[c][1] == lb) return c;
  return -1;
}

// One shell (segmented contraction).  `pos` / `scl` map the engine's internal component
// index (canonical Cartesian order, or for spherical shells with l >= 2 the canonical
// real-solid-harmonic order s_l..s_1, c_0..c_l) to the output function index inside the
// shell and its scale (norm_cont, Cartesian component norm or sign of the label).
struct ShellDev {
  double x, y, z;
  int l, nprim, prim_off, nout;
  int func_off, sph, pad0, pad1;
  double scl[kMaxCart];
  int8_t pos[kMaxCart];
  int8_t pad2[6];
};

// One primitive pair of a shell pair: zeta = a+b, P, X = P - A (A = first shell of the
// pair), C = c_a c_b N_a N_b exp(-ab/zeta |AB|^2) * sqrt(2) pi^{5/4} / zeta.
struct __align__(16) PrimPair {
  double zeta, izeta, Px, Py, Pz, Xx, Xy, Xz, C, pad;
};

struct PairDev {
  int shA, shB, prim_off, nprim;
  int cls, local, fo, nB;  // class, index within class, pair-function offset in class, nout(B)
  double ABx, ABy, ABz;
  int mol;                 // molecule of the pair in a batch (0 for a single basis)
  // conditioning of the recursions run from this pair as the bra: the largest |P - A|
  // sqrt(zeta) over its kept primitive pairs (0 for a one-centre pair); see pair_orient()
  float orient;
};

// Primitive pairs whose product factor exp(-ab/zeta |AB|^2) is below e^{-69} (1e-30) are left
// out of the primitive-pair lists (pair_precompute), except the pair's one of smallest argument.
constexpr double kPrimPairCut = 69.0;

// ab/(a+b) |AB|^2: the one expression for the product factor's argument, host and device.
__host__ __device__ inline double prim_pair_arg(double a, double b, double ab2) {
  return a * b / (a + b) * ab2;
}

// Index ia * nb + ib of the primitive pair of smallest argument (the first one on ties).
__host__ __device__ inline int kept_primitive_pair(const double* ea, int na, const double* eb,
                                                   int nb, double ab2) {
  double xmin = 0.0;
  int best = 0;
  for (int i = 0; i < na; ++i)
    for (int j = 0; j < nb; ++j) {
      const double x = prim_pair_arg(ea[i], eb[j], ab2);
      if ((i == 0 && j == 0) || x < xmin) {
        xmin = x;
        best = i * nb + j;
      }
    }
  return best;
}

// A quartet of a diagonal class block (bra and ket pairs of one class, lA + lB >= 3:
// block_orients) runs with either pair as the bra: the one whose recursions are better
// conditioned (smaller `orient`).  Its values
// belong to the block's entry whose row pair has the larger index in the class, so a quartet
// run with the other pair as the bra stores them transposed.
__device__ __forceinline__ bool quartet_transposed(const PairDev& P, const PairDev& Q) {
  return P.cls == Q.cls && P.local < Q.local;
}

// Per class block: where its quartets live in the work list and in the compact store.
struct BlockDev {
  long long base;   // element offset of the block matrix in the compact store
  long long ncols;  // pair functions of the ket class
  long long work_off, work_cap;
};

// Arguments of one class kernel launch.
struct EriLaunch {
  const int2* work;         // (bra pair, ket pair) per quartet of this block
  const int* work_count;    // device counter (screened count) or nullptr
  long long work_off, nwork;  // nwork = capacity; actual count read from work_count
  const PairDev* pairs;
  const PrimPair* prims;
  const ShellDev* shells;
  const double* boys_tab;   // [kBoysNGrid][kBoysOrders + 1], last column e^{-T_n}
  double* out;              // compact store
  long long base, ncols;
  int mode;                 // 0 = write block, 1 = Schwarz diagonal (max |.| -> qout)
  int team;                 // lanes per quartet in the register kernel (1..32, power of two)
  int fp32;                 // register kernel: 1 = FP32 recursions (mixed form)
  int reverse;              // quartet w is work[work_off + nwork - 1 - w] (FP32 list)
  // mode 2 (Coulomb matrix): J[a][b] += sum_cd (ab|cd) D[c][d] over the unique quartets
  const double* D;          // nbf x nbf, symmetric
  double* J;                // nbf x nbf, accumulated with atomics
  long long nbf;
  double* qout;             // per-pair Schwarz value (mode 1)
  int* status;              // device error flag
  // batch of molecules: the block's base and column count in each molecule's compact store,
  // indexed by PairDev::mol (nullptr: base / ncols above)
  const long long* mol_base;
  const long long* mol_ncols;
  // two-electron operator: 0 = 1/r, 1 = erf(omega r)/r, 2 = erfc(omega r)/r
  int potential;
  double omega;
  // heavy classes that have both kernels: 0 = split register kernel, 1 = line kernel
  int variant;
  // work counter of this launch, zero before it starts: in the heavy-class kernels warps (split
  // kernel: CTAs) take their next quartets from it with atomicAdd, so that a CTA that becomes
  // resident late (class blocks share the GPU with other blocks on other streams) takes less
  // work.  nullptr, and in the light-class register kernel: the static order, quartet w to
  // warp w mod (warps in the grid).
  unsigned long long* ticket;
  // debug builds (GBX_DEBUG_BOUNDS): fault word of the call and the length of `out` in
  // elements (mode 0 stores); nullptr: this launch's stores are not checked
  unsigned long long* fault;
  long long out_len;
};

// Next work ticket of a warp (every lane of the warp calls it; lane 0 draws).
__device__ __forceinline__ long long warp_ticket(unsigned long long* t, int lane) {
  unsigned long long v = 0;
  if (lane == 0) v = atomicAdd(t, 1ull);
  return (long long)__shfl_sync(0xffffffffu, v, 0);
}

// ----------------------------------------------------------------- debug bounds checks
// Builds compiled with -DGBX_DEBUG_BOUNDS=1 (libgbx_eri_debug.so) check the index of every
// store of the class kernels, the work-list build, the zero fill, the expansions and the J / K
// scatter, and of the expansions' compact-store reads, against the array it addresses.  An
// index outside it is recorded in the call's fault word (the first one: site in the top byte,
// index below) and the access is skipped; the entry point then returns GBX_ERR_INVALID naming
// both.  Release builds compile the checks away.  Launches given no fault word are unchecked.
#ifndef GBX_DEBUG_BOUNDS
#define GBX_DEBUG_BOUNDS 0
#endif
enum BoundsSite : int {
  kSiteClassStore = 1,   // class kernel store into the compact store
  kSiteWorkList = 2,     // work-list build (FP64, FP32 and zero lists)
  kSiteZeroFill = 3,     // zero_quartets
  kSiteExpand = 4,       // expansion store into the N^4 tensor (or a host-copy slab)
  kSiteCompactRead = 5,  // expansion / J-K read of the compact store
  kSiteJK = 6,           // Coulomb / exchange matrix scatter
};

__device__ __forceinline__ bool gbx_in_bounds(unsigned long long* fault, int site, long long i,
                                              long long n) {
#if GBX_DEBUG_BOUNDS
  if (!fault || (i >= 0 && i < n)) return true;
  const unsigned long long idx = i < 0 ? 0x00ffffffffffffffull : (unsigned long long)i;
  atomicCAS(fault, 0ull, ((unsigned long long)site << 56) | (idx & 0x00ffffffffffffffull));
  return false;
#else
  (void)fault;
  (void)site;
  (void)i;
  (void)n;
  return true;
#endif
}

// a.out[i] = v: a class kernel's store into the compact store.
__device__ __forceinline__ void out_store(const EriLaunch& a, long long i, double v) {
  if (gbx_in_bounds(a.fault, kSiteClassStore, i, a.out_len)) a.out[i] = v;
}

// J[i] += v: a Coulomb-mode contribution (J is nbf x nbf).
__device__ __forceinline__ void j_add(const EriLaunch& a, long long i, double v) {
  if (gbx_in_bounds(a.fault, kSiteJK, i, a.nbf * a.nbf)) atomicAdd(a.J + i, v);
}

// Destination block of a quartet whose bra pair is P.
__device__ __forceinline__ void block_dest(const EriLaunch& a, const PairDev& P, long long& base,
                                           long long& ncols) {
  if (a.mol_base) {
    base = a.mol_base[P.mol];
    ncols = a.mol_ncols[P.mol];
  } else {
    base = a.base;
    ncols = a.ncols;
  }
}

}  // namespace gbx
