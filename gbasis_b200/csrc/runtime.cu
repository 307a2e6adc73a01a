// Host runtime + C ABI of the ERI engine: basis packing, pair/class bookkeeping, device
// buffers, kernel launches (pair precompute, Schwarz/work-list compaction, class kernels,
// full-tensor expansion) and error reporting.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "gbx_eri.h"
#include "gbx_common.cuh"
#include "runtime.h"

namespace gbx {

// ------------------------------------------------------------------------- errors
static thread_local std::string g_last_error;

int set_error(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

const char* gbx_last_error_str() { return g_last_error.c_str(); }

int cuda_status(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return GBX_OK;
  if (e == cudaErrorMemoryAllocation)
    return set_error(GBX_ERR_OOM, "%s: %s", what, cudaGetErrorString(e));
  return set_error(GBX_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}

#define GBX_CUDA(call, what)                        \
  do {                                              \
    int _s = cuda_status((call), (what));           \
    if (_s != GBX_OK) return _s;                    \
  } while (0)

// ------------------------------------------------------------------ Boys table
// F_m(T) = e^{-T} sum_k (2T)^k / ((2m+1)(2m+3)...(2m+2k+1)): every term is positive, so
// the sum in long double is accurate to ~1e-18 relative for the whole grid.
static long double boys_series(int m, long double T) {
  long double term = 1.0L / (2 * m + 1), sum = term;
  for (int k = 1; k < 4000; ++k) {
    term *= 2.0L * T / (2 * m + 2 * k + 1);
    sum += term;
    if (term < sum * 1e-22L) break;
  }
  return expl(-T) * sum;
}

static std::mutex g_boys_mu;
static double* g_boys_dev[64] = {nullptr};

void boys_host_table(double* h) {
  for (int n = 0; n < kBoysNGrid; ++n) {
    const long double T = (long double)n / 10.0L;
    for (int m = 0; m < kBoysOrders; ++m)
      h[(size_t)n * (kBoysOrders + 1) + m] = (double)boys_series(m, T);
    h[(size_t)n * (kBoysOrders + 1) + kBoysOrders] = (double)expl(-T);
  }
}

int boys_table(int device, const double** out) {
  std::lock_guard<std::mutex> lk(g_boys_mu);
  if (device < 0 || device >= 64) return set_error(GBX_ERR_INVALID, "bad device %d", device);
  if (!g_boys_dev[device]) {
    std::vector<double> h((size_t)kBoysNGrid * (kBoysOrders + 1));
    boys_host_table(h.data());
    double* d = nullptr;
    GBX_CUDA(cudaMalloc(&d, h.size() * sizeof(double)), "cudaMalloc(boys table)");
    GBX_CUDA(cudaMemcpy(d, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice),
             "upload boys table");
    g_boys_dev[device] = d;
  }
  *out = g_boys_dev[device];
  return GBX_OK;
}

// ------------------------------------------------------------------ basis setup
// Conditioning of a pair's recursions when it is the bra: the vertical recursion builds
// angular momentum on A from the product centre P of each primitive pair, and its values grow
// like (|P - A| sqrt(zeta))^e while the results the horizontal recursion makes of them do not;
// a diffuse A primitive with a tight B primitive puts P near B.  The score is the largest
// |P - A| sqrt(zeta) = b |AB| / sqrt(a + b) over the primitive pairs pair_precompute keeps.
// Measured on 151 same-class (dd|dd) quartets of the batch workload against values summed
// primitive quartet by primitive quartet: the bra in the reference's order missed by up to
// 8.3e-7; the pair of smaller score as the bra by at most 2.6e-9, the best either order gives.
float pair_orient(const ShellDev& A, const ShellDev& Bs, const double* exps, double ab2) {
  const double ab = sqrt(ab2);
  const int keep0 = kept_primitive_pair(exps + A.prim_off, A.nprim, exps + Bs.prim_off, Bs.nprim, ab2);
  double sc = 0.0;
  for (int i = 0; i < A.nprim; ++i)
    for (int j = 0; j < Bs.nprim; ++j) {
      const double a = exps[A.prim_off + i], b = exps[Bs.prim_off + j];
      if (prim_pair_arg(a, b, ab2) > kPrimPairCut && i * Bs.nprim + j != keep0) continue;
      sc = std::max(sc, b * ab / sqrt(a + b));
    }
  return (float)sc;
}

struct DeviceGuard {
  int prev = -1;
  explicit DeviceGuard(int dev) {
    cudaGetDevice(&prev);
    if (prev != dev) cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    cudaGetDevice(&cur);
    if (prev >= 0 && cur != prev) cudaSetDevice(prev);
  }
};

// ------------------------------------------------------------ debug bounds checks
int check_bounds_fault(unsigned long long* d_fault, cudaStream_t st, const char* what) {
#if GBX_DEBUG_BOUNDS
  if (!d_fault) return GBX_OK;
  unsigned long long f = 0;
  GBX_CUDA(cudaStreamSynchronize(st), "bounds check: synchronize");
  GBX_CUDA(cudaMemcpy(&f, d_fault, sizeof(f), cudaMemcpyDeviceToHost), "bounds check: read");
  if (!f) return GBX_OK;
  GBX_CUDA(cudaMemset(d_fault, 0, sizeof(f)), "bounds check: clear");
  static const char* const sites[] = {"?", "class-kernel store", "work-list build", "zero fill",
                                      "expansion store", "compact-store read", "J/K scatter"};
  const unsigned site = (unsigned)(f >> 56);
  const unsigned long long idx = f & 0x00ffffffffffffffull;
  return set_error(GBX_ERR_INVALID, "%s: out-of-range index %llu at the %s", what, idx,
                   sites[site < 7 ? site : 0]);
#else
  (void)d_fault;
  (void)st;
  (void)what;
  return GBX_OK;
#endif
}

int alloc_fault_word(unsigned long long** d_fault) {
  *d_fault = nullptr;
#if GBX_DEBUG_BOUNDS
  GBX_CUDA(cudaMalloc((void**)d_fault, sizeof(unsigned long long)), "cudaMalloc(fault word)");
  GBX_CUDA(cudaMemset(*d_fault, 0, sizeof(unsigned long long)), "clear fault word");
#endif
  return GBX_OK;
}

// ------------------------------------------------------------------- block cache
// Device blocks a basis gives back are kept for the next basis in the process, up to
// kBlockCacheBytes per device: the public full-tensor call builds and drops a basis every time,
// and cudaFree (which waits for the whole device) plus cudaMalloc of the compact store and the
// staging slabs cost milliseconds per call.  A block is reused for a request of at least half
// its size.  gbx_release_cached_memory() frees the cache.
constexpr size_t kBlockCacheBytes = size_t(2) << 30;
struct CachedBlock {
  int device;
  void* p;
  size_t bytes;
};
static std::mutex g_block_mu;
static std::vector<CachedBlock> g_blocks;

static void* cache_take(int device, size_t bytes, size_t* got) {
  std::lock_guard<std::mutex> lk(g_block_mu);
  int best = -1;
  for (int i = 0; i < (int)g_blocks.size(); ++i) {
    const CachedBlock& b = g_blocks[i];
    if (b.device != device || b.bytes < bytes || b.bytes / 2 > bytes) continue;
    if (best < 0 || b.bytes < g_blocks[best].bytes) best = i;
  }
  if (best < 0) return nullptr;
  void* p = g_blocks[best].p;
  *got = g_blocks[best].bytes;
  g_blocks.erase(g_blocks.begin() + best);
  return p;
}

// The caller has made sure no work on the device still uses p.
static void cache_give(int device, void* p, size_t bytes) {
  if (!p) return;
  {
    std::lock_guard<std::mutex> lk(g_block_mu);
    size_t held = 0;
    for (const CachedBlock& b : g_blocks)
      if (b.device == device) held += b.bytes;
    if (held + bytes <= kBlockCacheBytes) {
      g_blocks.push_back({device, p, bytes});
      return;
    }
  }
  cudaFree(p);
}

Basis::~Basis() {
  // A basis that never allocated device memory nor created a stream or event (host
  // bookkeeping only, as the allocation-free entry point uses it) touches no device state
  // here: no device switch and no device-wide synchronisation.
  bool owns = !dev_allocs.empty() || fork || copy_stream || !aux.empty() || !join.empty() ||
              !blk_ev.empty();
  for (cudaEvent_t e : ev) owns = owns || e;
  for (cudaEvent_t e : stage_ready) owns = owns || e;
  for (cudaEvent_t e : stage_free) owns = owns || e;
  if (!owns) return;
  DeviceGuard g(device);
  // blocks go back to the cache only once nothing queued on the device can still use them
  // (what cudaFree would have waited for)
  if (cudaDeviceSynchronize() == cudaSuccess) {
    for (auto& a : dev_allocs) cache_give(device, a.first, a.second);
  } else {
    for (auto& a : dev_allocs) cudaFree(a.first);
  }
  for (cudaEvent_t& e : ev)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t& e : blk_ev)
    if (e) cudaEventDestroy(e);
  for (cudaStream_t& x : aux)
    if (x) cudaStreamDestroy(x);
  for (cudaEvent_t& e : join)
    if (e) cudaEventDestroy(e);
  if (fork) cudaEventDestroy(fork);
  for (cudaEvent_t& e : stage_ready)
    if (e) cudaEventDestroy(e);
  for (cudaEvent_t& e : stage_free)
    if (e) cudaEventDestroy(e);
  if (copy_stream) cudaStreamDestroy(copy_stream);
}

int Basis::alloc(void** p, size_t bytes, const char* what) {
  if (bytes == 0) bytes = 16;
  size_t got = 0;
  *p = cache_take(device, bytes, &got);
  if (!*p) {
    GBX_CUDA(cudaMalloc(p, bytes), what);
    got = bytes;
  }
  dev_allocs.push_back({*p, got});
  return GBX_OK;
}

void Basis::release(void* p) {
  for (size_t i = 0; i < dev_allocs.size(); ++i) {
    if (dev_allocs[i].first != p) continue;
    // the block may still be read by queued work of this basis: wait for the device, as
    // cudaFree would
    if (cudaDeviceSynchronize() == cudaSuccess) cache_give(device, p, dev_allocs[i].second);
    else cudaFree(p);
    dev_allocs.erase(dev_allocs.begin() + i);
    return;
  }
}

int Basis::ensure_scratch(size_t compact_elems, size_t work_elems) {
  if (compact_elems > compact_cap) {
    if (d_compact) {
      release(d_compact);
      d_compact = nullptr;
    }
    int s = alloc((void**)&d_compact, compact_elems * sizeof(double), "cudaMalloc(compact store)");
    if (s) return s;
    compact_cap = compact_elems;
  }
  (void)work_elems;
  return GBX_OK;
}

int Basis::ensure_out(size_t elems) {
  if (elems <= out_cap) return GBX_OK;
  if (d_out) {
    release(d_out);
    d_out = nullptr;
    out_cap = 0;
  }
  int s = alloc((void**)&d_out, elems * sizeof(double), "cudaMalloc(full tensor)");
  if (s) return s;
  out_cap = elems;
  return GBX_OK;
}

int build_basis(Basis& B, int n, const int* angmom, const int* nprim, const double* center,
                       const double* exps, const double* coefs, const int* nout, const int* sph,
                       const int8_t* pos, const double* scl) {
  NvtxRange range("gbx build basis");
  B.shells.resize(n);
  int prim_total = 0, func = 0;
  for (int s = 0; s < n; ++s) {
    if (angmom[s] < 0) return set_error(GBX_ERR_INVALID, "shell %d: negative angmom", s);
    if (angmom[s] > B.lmax_supported)
      return set_error(GBX_ERR_UNSUPPORTED,
                       "shell %d: angular momentum %d above the compiled maximum %d", s,
                       angmom[s], B.lmax_supported);
    if (nprim[s] <= 0) return set_error(GBX_ERR_INVALID, "shell %d: no primitives", s);
    const int nint = (sph[s] && angmom[s] >= 2) ? 2 * angmom[s] + 1 : ncart(angmom[s]);
    if (nout[s] != nint)
      return set_error(GBX_ERR_INVALID, "shell %d: nout %d, expected %d", s, nout[s], nint);
    ShellDev& d = B.shells[s];
    memset(&d, 0, sizeof(d));
    d.x = center[3 * s];
    d.y = center[3 * s + 1];
    d.z = center[3 * s + 2];
    d.l = angmom[s];
    d.nprim = nprim[s];
    d.prim_off = prim_total;
    d.nout = nout[s];
    d.func_off = func;
    d.sph = sph[s] ? 1 : 0;
    for (int c = 0; c < kMaxCart; ++c) {
      d.scl[c] = scl[kMaxCart * s + c];
      d.pos[c] = pos[kMaxCart * s + c];
    }
    for (int c = 0; c < nint; ++c)
      if (d.pos[c] < 0 || d.pos[c] >= nout[s])
        return set_error(GBX_ERR_INVALID, "shell %d: component %d maps outside the shell", s, c);
    for (int k = 0; k < nprim[s]; ++k)
      if (!(exps[prim_total + k] > 0.0))
        return set_error(GBX_ERR_INVALID, "shell %d: exponents must be positive", s);
    prim_total += nprim[s];
    func += nout[s];
  }
  B.nbf = func;
  B.h_exps.assign(exps, exps + prim_total);
  B.h_coefs.assign(coefs, coefs + prim_total);

  // pairs: i <= j, stored with the shell of larger maximum exponent first (the vertical
  // recursion runs on it: P - A stays small, which keeps the Obara-Saika and transfer
  // recursions from cancelling digits on diffuse partners); ties: higher l, lower index.
  // Sorted by (class, nprim desc).
  struct HP {
    int a, b, cls, nprim, i, j;
  };
  std::vector<double> emax(n, 0.0);
  for (int s2 = 0, off = 0; s2 < n; off += nprim[s2], ++s2)
    for (int k = 0; k < nprim[s2]; ++k) emax[s2] = std::max(emax[s2], exps[off + k]);
  std::vector<HP> hp;
  hp.reserve((size_t)n * (n + 1) / 2);
  for (int i = 0; i < n; ++i)
    for (int j = i; j < n; ++j) {
      int a = i, b = j;
      if (emax[j] > emax[i] || (emax[j] == emax[i] && angmom[j] > angmom[i])) std::swap(a, b);
      hp.push_back({a, b, pair_class_index(angmom[a], angmom[b]), nprim[a] * nprim[b], i, j});
    }
  std::stable_sort(hp.begin(), hp.end(), [](const HP& x, const HP& y) {
    if (x.cls != y.cls) return x.cls < y.cls;
    return x.nprim > y.nprim;
  });
  const int np = (int)hp.size();
  B.pairs.resize(np);
  B.pair_of.assign((size_t)n * n, -1);
  B.class_first.assign(kNumPairClasses + 1, 0);
  B.class_count.assign(kNumPairClasses, 0);
  B.class_funcs.assign(kNumPairClasses, 0);
  long long prim_pairs = 0;
  for (int p = 0; p < np; ++p) {
    const HP& h = hp[p];
    PairDev& d = B.pairs[p];
    memset(&d, 0, sizeof(d));
    d.shA = h.a;
    d.shB = h.b;
    d.prim_off = (int)prim_pairs;
    d.nprim = h.nprim;
    d.cls = h.cls;
    d.local = B.class_count[h.cls]++;
    d.fo = (int)B.class_funcs[h.cls];
    d.nB = B.shells[h.b].nout;
    B.class_funcs[h.cls] += (long long)B.shells[h.a].nout * B.shells[h.b].nout;
    d.ABx = B.shells[h.a].x - B.shells[h.b].x;
    d.ABy = B.shells[h.a].y - B.shells[h.b].y;
    d.ABz = B.shells[h.a].z - B.shells[h.b].z;
    d.orient = pair_orient(B.shells[h.a], B.shells[h.b], exps, d.ABx * d.ABx + d.ABy * d.ABy + d.ABz * d.ABz);
    prim_pairs += h.nprim;
    // orientation bit: 1 if the first function index of the ordered pair (i,j) lives
    // on the pair's B shell
    B.pair_of[(size_t)h.a * n + h.b] = p << 1;
    if (h.a != h.b) B.pair_of[(size_t)h.b * n + h.a] = (p << 1) | 1;
  }
  for (int c = 0; c < kNumPairClasses; ++c) B.class_first[c + 1] = B.class_first[c] + B.class_count[c];
  B.n_prim_pairs = prim_pairs;

  // class blocks (cb >= ck) that have quartets
  B.blocks.clear();
  B.block_table.assign((size_t)kNumPairClasses * kNumPairClasses, BlockDev{-1, 0, 0, 0});
  long long base = 0, work = 0;
  for (int cb = 0; cb < kNumPairClasses; ++cb)
    for (int ck = 0; ck <= cb; ++ck) {
      const long long nb = B.class_count[cb], nk = B.class_count[ck];
      if (nb == 0 || nk == 0) continue;
      HostBlock hb;
      hb.cb = cb;
      hb.ck = ck;
      hb.nb = nb;
      hb.nk = nk;
      hb.tri = (cb == ck);
      hb.ncand = hb.tri ? nb * (nb + 1) / 2 : nb * nk;
      hb.dev.base = base;
      hb.dev.ncols = B.class_funcs[ck];
      hb.dev.work_off = work;
      hb.dev.work_cap = hb.ncand;
      base += B.class_funcs[cb] * B.class_funcs[ck];
      work += hb.ncand;
      B.block_table[(size_t)cb * kNumPairClasses + ck] = hb.dev;
      B.blocks.push_back(hb);
    }
  B.compact_elems = base;
  B.n_quartets = work;
  // function-pair keys of the expansion: (class << 56) | (index in class << 32) | block row
  {
    std::vector<int> fsh(B.nbf), fcomp(B.nbf);
    for (int sh = 0; sh < n; ++sh)
      for (int c = 0; c < B.shells[sh].nout; ++c) {
        fsh[B.shells[sh].func_off + c] = sh;
        fcomp[B.shells[sh].func_off + c] = c;
      }
    B.h_ftab.resize((size_t)B.nbf * B.nbf);
    for (long long x = 0; x < B.nbf; ++x)
      for (long long y = 0; y < B.nbf; ++y) {
        const int pe = B.pair_of[(size_t)fsh[x] * n + fsh[y]];
        const PairDev& p = B.pairs[pe >> 1];
        const long long row = p.fo + ((pe & 1) ? (long long)fcomp[y] * p.nB + fcomp[x]
                                               : (long long)fcomp[x] * p.nB + fcomp[y]);
        B.h_ftab[(size_t)x * B.nbf + y] =
            ((long long)p.cls << 56) | ((long long)p.local << 32) | row;
      }
    // row-staged expansion: global pair-function index (class-major), the ordered function
    // pairs of each pair function and the pair each one belongs to
    B.pf_first.assign(kNumPairClasses + 1, 0);
    for (int c = 0; c < kNumPairClasses; ++c) B.pf_first[c + 1] = B.pf_first[c] + B.class_funcs[c];
    const long long npf = B.pf_first[kNumPairClasses];
    B.h_gtab.resize((size_t)B.nbf * B.nbf);
    B.h_rowinfo.assign((size_t)npf, make_int4(-1, -1, 0, 0));
    for (long long x = 0; x < B.nbf; ++x)
      for (long long y = 0; y < B.nbf; ++y) {
        const long long k = B.h_ftab[(size_t)x * B.nbf + y];
        const int cls = (int)(k >> 56);
        const long long g = B.pf_first[cls] + (k & 0xffffffffLL);
        B.h_gtab[(size_t)x * B.nbf + y] = (int)g;
        int4& ri = B.h_rowinfo[(size_t)g];
        if (ri.x < 0) {
          ri = make_int4((int)x, (int)y, 0, (int)((k >> 32) & 0xffffff));
        } else if (ri.x == (int)y && ri.y == (int)x) {
          ri.z = 1;  // (y, x) is the mirror of the stored ordered pair
        }
      }
  }
  // default lanes-per-quartet: about four primitive quartets per lane, fewer lanes when the
  // accumulator set (reduced across the team by shuffles) is large
  std::vector<double> cprims(kNumPairClasses, 0.0);
  for (const PairDev& p : B.pairs) cprims[p.cls] += p.nprim;
  for (int c = 0; c < kNumPairClasses; ++c)
    if (B.class_count[c]) cprims[c] /= (double)B.class_count[c];
  for (HostBlock& h : B.blocks) {
    h.avg_prims = cprims[h.cb] * cprims[h.ck];
    const int la = kPairClassL[h.cb][0], lb = kPairClassL[h.cb][1];
    const int lc = kPairClassL[h.ck][0], ld = kPairClassL[h.ck][1];
    int ne = 0, nf = 0;
    for (int e = la; e <= la + lb; ++e) ne += ncart(e);
    for (int f = lc; f <= lc + ld; ++f) nf += ncart(f);
    const int cap = ne * nf > 100 ? 2 : (ne * nf > 40 ? 8 : 32);
    int t = 1;
    while (t < cap && h.avg_prims / (2 * t) >= 4.0) t *= 2;
    h.team = t;
  }
  // launch order: estimated work, largest first
  std::vector<double> cost(B.blocks.size());
  for (size_t k = 0; k < B.blocks.size(); ++k) {
    const HostBlock& h = B.blocks[k];
    const int la = kPairClassL[h.cb][0], lb = kPairClassL[h.cb][1];
    const int lc = kPairClassL[h.ck][0], ld = kPairClassL[h.ck][1];
    cost[k] = (double)h.ncand * (h.avg_prims + 4.0) * ncart(la) * ncart(lb) * ncart(lc) * ncart(ld);
  }
  B.launch_order.resize(B.blocks.size());
  for (size_t k = 0; k < B.blocks.size(); ++k) B.launch_order[k] = (int)k;
  std::stable_sort(B.launch_order.begin(), B.launch_order.end(),
                   [&](int x, int y) { return cost[x] > cost[y]; });
  return GBX_OK;
}

}  // namespace gbx

using namespace gbx;

struct gbx_basis {
  std::unique_ptr<Basis> impl;
};

namespace gbx {
int coulomb_entry(gbx_basis* b, const double* D, double tau, double* J, cudaStream_t st,
                  double skip, double fp32) {
  Basis& B = *b->impl;
  DeviceGuard g(B.device);
  const int s = run_coulomb(B, D, tau, J, st, skip, fp32);
  return s ? s : check_bounds_fault(B.d_fault, st, "gbx_eri_coulomb_j");
}
int jk_entry(gbx_basis* b, const double* D, double tau, double* J, double* K, cudaStream_t st) {
  Basis& B = *b->impl;
  DeviceGuard g(B.device);
  const int s = run_jk(B, D, tau, J, K, st);
  return s ? s : check_bounds_fault(B.d_fault, st, "gbx_eri_jk");
}
int point_charge_entry(gbx_basis* b, int npoints, const double* coords, const double* charges,
                       int sum, double* out, cudaStream_t st) {
  Basis& B = *b->impl;
  DeviceGuard g(B.device);
  return run_point_charge(B, npoints, coords, charges, sum, out, st);
}
}  // namespace gbx

extern "C" {

int gbx_basis_set_potential(gbx_basis* b, int potential, double omega) {
  if (!b) return set_error(GBX_ERR_INVALID, "gbx_basis_set_potential: null basis");
  if (potential < 0 || potential > 2)
    return set_error(GBX_ERR_INVALID, "potential must be 0 (1/r), 1 (erf) or 2 (erfc), got %d",
                     potential);
  if (potential != 0 && !(omega > 0.0 && omega < 1e300))
    return set_error(GBX_ERR_INVALID, "omega must be a positive finite number for erf/erfc");
  b->impl->potential = potential;
  b->impl->omega = potential ? omega : 0.0;
  return GBX_OK;
}

int gbx_release_cached_memory(void) {
  std::vector<CachedBlock> blocks;
  {
    std::lock_guard<std::mutex> lk(g_block_mu);
    blocks.swap(g_blocks);
  }
  for (const CachedBlock& b : blocks) {
    DeviceGuard g(b.device);
    cudaFree(b.p);
  }
  return GBX_OK;
}

int gbx_debug_bounds(int* on) {
  if (!on) return set_error(GBX_ERR_INVALID, "gbx_debug_bounds: null argument");
  *on = GBX_DEBUG_BOUNDS ? 1 : 0;
  return GBX_OK;
}

int gbx_last_error(char* buf, size_t len) {
  if (!buf || len == 0) return GBX_ERR_INVALID;
  snprintf(buf, len, "%s", g_last_error.c_str());
  return GBX_OK;
}

int gbx_basis_create(gbx_basis** out, int n_shells, const int* angmom, const int* nprim,
                     const double* center, const double* exps, const double* coefs,
                     const int* nout, const int* sph, const int8_t* pos, const double* scl,
                     int device) {
  if (!out || n_shells <= 0 || !angmom || !nprim || !center || !exps || !coefs || !nout ||
      !sph || !pos || !scl)
    return set_error(GBX_ERR_INVALID, "gbx_basis_create: null argument or empty basis");
  *out = nullptr;
  int ndev = 0;
  GBX_CUDA(cudaGetDeviceCount(&ndev), "cudaGetDeviceCount");
  if (device < 0 || device >= ndev)
    return set_error(GBX_ERR_INVALID, "device %d not present (%d devices)", device, ndev);
  auto B = std::make_unique<Basis>();
  B->device = device;
  B->lmax_supported = compiled_lmax();
  int s = build_basis(*B, n_shells, angmom, nprim, center, exps, coefs, nout, sph, pos, scl);
  if (s) return s;
  DeviceGuard g(device);
  s = upload_basis(*B);
  if (s) return s;
  *out = new gbx_basis{std::move(B)};
  return GBX_OK;
}

int gbx_basis_destroy(gbx_basis* b) {
  delete b;
  return GBX_OK;
}

int gbx_basis_nbf(const gbx_basis* b, int64_t* nbf) {
  if (!b || !nbf) return set_error(GBX_ERR_INVALID, "gbx_basis_nbf: null argument");
  *nbf = b->impl->nbf;
  return GBX_OK;
}

int gbx_basis_stats(const gbx_basis* b, int64_t* n_quartets, int64_t* compact_bytes) {
  if (!b) return set_error(GBX_ERR_INVALID, "gbx_basis_stats: null basis");
  if (n_quartets) *n_quartets = b->impl->n_quartets;
  if (compact_bytes) *compact_bytes = b->impl->compact_elems * (int64_t)sizeof(double);
  return GBX_OK;
}

int gbx_eri_full(gbx_basis* b, int notation, double tau, double* out, void* stream) {
  if (!b || !out) return set_error(GBX_ERR_INVALID, "gbx_eri_full: null argument");
  if (notation != GBX_CHEMIST && notation != GBX_PHYSICIST)
    return set_error(GBX_ERR_INVALID, "notation must be GBX_CHEMIST or GBX_PHYSICIST");
  if (!(tau >= 0.0)) return set_error(GBX_ERR_INVALID, "schwarz threshold must be >= 0");
  Basis& B = *b->impl;
  DeviceGuard g(B.device);
  const int s = run_full(B, notation, tau, out, (cudaStream_t)stream);
  return s ? s : check_bounds_fault(B.d_fault, (cudaStream_t)stream, "gbx_eri_full");
}

int gbx_eri_full_mixed(gbx_basis* b, int notation, double skip, double fp32, double* out,
                       void* stream) {
  if (!b || !out) return set_error(GBX_ERR_INVALID, "gbx_eri_full_mixed: null argument");
  if (notation != GBX_CHEMIST && notation != GBX_PHYSICIST)
    return set_error(GBX_ERR_INVALID, "notation must be GBX_CHEMIST or GBX_PHYSICIST");
  if (!(skip >= 0.0) || !(fp32 >= 0.0))
    return set_error(GBX_ERR_INVALID, "thresholds must be >= 0");
  Basis& B = *b->impl;
  DeviceGuard g(B.device);
  const int s = run_full(B, notation, 0.0, out, (cudaStream_t)stream, skip, fp32);
  return s ? s : check_bounds_fault(B.d_fault, (cudaStream_t)stream, "gbx_eri_full_mixed");
}

int gbx_eri_unique(gbx_basis* b, double skip, double fp32, void* stream) {
  if (!b) return set_error(GBX_ERR_INVALID, "gbx_eri_unique: null basis");
  if (!(skip >= 0.0) || !(fp32 >= 0.0))
    return set_error(GBX_ERR_INVALID, "thresholds must be >= 0");
  Basis& B = *b->impl;
  DeviceGuard g(B.device);
  const int s = run_compact(B, 0.0, (cudaStream_t)stream, skip, fp32);
  return s ? s : check_bounds_fault(B.d_fault, (cudaStream_t)stream, "gbx_eri_unique");
}

int gbx_compact_view(gbx_basis* b, const double** dev_ptr, int64_t* n_elems) {
  if (!b || !dev_ptr || !n_elems) return set_error(GBX_ERR_INVALID, "gbx_compact_view: null argument");
  const Basis& B = *b->impl;
  *dev_ptr = B.d_compact;
  *n_elems = B.d_compact ? B.compact_elems : 0;
  return GBX_OK;
}

int gbx_unique_values(gbx_basis* b, int64_t n, const int64_t* idx4, double* out_host,
                      void* stream) {
  if (!b || n < 0 || (n > 0 && (!idx4 || !out_host)))
    return set_error(GBX_ERR_INVALID, "gbx_unique_values: null argument");
  Basis& B = *b->impl;
  DeviceGuard g(B.device);
  return unique_values(B, n, reinterpret_cast<const long long*>(idx4), out_host,
                       (cudaStream_t)stream);
}

int gbx_eri_full_host(gbx_basis* b, int notation, double tau, double* out_host, void* stream) {
  if (!b || !out_host) return set_error(GBX_ERR_INVALID, "gbx_eri_full_host: null argument");
  if (notation != GBX_CHEMIST && notation != GBX_PHYSICIST)
    return set_error(GBX_ERR_INVALID, "notation must be GBX_CHEMIST or GBX_PHYSICIST");
  if (!(tau >= 0.0)) return set_error(GBX_ERR_INVALID, "schwarz threshold must be >= 0");
  Basis& B = *b->impl;
  DeviceGuard g(B.device);
  const int s = run_full_host(B, notation, tau, out_host, (cudaStream_t)stream);
  return s ? s : check_bounds_fault(B.d_fault, (cudaStream_t)stream, "gbx_eri_full_host");
}

int gbx_schwarz_bounds(gbx_basis* b, double* q_host) {
  if (!b || !q_host) return set_error(GBX_ERR_INVALID, "gbx_schwarz_bounds: null argument");
  Basis& B = *b->impl;
  DeviceGuard g(B.device);
  int s = ensure_schwarz(B, nullptr);
  if (s) return s;
  const int n = (int)B.shells.size();
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < n; ++j) {
      const int pe = B.pair_of[(size_t)i * n + j];
      q_host[(size_t)i * n + j] = B.h_q[pe >> 1];
    }
  return GBX_OK;
}

int gbx_set_profiling(gbx_basis* b, int on) {
  if (!b) return set_error(GBX_ERR_INVALID, "gbx_set_profiling: null basis");
  Basis& B = *b->impl;
  DeviceGuard g(B.device);
  if (on && !B.ev[0])
    for (cudaEvent_t& e : B.ev) GBX_CUDA(cudaEventCreate(&e), "cudaEventCreate");
  if (on && B.blk_ev.empty()) {
    B.blk_ev.resize(B.blocks.size() + 1);
    for (cudaEvent_t& e : B.blk_ev) GBX_CUDA(cudaEventCreate(&e), "cudaEventCreate");
  }
  B.profiling = on != 0;
  B.profile_level = on;
  return GBX_OK;
}

int gbx_phase_times(gbx_basis* b, double* ms) {
  if (!b || !ms) return set_error(GBX_ERR_INVALID, "gbx_phase_times: null argument");
  Basis& B = *b->impl;
  if (!B.profiling) return set_error(GBX_ERR_INVALID, "profiling is off for this basis");
  DeviceGuard g(B.device);
  GBX_CUDA(cudaEventSynchronize(B.ev[3]), "phase events");
  for (int i = 0; i < 3; ++i) {
    float t = 0.f;
    GBX_CUDA(cudaEventElapsedTime(&t, B.ev[i], B.ev[i + 1]), "phase elapsed time");
    ms[i] = t;
  }
  return GBX_OK;
}

int gbx_num_blocks(const gbx_basis* b, int* n) {
  if (!b || !n) return set_error(GBX_ERR_INVALID, "gbx_num_blocks: null argument");
  *n = (int)b->impl->blocks.size();
  return GBX_OK;
}

int gbx_block_info(const gbx_basis* b, int k, int* cls4, int* team, double* avg_prims,
                   int64_t* n_quartets) {
  if (!b) return set_error(GBX_ERR_INVALID, "gbx_block_info: null basis");
  const Basis& B = *b->impl;
  if (k < 0 || k >= (int)B.blocks.size()) return set_error(GBX_ERR_INVALID, "block %d out of range", k);
  const HostBlock& h = B.blocks[k];
  if (cls4) {
    cls4[0] = kPairClassL[h.cb][0];
    cls4[1] = kPairClassL[h.cb][1];
    cls4[2] = kPairClassL[h.ck][0];
    cls4[3] = kPairClassL[h.ck][1];
  }
  if (team) *team = h.team;
  if (avg_prims) *avg_prims = h.avg_prims;
  if (n_quartets) *n_quartets = B.counts_on_host ? h.j_computed : h.ncand;
  return GBX_OK;
}

int gbx_set_team(gbx_basis* b, int k, int team) {
  if (!b) return set_error(GBX_ERR_INVALID, "gbx_set_team: null basis");
  Basis& B = *b->impl;
  if (k < 0 || k >= (int)B.blocks.size()) return set_error(GBX_ERR_INVALID, "block %d out of range", k);
  if (team < 1 || team > 32 || (team & (team - 1)))
    return set_error(GBX_ERR_INVALID, "team must be a power of two in [1, 32]");
  B.blocks[k].team = team;
  return GBX_OK;
}

int gbx_set_block_config(gbx_basis* b, int k, int variant, int ctas_per_sm) {
  if (!b) return set_error(GBX_ERR_INVALID, "gbx_set_block_config: null basis");
  Basis& B = *b->impl;
  if (k < 0 || k >= (int)B.blocks.size()) return set_error(GBX_ERR_INVALID, "block %d out of range", k);
  if (variant < 0 || variant > 2) return set_error(GBX_ERR_INVALID, "variant must be 0, 1 or 2");
  if (ctas_per_sm < 1 || ctas_per_sm > 32)
    return set_error(GBX_ERR_INVALID, "ctas_per_sm must be in [1, 32]");
  B.blocks[k].variant = variant;
  B.blocks[k].ctas_per_sm = ctas_per_sm;
  return GBX_OK;
}

int gbx_basis_set_streams(gbx_basis* b, int n_streams) {
  if (!b) return set_error(GBX_ERR_INVALID, "gbx_basis_set_streams: null basis");
  if (n_streams < 1 || n_streams > kMaxAuxStreams)
    return set_error(GBX_ERR_INVALID, "n_streams must be in [1, %d]", kMaxAuxStreams);
  b->impl->n_streams = n_streams;
  return GBX_OK;
}

int gbx_block_times(gbx_basis* b, double* ms, int n) {
  if (!b || !ms) return set_error(GBX_ERR_INVALID, "gbx_block_times: null argument");
  Basis& B = *b->impl;
  if (!B.profiling || B.blk_ev.empty())
    return set_error(GBX_ERR_INVALID, "profiling is off for this basis");
  if (n < (int)B.blocks.size()) return set_error(GBX_ERR_INVALID, "array too short");
  DeviceGuard g(B.device);
  GBX_CUDA(cudaEventSynchronize(B.blk_ev.back()), "block events");
  if (B.profile_level < 2) return set_error(GBX_ERR_INVALID, "per-block timing needs level 2");
  for (size_t i = 0; i < B.blocks.size(); ++i) {
    float t = 0.f;
    GBX_CUDA(cudaEventElapsedTime(&t, B.blk_ev[i], B.blk_ev[i + 1]), "block elapsed time");
    ms[B.launch_order.empty() ? i : B.launch_order[i]] = t;
  }
  return GBX_OK;
}

int gbx_basis_set_groups(gbx_basis* b, const int* group) {
  if (!b || !group) return set_error(GBX_ERR_INVALID, "gbx_basis_set_groups: null argument");
  Basis& B = *b->impl;
  const int n = (int)B.shells.size();
  B.group.assign(group, group + n);
  for (int i = 0; i < n; ++i)
    if (group[i] < 0) return set_error(GBX_ERR_INVALID, "negative shell group");
  B.schwarz_ready = false;
  return GBX_OK;
}

int gbx_last_counts(const gbx_basis* b, int64_t* computed, int64_t* screened) {
  if (!b) return set_error(GBX_ERR_INVALID, "gbx_last_counts: null basis");
  Basis& B = *b->impl;
  if (B.counts_on_host) {
    if (computed) *computed = B.last_computed;
    if (screened) *screened = B.last_screened;
    return GBX_OK;
  }
  int64_t n64 = 0, n32 = 0, nleft = 0;
  int s = gbx_mixed_counts(b, &n64, &n32, &nleft);
  if (s) return s;
  if (computed) *computed = n64 + n32;
  if (screened) *screened = B.n_quartets - n64 - n32;
  return GBX_OK;
}

int gbx_basis_set_fp32_lists(gbx_basis* b, int64_t min_quartets, int64_t share) {
  if (!b || min_quartets < 0 || share < 1)
    return set_error(GBX_ERR_INVALID, "gbx_basis_set_fp32_lists: need min >= 0 and share >= 1");
  Basis& B = *b->impl;
  B.fp32_min = min_quartets;
  B.fp32_share = share;
  B.mix_n32.clear();  // recount the lists at the next mixed call
  return GBX_OK;
}

int gbx_mixed_counts(const gbx_basis* b, int64_t* n_fp64, int64_t* n_fp32, int64_t* n_left_out) {
  if (!b) return set_error(GBX_ERR_INVALID, "gbx_mixed_counts: null basis");
  Basis& B = *b->impl;
  if (n_fp64) *n_fp64 = 0;
  if (n_fp32) *n_fp32 = 0;
  if (n_left_out) *n_left_out = 0;
  if (!B.d_counts) return GBX_OK;  // no compact-store call yet
  DeviceGuard g(B.device);
  const int nblk = (int)B.blocks.size();
  std::vector<int> c(nblk), c32(nblk, 0);
  GBX_CUDA(cudaMemcpy(c.data(), B.d_counts, nblk * sizeof(int), cudaMemcpyDeviceToHost),
           "read quartet counters");
  if (B.last_mixed && B.d_counts32)
    GBX_CUDA(cudaMemcpy(c32.data(), B.d_counts32, nblk * sizeof(int), cudaMemcpyDeviceToHost),
             "read FP32 quartet counters");
  long long t64 = 0, t32 = 0;
  for (int k = 0; k < nblk; ++k) {
    t64 += c[k];
    t32 += c32[k];
  }
  if (n_fp64) *n_fp64 = t64;
  if (n_fp32) *n_fp32 = t32;
  // left out: every quartet not computed (the mixed form's skip, or a Schwarz threshold)
  if (n_left_out) *n_left_out = B.n_quartets - t64 - t32;
  return GBX_OK;
}

}  // extern "C"
