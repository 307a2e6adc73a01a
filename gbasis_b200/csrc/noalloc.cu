// Allocation-free variant of the full-tensor call: gbx_eri_full_noalloc.
//
// Who needs it: callers that cannot call cudaMalloc while they run us.  Typical cases are
// processes whose device memory is owned by another allocator (frameworks that reserve
// most of the GPU up front, so a library's own cudaMalloc fails even though the work is
// small), and pipelines that cannot afford the device-wide synchronisation cudaFree
// implies.  They pass the basis (host arrays) and the output tensor (device memory they
// own); every intermediate this call needs — shell and pair records, primitive pairs, the
// Boys table, the quartet work list and its counters, the compact integral store — is
// carved out of one file-scope static device array of kNoAllocScratchBytes (64 MiB), which
// every GPU that loads this library holds until the process exits.
//
// Set-up: the first call on a device (with that device current) resolves the array's
// device address with cudaGetSymbolAddress; make that first call before any stream
// capture.  All calls share the one array and it keeps the previous call's contents, so the
// call rewrites every region it reads and clears its counters itself; calls that overlap on
// the GPU (different streams, or several host threads) race on it and must be serialised by
// the caller.  Bases whose working set does not fit are rejected with GBX_ERR_INVALID.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <vector>

#include "gbx_eri.h"
#include "pipeline_kernels.cuh"
#include "runtime.h"

namespace gbx {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(64) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mu;
void* g_noalloc_ptr[64] = {nullptr};
double g_boys_host[kBoysNGrid * (kBoysOrders + 1)];
bool g_boys_host_ready = false;

struct Carve {
  size_t off = 0;
  size_t take(size_t bytes) {
    const size_t o = (off + 255) & ~size_t(255);
    off = o + std::max<size_t>(bytes, 1);
    return o;
  }
};

}  // namespace
}  // namespace gbx

using namespace gbx;

extern "C" int gbx_eri_full_noalloc(int n_shells, const int* angmom, const int* nprim,
                                    const double* center, const double* exps,
                                    const double* coefs, const int* nout, const int* sph,
                                    const int8_t* pos, const double* scl, int notation,
                                    double* out, void* stream) {
  if (n_shells <= 0 || !angmom || !nprim || !center || !exps || !coefs || !nout || !sph ||
      !pos || !scl || !out)
    return set_error(GBX_ERR_INVALID, "gbx_eri_full_noalloc: null argument or empty basis");
  if (notation != GBX_CHEMIST && notation != GBX_PHYSICIST)
    return set_error(GBX_ERR_INVALID, "notation must be GBX_CHEMIST or GBX_PHYSICIST");
  int dev = 0;
  int s = cuda_status(cudaGetDevice(&dev), "cudaGetDevice");
  if (s) return s;
  if (dev < 0 || dev >= 64) return set_error(GBX_ERR_INVALID, "device %d out of range", dev);
  std::lock_guard<std::mutex> lk(g_noalloc_mu);

  // set-up, once per device: the device address of the static scratch array
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    s = cuda_status(cudaGetSymbolAddress(&p, g_noalloc_scratch), "cudaGetSymbolAddress(scratch)");
    if (s) return s;
    g_noalloc_ptr[dev] = p;
  }
  if (!g_boys_host_ready) {
    boys_host_table(g_boys_host);
    g_boys_host_ready = true;
  }
  unsigned char* base = static_cast<unsigned char*>(g_noalloc_ptr[dev]);

  // host bookkeeping (pairs, classes, blocks) exactly as for a basis handle
  Basis B;
  B.device = dev;
  B.lmax_supported = compiled_lmax();
  s = build_basis(B, n_shells, angmom, nprim, center, exps, coefs, nout, sph, pos, scl);
  if (s) return s;
  const int n = (int)B.shells.size();
  const int np = (int)B.pairs.size();
  const int nblk = (int)B.blocks.size();
  std::vector<int> fsh(B.nbf), fcomp(B.nbf);
  for (int sh = 0; sh < n; ++sh)
    for (int c = 0; c < B.shells[sh].nout; ++c) {
      fsh[B.shells[sh].func_off + c] = sh;
      fcomp[B.shells[sh].func_off + c] = c;
    }
  std::vector<BuildBlock> bb(nblk);
  std::vector<int2> cmap;
  for (int k = 0; k < nblk; ++k) {
    const HostBlock& h = B.blocks[k];
    bb[k] = BuildBlock{(int)B.class_first[h.cb], (int)h.nb, (int)B.class_first[h.ck], (int)h.nk,
                       h.tri ? 1 : 0, k, h.dev.work_off, h.ncand, 0,
                       block_orients(h.cb, h.ck) ? 1 : 0};
    for (long long c0 = 0; c0 < h.ncand; c0 += 256) cmap.push_back(make_int2(k, (int)c0));
  }
  std::vector<int4> pinfo(np);
  for (int p = 0; p < np; ++p)
    pinfo[p] = make_int4(B.pairs[p].cls, B.pairs[p].local, B.pairs[p].fo, B.pairs[p].nB);

  // carve the scratch array
  Carve cv;
  const size_t o_shells = cv.take(n * sizeof(ShellDev));
  const size_t o_pairs = cv.take(np * sizeof(PairDev));
  const size_t o_prims = cv.take(B.n_prim_pairs * sizeof(PrimPair));
  const size_t o_exps = cv.take(B.h_exps.size() * sizeof(double));
  const size_t o_coefs = cv.take(B.h_coefs.size() * sizeof(double));
  const size_t o_pair_of = cv.take((size_t)n * n * sizeof(int));
  const size_t o_fsh = cv.take(B.nbf * sizeof(int));
  const size_t o_fcomp = cv.take(B.nbf * sizeof(int));
  const size_t o_blocks = cv.take(B.block_table.size() * sizeof(BlockDev));
  const size_t o_bb = cv.take(nblk * sizeof(BuildBlock));
  const size_t o_cmap = cv.take(cmap.size() * sizeof(int2));
  const size_t o_pinfo = cv.take(np * sizeof(int4));
  const size_t o_counts = cv.take(nblk * sizeof(int));
  const size_t o_ftab = cv.take(B.h_ftab.size() * sizeof(long long));
  const size_t o_work = cv.take((size_t)B.n_quartets * sizeof(int2));
  const size_t o_boys = cv.take(sizeof(g_boys_host));
  const size_t o_compact = cv.take((size_t)B.compact_elems * sizeof(double));
  if (cv.off > kNoAllocScratchBytes)
    return set_error(GBX_ERR_INVALID,
                     "gbx_eri_full_noalloc: this basis needs %.1f MiB of device scratch; the "
                     "allocation-free entry point is limited to %zu MiB (use gbx_eri_full)",
                     cv.off / 1048576.0, kNoAllocScratchBytes >> 20);

  cudaStream_t st = (cudaStream_t)stream;
  auto up = [&](size_t off, const void* src, size_t bytes) {
    return bytes ? cuda_status(cudaMemcpyAsync(base + off, src, bytes, cudaMemcpyHostToDevice, st),
                               "upload to scratch")
                 : GBX_OK;
  };
  if ((s = up(o_shells, B.shells.data(), n * sizeof(ShellDev))) ||
      (s = up(o_pairs, B.pairs.data(), np * sizeof(PairDev))) ||
      (s = up(o_exps, B.h_exps.data(), B.h_exps.size() * sizeof(double))) ||
      (s = up(o_coefs, B.h_coefs.data(), B.h_coefs.size() * sizeof(double))) ||
      (s = up(o_pair_of, B.pair_of.data(), (size_t)n * n * sizeof(int))) ||
      (s = up(o_fsh, fsh.data(), B.nbf * sizeof(int))) ||
      (s = up(o_fcomp, fcomp.data(), B.nbf * sizeof(int))) ||
      (s = up(o_blocks, B.block_table.data(), B.block_table.size() * sizeof(BlockDev))) ||
      (s = up(o_bb, bb.data(), nblk * sizeof(BuildBlock))) ||
      (s = up(o_cmap, cmap.data(), cmap.size() * sizeof(int2))) ||
      (s = up(o_pinfo, pinfo.data(), np * sizeof(int4))) ||
      (s = up(o_boys, g_boys_host, sizeof(g_boys_host))) ||
      (s = up(o_ftab, B.h_ftab.data(), B.h_ftab.size() * sizeof(long long))))
    return s;
  // the previous call's counters are still in the array: clear them
  if ((s = cuda_status(cudaMemsetAsync(base + o_counts, 0, nblk * sizeof(int), st),
                       "clear counters")))
    return s;

  auto* d_shells = reinterpret_cast<ShellDev*>(base + o_shells);
  auto* d_pairs = reinterpret_cast<PairDev*>(base + o_pairs);
  auto* d_prims = reinterpret_cast<PrimPair*>(base + o_prims);
  auto* d_counts = reinterpret_cast<int*>(base + o_counts);
  auto* d_work = reinterpret_cast<int2*>(base + o_work);
  auto* d_compact = reinterpret_cast<double*>(base + o_compact);
  pair_precompute<<<(np + 127) / 128, 128, 0, st>>>(
      d_pairs, np, d_shells, reinterpret_cast<const double*>(base + o_exps),
      reinterpret_cast<const double*>(base + o_coefs), d_prims);
  if ((s = cuda_status(cudaGetLastError(), "pair_precompute launch"))) return s;
  build_work<<<(int)cmap.size(), 256, 0, st>>>(reinterpret_cast<const int2*>(base + o_cmap),
                                               reinterpret_cast<const BuildBlock*>(base + o_bb),
                                               nullptr, 0.0, d_work, d_counts,
                                               MixedParams{nullptr, 0.0, 0.0, nullptr},
                                               d_pairs);
  if ((s = cuda_status(cudaGetLastError(), "build_work launch"))) return s;
  int nsm = 1;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  for (int i = 0; i < nblk; ++i) {
    // largest blocks first, each with the default lanes per quartet of a basis handle
    const int k = B.launch_order.empty() ? i : B.launch_order[i];
    const HostBlock& h = B.blocks[k];
    EriLaunch a;
    memset(&a, 0, sizeof(a));
    a.work = d_work;
    a.work_count = d_counts + k;
    a.work_off = h.dev.work_off;
    a.nwork = h.ncand;
    a.pairs = d_pairs;
    a.prims = d_prims;
    a.shells = d_shells;
    a.boys_tab = reinterpret_cast<const double*>(base + o_boys);
    a.out = d_compact;
    a.base = h.dev.base;
    a.ncols = h.dev.ncols;
    a.mode = 0;
    a.team = h.team;
    const int grid = (int)std::max<long long>(
        1, std::min<long long>((h.ncand * h.team + 127) / 128, (long long)nsm * 8));
    if ((s = launch_class(kPairClassL[h.cb][0], kPairClassL[h.cb][1], kPairClassL[h.ck][0],
                          kPairClassL[h.ck][1], a, grid, st)))
      return s;
  }
  ExpandArgs e{};  // zeroed: no fault word (this call's stores are never bounds-checked)
  e.n = B.nbf;
  e.nsh = n;
  e.notation = notation;
  e.fsh = reinterpret_cast<const int*>(base + o_fsh);
  e.fcomp = reinterpret_cast<const int*>(base + o_fcomp);
  e.pair_of = reinterpret_cast<const int*>(base + o_pair_of);
  e.pinfo = reinterpret_cast<const int4*>(base + o_pinfo);
  e.blocks = reinterpret_cast<const BlockDev*>(base + o_blocks);
  e.compact = d_compact;
  e.out = out;
  e.ftab = reinterpret_cast<const long long*>(base + o_ftab);
  const long long rows = B.nbf * B.nbf * B.nbf;
  const int grid = (int)std::max<long long>(1, std::min<long long>((rows + 7) / 8, (long long)nsm * 16));
  expand_full<<<grid, 256, 0, st>>>(e);
  return cuda_status(cudaGetLastError(), "expand_full launch");
}
