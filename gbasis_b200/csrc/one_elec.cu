// Point-charge (nuclear-attraction) integrals V[a][b][c] = -q_c (a| 1/|r - R_c| |b).
//
// One thread per (shell pair, point charge): the primitive pairs of the shell pair are summed
// in registers, then the horizontal recursion, the transforms of spherical shells, the
// per-function scales (norm_cont, component norms) and the stores of the block and its
// transpose.  The primitive recursion is the class's generated (ab|ss) electron-repulsion
// recursion with the ket shrunk to the point: the Obara-Saika vertical recursion
//   [a+1_i]^(m) = PA_i [a]^(m) - PC_i [a]^(m+1) + a_i/(2 zeta) ([a-1_i]^(m) - [a-1_i]^(m+1))
// is the two-electron one with W - P = -(P - C) and rho/zeta = 1, and
// [0]^(m) = 2 pi / zeta exp(-ab/zeta |AB|^2) F_m(zeta |PC|^2) is the primitive pair's
// electron-repulsion prefactor times sqrt(2) pi^{-1/4}.
//
// Reference: gbasis/integrals/_one_elec_int.py:8-254 (recursions, norms, contraction),
// gbasis/integrals/point_charge.py:165-325 (sign, layout, dispatch),
// gbasis/integrals/nuclear_electron_attraction.py:8-42 (sum over the points).
#include <cstdio>

#include "eri_kernels.cuh"
#include "errors.h"
#include "gbx_eri.h"
#include "runtime.h"

#define GBX_CUDA(call, what)              \
  do {                                    \
    int _s = cuda_status((call), (what)); \
    if (_s != GBX_OK) return _s;          \
  } while (0)

namespace gbx {

struct PointArgs {
  const PairDev* pairs;
  const PrimPair* prims;
  const ShellDev* shells;
  const double* boys_tab;
  const double4* points;  // x, y, z, charge
  double* out;            // sum: nbf x nbf; else nbf x nbf x npoints
  long long nbf;
  int pair_first, npairs, npoints, sum;
};

template <int LA, int LB>
__global__ void __launch_bounds__(128) point_charge_block(const PointArgs a) {
  using C = gen::Cls<LA, LB, 0, 0>;
  constexpr int L = LA + LB;
  constexpr int NCA = ncart(LA), NCB = ncart(LB);
  // [0]^(m) prefactor over the electron-repulsion one stored in PrimPair::C:
  // (2 pi / zeta) / (sqrt(2) pi^{5/4} / zeta) = sqrt(2) pi^{-1/4}
  constexpr double kOneElec = 1.062251932027197;
  __shared__ double s_tab[kBoysNGrid * kBoysTaylor];
  __shared__ double s_exp[kBoysNGrid];
  stage_boys<L>(a.boys_tab, s_tab, s_exp);
  __syncthreads();
  const long long total = (long long)a.npairs * a.npoints;
  for (long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int p = a.pair_first + (int)(t / a.npoints);
    const int c = (int)(t % a.npoints);
    const PairDev P = a.pairs[p];
    const double4 pt = a.points[c];
    double acc[C::NE * C::NF];
#pragma unroll
    for (int i = 0; i < C::NE * C::NF; ++i) acc[i] = 0.0;
    for (int i = 0; i < P.nprim; ++i) {
      const PrimPair bp = a.prims[P.prim_off + i];
      const double PCx = bp.Px - pt.x, PCy = bp.Py - pt.y, PCz = bp.Pz - pt.z;
      const double T = bp.zeta * fma(PCx, PCx, fma(PCy, PCy, PCz * PCz));
      double F[L + 1];
      boys_eval<L>(T, s_tab, s_exp, F);
      const double pref = bp.C * kOneElec;
#pragma unroll
      for (int m = 0; m <= L; ++m) F[m] *= pref;
      C::template prim<double>(F, bp.Xx, bp.Xy, bp.Xz, -PCx, -PCy, -PCz, 0.5 * bp.izeta, 1.0,
                               0.0, 0.0, 0.0, 0.0, 0.0, acc);
    }
    double o[C::NAB * C::NCD];
    C::hrr(acc, P.ABx, P.ABy, P.ABz, 0.0, 0.0, 0.0, o);
    const ShellDev& sA = a.shells[P.shA];
    const ShellDev& sB = a.shells[P.shB];
    if (LB >= 2 && sB.sph) sph_axis<LB, NCA, 1>(o);
    if (LA >= 2 && sA.sph) sph_axis<LA, 1, NCB>(o);
    const int nAi = internal_count(sA), nBi = internal_count(sB);
    const double mq = -pt.w;
    const long long n = a.nbf;
#pragma unroll
    for (int ia = 0; ia < NCA; ++ia) {
      if (ia >= nAi) break;
      const long long fa = sA.func_off + sA.pos[ia];
      const double sa = sA.scl[ia] * mq;
#pragma unroll
      for (int ib = 0; ib < NCB; ++ib) {
        if (ib >= nBi) break;
        const long long fb = sB.func_off + sB.pos[ib];
        const double v = o[ia * NCB + ib] * sa * sB.scl[ib];
        if (a.sum) {
          atomicAdd(a.out + fa * n + fb, v);
          if (P.shA != P.shB) atomicAdd(a.out + fb * n + fa, v);
        } else {
          a.out[(fa * n + fb) * a.npoints + c] = v;
          if (P.shA != P.shB) a.out[(fb * n + fa) * a.npoints + c] = v;
        }
      }
    }
  }
}

template <int LA, int LB>
static int launch_pc(const PointArgs& a, int nsm, cudaStream_t st) {
  const long long total = (long long)a.npairs * a.npoints;
  const int grid = (int)std::max<long long>(1, std::min<long long>((total + 127) / 128, (long long)nsm * 8));
  point_charge_block<LA, LB><<<grid, 128, 0, st>>>(a);
  return cuda_status(cudaGetLastError(), "point_charge_block launch");
}

static int launch_pc_class(int la, int lb, const PointArgs& a, int nsm, cudaStream_t st) {
  switch (la * 4 + lb) {
#define GBX_PC(A, B) \
  case A * 4 + B:    \
    return launch_pc<A, B>(a, nsm, st);
    GBX_PC(0, 0) GBX_PC(0, 1) GBX_PC(0, 2) GBX_PC(0, 3)
    GBX_PC(1, 0) GBX_PC(1, 1) GBX_PC(1, 2) GBX_PC(1, 3)
    GBX_PC(2, 0) GBX_PC(2, 1) GBX_PC(2, 2) GBX_PC(2, 3)
    GBX_PC(3, 0) GBX_PC(3, 1) GBX_PC(3, 2) GBX_PC(3, 3)
#undef GBX_PC
    default:
      return set_error(GBX_ERR_UNSUPPORTED, "point charges: pair class (%d, %d)", la, lb);
  }
}

int run_point_charge(Basis& B, int npoints, const double* coords, const double* charges,
                     int sum, double* out, cudaStream_t st) {
  int s;
  const double* tab = nullptr;
  if ((s = boys_table(B.device, &tab))) return s;
  std::vector<double4> h(npoints);
  for (int i = 0; i < npoints; ++i)
    h[i] = make_double4(coords[3 * i], coords[3 * i + 1], coords[3 * i + 2], charges[i]);
  double4* d_pts = nullptr;
  if ((s = B.alloc((void**)&d_pts, (size_t)npoints * sizeof(double4), "cudaMalloc(point charges)")))
    return s;
  GBX_CUDA(cudaMemcpyAsync(d_pts, h.data(), (size_t)npoints * sizeof(double4),
                           cudaMemcpyHostToDevice, st), "copy point charges");
  const size_t out_elems = (size_t)B.nbf * B.nbf * (sum ? 1 : (size_t)npoints);
  if (sum) GBX_CUDA(cudaMemsetAsync(out, 0, out_elems * sizeof(double), st), "clear output");
  int dev = 0, nsm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  PointArgs a;
  a.pairs = B.d_pairs;
  a.prims = B.d_prims;
  a.shells = B.d_shells;
  a.boys_tab = tab;
  a.points = d_pts;
  a.out = out;
  a.nbf = B.nbf;
  a.npoints = npoints;
  a.sum = sum;
  for (int c = 0; c < kNumPairClasses; ++c) {
    if (B.class_count[c] == 0) continue;
    a.pair_first = (int)B.class_first[c];
    a.npairs = (int)B.class_count[c];
    if ((s = launch_pc_class(kPairClassL[c][0], kPairClassL[c][1], a, nsm, st))) return s;
  }
  // the points' buffer goes back once the kernels that read it are done
  GBX_CUDA(cudaStreamSynchronize(st), "point charges");
  B.release(d_pts);
  return GBX_OK;
}

int point_charge_entry(gbx_basis* b, int npoints, const double* coords, const double* charges,
                       int sum, double* out, cudaStream_t st);

}  // namespace gbx

extern "C" int gbx_point_charge(gbx_basis* b, int n_points, const double* coords,
                                const double* charges, int sum_points, double* out,
                                void* stream) {
  using namespace gbx;
  if (!b || !coords || !charges || !out)
    return set_error(GBX_ERR_INVALID, "gbx_point_charge: null argument");
  if (n_points <= 0) return set_error(GBX_ERR_INVALID, "gbx_point_charge: no point charges");
  for (int i = 0; i < 4 * n_points; ++i) {
    const double v = i < 3 * n_points ? coords[i] : charges[i - 3 * n_points];
    if (!(v == v) || v - v != 0.0)
      return set_error(GBX_ERR_INVALID, "gbx_point_charge: coordinates and charges must be finite");
  }
  return point_charge_entry(b, n_points, coords, charges, sum_points ? 1 : 0, out,
                            (cudaStream_t)stream);
}
