// Device Boys values on caller-given arguments: gbx_boys_eval.
//
// The class kernels evaluate F_0..F_L(T) with boys_eval<L> (eri_kernels.cuh) from the
// shared-memory Taylor table; this entry point runs exactly that device function on a list
// of arguments so that it can be checked on its own against F_m(T) = 1F1(m+1/2; m+3/2; -T)
// / (2m+1) (gbasis/integrals/boys_functions.py:26-63), across the switch from the tabulated
// Taylor expansion to the asymptotic form at T = kBoysTMax.
#include <cmath>
#include <vector>

#include "eri_kernels.cuh"
#include "gbx_eri.h"
#include "runtime.h"

namespace gbx {
namespace {

template <int L>
__global__ void __launch_bounds__(128) boys_values(const double* __restrict__ tab,
                                                   const double* __restrict__ T, long long n,
                                                   double* __restrict__ F) {
  __shared__ double s_tab[kBoysNGrid * kBoysTaylor];
  __shared__ double s_exp[kBoysNGrid];
  stage_boys<L>(tab, s_tab, s_exp);
  __syncthreads();
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double t = T[i];
    double f[L + 1];
    if (t >= 0.0 && t <= 1e300) {  // the host rejects anything else; never index the table with it
      boys_eval<L>(t, s_tab, s_exp, f);
    } else {
#pragma unroll
      for (int m = 0; m <= L; ++m) f[m] = __longlong_as_double(0x7ff8000000000000LL);
    }
#pragma unroll
    for (int m = 0; m <= L; ++m) F[i * (L + 1) + m] = f[m];
  }
}

template <int L>
int launch_boys(int m_max, const double* tab, const double* T, long long n, double* F,
                cudaStream_t st) {
  if constexpr (L > kBoysMMax) {
    return set_error(GBX_ERR_INVALID, "m_max %d above %d", m_max, kBoysMMax);
  } else {
    if (m_max != L) return launch_boys<L + 1>(m_max, tab, T, n, F, st);
    const int grid = (int)std::max<long long>(1, std::min<long long>((n + 127) / 128, 1184));
    boys_values<L><<<grid, 128, 0, st>>>(tab, T, n, F);
    return cuda_status(cudaGetLastError(), "boys_values launch");
  }
}

}  // namespace
}  // namespace gbx

using namespace gbx;

extern "C" int gbx_boys_eval(int m_max, int64_t n, const double* T, double* F) {
  if (n < 0 || (n > 0 && (!T || !F))) return set_error(GBX_ERR_INVALID, "gbx_boys_eval: null argument");
  if (m_max < 0 || m_max > kBoysMMax)
    return set_error(GBX_ERR_INVALID, "gbx_boys_eval: m_max %d outside [0, %d]", m_max, kBoysMMax);
  for (int64_t i = 0; i < n; ++i)
    if (!(T[i] >= 0.0) || !std::isfinite(T[i]))
      return set_error(GBX_ERR_INVALID, "gbx_boys_eval: T[%lld] = %g is not a finite value >= 0",
                       (long long)i, T[i]);
  if (n == 0) return GBX_OK;
  int dev = 0;
  int s = cuda_status(cudaGetDevice(&dev), "cudaGetDevice");
  if (s) return s;
  const double* tab = nullptr;
  if ((s = boys_table(dev, &tab))) return s;
  double *dT = nullptr, *dF = nullptr;
  const size_t nf = (size_t)n * (m_max + 1);
  if ((s = cuda_status(cudaMalloc(&dT, n * sizeof(double)), "cudaMalloc(T)"))) return s;
  if ((s = cuda_status(cudaMalloc(&dF, nf * sizeof(double)), "cudaMalloc(F)"))) {
    cudaFree(dT);
    return s;
  }
  s = cuda_status(cudaMemcpy(dT, T, n * sizeof(double), cudaMemcpyHostToDevice), "upload T");
  if (!s) s = launch_boys<0>(m_max, tab, dT, n, dF, 0);
  if (!s) s = cuda_status(cudaMemcpy(F, dF, nf * sizeof(double), cudaMemcpyDeviceToHost), "download F");
  cudaFree(dT);
  cudaFree(dF);
  return s;
}
