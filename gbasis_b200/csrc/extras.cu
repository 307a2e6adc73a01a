// Auxiliary entry points: 4-index transform (cuBLAS DGEMM chain), FP64 FMA-rate probe.
#include <cublas_v2.h>

#include <cstdio>

#include "gbx_eri.h"
#include "gbx_common.cuh"
#include "runtime.h"

using namespace gbx;

namespace gbx {
int coulomb_entry(gbx_basis* b, const double* D, double tau, double* J, cudaStream_t st,
                  double skip = 0.0, double fp32 = 0.0);
int jk_entry(gbx_basis* b, const double* D, double tau, double* J, double* K, cudaStream_t st);
}

namespace {

struct CublasHandle {
  cublasHandle_t h = nullptr;
  ~CublasHandle() {
    if (h) cublasDestroy(h);
  }
};
thread_local CublasHandle t_cublas;

// Chains of dependent FMAs, 8 independent chains per thread.
__global__ void fp64_fma_probe(double* out, int iters, double a, double b) {
  double x0 = threadIdx.x * 1e-9, x1 = x0 + 1e-3, x2 = x0 + 2e-3, x3 = x0 + 3e-3;
  double x4 = x0 + 4e-3, x5 = x0 + 5e-3, x6 = x0 + 6e-3, x7 = x0 + 7e-3;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int k = 0; k < 16; ++k) {
      x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
      x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
  }
  const double s = x0 + x1 + x2 + x3 + x4 + x5 + x6 + x7;
  if (s == 1.2345) out[blockIdx.x] = s;  // keeps the chains live
}

// FP64 tensor-core rate: 8 independent chains of mma.sync m8n8k4 (512 flops per warp each).
__global__ void fp64_mma_probe(double* out, int iters, double a, double b) {
  double c[8][2];
#pragma unroll
  for (int k = 0; k < 8; ++k) c[k][0] = c[k][1] = threadIdx.x * 1e-9 + k * 1e-3;
  const double av = a + threadIdx.x * 1e-12, bv = b;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int r = 0; r < 2; ++r) {
#pragma unroll
      for (int k = 0; k < 8; ++k)
        asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                     : "+d"(c[k][0]), "+d"(c[k][1])
                     : "d"(av), "d"(bv));
    }
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += c[k][0] + c[k][1];
  if (s == 1.2345) out[blockIdx.x] = s;
}

// FP32 FMA rate: as fp64_fma_probe in single precision.
__global__ void fp32_fma_probe(double* out, int iters, float a, float b) {
  float x[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) x[k] = threadIdx.x * 1e-9f + k * 1e-3f;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int r = 0; r < 16; ++r) {
#pragma unroll
      for (int k = 0; k < 8; ++k) x[k] = fmaf(x[k], a, b);
    }
  }
  float s = 0.f;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += x[k];
  if (s == 1.2345f) out[blockIdx.x] = s;
}

}  // namespace

extern "C" {

int gbx_pipe_peak(int device, int pipe, double* tflops) {
  if (!tflops || pipe < 0 || pipe > 2)
    return set_error(GBX_ERR_INVALID, "gbx_pipe_peak: pipe must be 0 (FP64 FMA), 1 (FP64 mma) or 2 (FP32 FMA)");
  if (pipe == 0) return gbx_fp64_peak(device, tflops);
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(device);
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  double* d = nullptr;
  int s = cuda_status(cudaMalloc(&d, 4096 * sizeof(double)), "cudaMalloc(probe)");
  if (s) {
    cudaSetDevice(prev);
    return s;
  }
  const int blocks = nsm * 8, threads = 256, iters = pipe == 1 ? 1024 : 4096;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  auto run = [&](int it) {
    if (pipe == 1) fp64_mma_probe<<<blocks, threads>>>(d, it, 0.999999, 1e-7);
    else fp32_fma_probe<<<blocks, threads>>>(d, it, 0.999999f, 1e-7f);
  };
  run(16);  // warm-up
  float best = 1e30f;
  for (int rep = 0; rep < 5; ++rep) {
    cudaEventRecord(e0);
    run(iters);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  s = cuda_status(cudaGetLastError(), "pipe probe");
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d);
  cudaSetDevice(prev);
  if (s) return s;
  const double warps = (double)blocks * threads / 32;
  const double flops = pipe == 1 ? 512.0 * 16 * iters * warps                  // 16 mma per iteration
                                 : 2.0 * 8 * 16 * (double)iters * blocks * threads;
  *tflops = flops / (best * 1e-3) / 1e12;
  return GBX_OK;
}

int gbx_lincomb(const double* in, int64_t n, const double* T, int64_t n_orb, double* out,
                double* work, void* stream) {
  if (!in || !T || !out || !work || n <= 0 || n_orb <= 0)
    return set_error(GBX_ERR_INVALID, "gbx_lincomb: bad argument");
  if (!t_cublas.h && cublasCreate(&t_cublas.h) != CUBLAS_STATUS_SUCCESS)
    return set_error(GBX_ERR_CUDA, "cublasCreate failed");
  cublasSetStream(t_cublas.h, (cudaStream_t)stream);
  const int64_t M = n > n_orb ? n : n_orb;
  double* w0 = work;
  double* w1 = work + M * M * M * M;
  const double* src[4] = {in, w0, w1, w0};
  double* dst[4] = {w0, w1, w0, out};
  int64_t rest = n * n * n;  // size of the uncontracted trailing axes
  const double one = 1.0, zero = 0.0;
  for (int step = 0; step < 4; ++step) {
    // row-major X[a][r] (a < n) -> Y[r][o] = sum_a T[o][a] X[a][r]; next step sees Y as
    // [next original axis][rest'] with the new orbital axis appended last.
    cublasStatus_t st = cublasDgemm(t_cublas.h, CUBLAS_OP_T, CUBLAS_OP_T, (int)n_orb, (int)rest,
                                    (int)n, &one, T, (int)n, src[step], (int)rest, &zero,
                                    dst[step], (int)n_orb);
    if (st != CUBLAS_STATUS_SUCCESS) return set_error(GBX_ERR_CUDA, "cublasDgemm failed (%d)", (int)st);
    rest = rest / n * n_orb;
  }
  return cuda_status(cudaGetLastError(), "gbx_lincomb");
}

int gbx_fp64_peak(int device, double* tflops) {
  if (!tflops) return set_error(GBX_ERR_INVALID, "gbx_fp64_peak: null argument");
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(device);
  int nsm = 0;
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, device);
  double* d = nullptr;
  int s = cuda_status(cudaMalloc(&d, 4096 * sizeof(double)), "cudaMalloc(probe)");
  if (s) return s;
  const int blocks = nsm * 8, threads = 256, iters = 4096;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  fp64_fma_probe<<<blocks, threads>>>(d, 64, 0.999999, 1e-7);  // warm-up
  float best = 1e30f;
  for (int rep = 0; rep < 5; ++rep) {
    cudaEventRecord(e0);
    fp64_fma_probe<<<blocks, threads>>>(d, iters, 0.999999, 1e-7);
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (ms < best) best = ms;
  }
  s = cuda_status(cudaGetLastError(), "fp64 probe");
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaFree(d);
  cudaSetDevice(prev);
  if (s) return s;
  const double flops = 2.0 * 8 * 16 * (double)iters * blocks * threads;
  *tflops = flops / (best * 1e-3) / 1e12;
  return GBX_OK;
}

int gbx_eri_coulomb_j(gbx_basis* b, const double* D, double tau, double* J, void* stream) {
  if (!b || !D || !J) return set_error(GBX_ERR_INVALID, "gbx_eri_coulomb_j: null argument");
  if (!(tau >= 0.0)) return set_error(GBX_ERR_INVALID, "schwarz threshold must be >= 0");
  return gbx::coulomb_entry(b, D, tau, J, (cudaStream_t)stream);
}

int gbx_eri_coulomb_j_mixed(gbx_basis* b, const double* D, double skip, double fp32, double* J,
                            void* stream) {
  if (!b || !D || !J) return set_error(GBX_ERR_INVALID, "gbx_eri_coulomb_j_mixed: null argument");
  if (!(skip > 0.0) || !(fp32 >= skip) || !(fp32 < 1.0))
    return set_error(GBX_ERR_INVALID, "need 0 < skip <= fp32 < 1 (got %g, %g)", skip, fp32);
  return gbx::coulomb_entry(b, D, 0.0, J, (cudaStream_t)stream, skip, fp32);
}

int gbx_eri_jk(gbx_basis* b, const double* D, double tau, double* J, double* K, void* stream) {
  if (!b || !D || !J || !K) return set_error(GBX_ERR_INVALID, "gbx_eri_jk: null argument");
  if (J == K) return set_error(GBX_ERR_INVALID, "gbx_eri_jk: J and K must be different buffers");
  if (!(tau >= 0.0)) return set_error(GBX_ERR_INVALID, "schwarz threshold must be >= 0");
  return gbx::jk_entry(b, D, tau, J, K, (cudaStream_t)stream);
}

}  // extern "C"
