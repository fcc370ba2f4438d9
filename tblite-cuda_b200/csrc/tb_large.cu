// Dense path for structures above the in-house eigensolver's stated size.
//
// The batched one-CTA-per-structure kernels (k_cholesky, k_trinv, k_syev)
// keep every matrix of a structure on one SM; past about a thousand AOs that
// SM, not the GPU, sets the time.  Structures with more AOs than the stated
// bound (tb_options.solver; 1216 by default) are therefore factorised and
// diagonalised by cuSOLVER's 64-bit dense API, one structure at a time on the
// run's stream, writing the SAME layouts the in-house kernels write:
//  * X = L^-T, row-major upper triangular (k_trinv's output): Xpotrf (lower)
//    and Xtrtri (lower, non-unit) on a column-major copy of S leave L^-1 in
//    the lower triangle, which read row-major is L^-T; the strict lower
//    triangle of the row-major view still holds S and is cleared.
//  * eigenvectors one per row of Z, ascending w, perm = identity (k_syev's
//    output): Xsyevd (jobz V) stores eigenvector j in column j of a
//    column-major matrix, i.e. row j of the row-major view.
// Everything else of the SCF (GEMMs, Fock, Fermi, Mulliken, mixing) runs the
// same kernels for every size.
#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <string>

#include "tb_common.cuh"
#include "tb_kernels.h"

namespace tb {

namespace {

const char* cusolver_name(cusolverStatus_t s) {
  switch (s) {
    case CUSOLVER_STATUS_SUCCESS: return "success";
    case CUSOLVER_STATUS_NOT_INITIALIZED: return "not initialized";
    case CUSOLVER_STATUS_ALLOC_FAILED: return "allocation failed";
    case CUSOLVER_STATUS_INVALID_VALUE: return "invalid value";
    case CUSOLVER_STATUS_ARCH_MISMATCH: return "architecture mismatch";
    case CUSOLVER_STATUS_EXECUTION_FAILED: return "execution failed";
    case CUSOLVER_STATUS_INTERNAL_ERROR: return "internal error";
    case CUSOLVER_STATUS_NOT_SUPPORTED: return "not supported";
    default: return "error";
  }
}

#define LS_CHECK(call)                                                               \
  do {                                                                               \
    cusolverStatus_t s_ = (call);                                                    \
    if (s_ != CUSOLVER_STATUS_SUCCESS) return std::string(#call) + ": " + cusolver_name(s_); \
  } while (0)
#define LS_CUDA(call)                                                                \
  do {                                                                               \
    cudaError_t e_ = (call);                                                         \
    if (e_ != cudaSuccess) return std::string(#call) + ": " + cudaGetErrorString(e_); \
  } while (0)

// Clears the strict lower triangle of the row-major X and turns the two
// factorisation infos into the structure's status.
__global__ void k_lib_factor_post(double* __restrict__ X, int n, const int* __restrict__ info,
                                  int* __restrict__ status) {
  const long long nn = (long long)n * n;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nn; e += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(e / n), c = (int)(e - (long long)r * n);
    if (r > c) X[e] = 0.0;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && (info[0] != 0 || info[1] != 0)) *status = kStNotSpd;
}

// perm = identity (Xsyevd returns ascending eigenvalues), info -> status.
__global__ void k_lib_syev_post(int* __restrict__ perm, int n, const int* __restrict__ info, int* __restrict__ status) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) perm[j] = j;
  if (blockIdx.x == 0 && threadIdx.x == 0 && info[0] != 0) *status = kStEigenFailed;
}

// FP32 variant: ascending eigenvalues widened to FP64.
__global__ void k_lib_syev32_post(int* __restrict__ perm, const float* __restrict__ wtmp, double* __restrict__ w,
                                  int n, const int* __restrict__ info, int* __restrict__ status) {
  for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    perm[j] = j;
    w[j] = (double)wtmp[j];
  }
  if (blockIdx.x == 0 && threadIdx.x == 0 && info[0] != 0) *status = kStEigenFailed;
}

inline int grid_for(long long items) {
  const long long g = (items + 255) / 256;
  return (int)(g < 148 * 16 ? (g < 1 ? 1 : g) : 148 * 16);
}

}  // namespace

LargeSolver::~LargeSolver() {
  if (params) cusolverDnDestroyParams(static_cast<cusolverDnParams_t>(params));
  if (handle) cusolverDnDestroy(static_cast<cusolverDnHandle_t>(handle));
}

std::string LargeSolver::init() {
  if (handle) return "";
  cusolverDnHandle_t h = nullptr;
  LS_CHECK(cusolverDnCreate(&h));
  handle = h;
  cusolverDnParams_t p = nullptr;
  LS_CHECK(cusolverDnCreateParams(&p));
  params = p;
  return "";
}

std::string LargeSolver::workspace(int n, size_t* dev_bytes) {
  std::string err = init();
  if (!err.empty()) return err;
  auto h = static_cast<cusolverDnHandle_t>(handle);
  auto p = static_cast<cusolverDnParams_t>(params);
  size_t d1 = 0, h1 = 0, d2 = 0, h2 = 0, d3 = 0, h3 = 0;
  // sizes depend only on n; the matrix pointers are not read
  LS_CHECK(cusolverDnXpotrf_bufferSize(h, p, CUBLAS_FILL_MODE_LOWER, n, CUDA_R_64F, nullptr, n, CUDA_R_64F, &d1, &h1));
  LS_CHECK(cusolverDnXtrtri_bufferSize(h, CUBLAS_FILL_MODE_LOWER, CUBLAS_DIAG_NON_UNIT, n, CUDA_R_64F, nullptr, n, &d2,
                                       &h2));
  LS_CHECK(cusolverDnXsyevd_bufferSize(h, p, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, CUDA_R_64F, nullptr,
                                       n, CUDA_R_64F, nullptr, CUDA_R_64F, &d3, &h3));
  size_t d4 = 0, h4 = 0;
  LS_CHECK(cusolverDnXsyevd_bufferSize(h, p, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, CUDA_R_32F, nullptr,
                                       n, CUDA_R_32F, nullptr, CUDA_R_32F, &d4, &h4));
  size_t d = d1 > d2 ? d1 : d2;
  d = d > d3 ? d : d3;
  d = d > d4 ? d : d4;
  size_t hb = h1 > h2 ? h1 : h2;
  hb = hb > h3 ? hb : h3;
  hb = hb > h4 ? hb : h4;
  if (host.size() < hb) host.resize(hb);
  *dev_bytes = d;
  return "";
}

std::string LargeSolver::factor(cudaStream_t st, const double* S, double* X, int n, void* dwork, size_t dbytes,
                                int* info, int* status) {
  std::string err = init();
  if (!err.empty()) return err;
  auto h = static_cast<cusolverDnHandle_t>(handle);
  auto p = static_cast<cusolverDnParams_t>(params);
  LS_CHECK(cusolverDnSetStream(h, st));
  LS_CUDA(cudaMemcpyAsync(X, S, (size_t)n * n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  void* hw = host.empty() ? nullptr : host.data();
  LS_CHECK(cusolverDnXpotrf(h, p, CUBLAS_FILL_MODE_LOWER, n, CUDA_R_64F, X, n, CUDA_R_64F, dwork, dbytes, hw,
                            host.size(), info));
  LS_CHECK(cusolverDnXtrtri(h, CUBLAS_FILL_MODE_LOWER, CUBLAS_DIAG_NON_UNIT, n, CUDA_R_64F, X, n, dwork, dbytes, hw,
                            host.size(), info + 1));
  k_lib_factor_post<<<grid_for((long long)n * n), 256, 0, st>>>(X, n, info, status);
  LS_CUDA(cudaGetLastError());
  return "";
}

std::string LargeSolver::syev(cudaStream_t st, const double* A, double* Z, double* w, int* perm, int n, void* dwork,
                              size_t dbytes, int* info, int* status) {
  std::string err = init();
  if (!err.empty()) return err;
  auto h = static_cast<cusolverDnHandle_t>(handle);
  auto p = static_cast<cusolverDnParams_t>(params);
  LS_CHECK(cusolverDnSetStream(h, st));
  LS_CUDA(cudaMemcpyAsync(Z, A, (size_t)n * n * sizeof(double), cudaMemcpyDeviceToDevice, st));
  void* hw = host.empty() ? nullptr : host.data();
  LS_CHECK(cusolverDnXsyevd(h, p, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, CUDA_R_64F, Z, n, CUDA_R_64F,
                            w, CUDA_R_64F, dwork, dbytes, hw, host.size(), info));
  k_lib_syev_post<<<grid_for(n), 256, 0, st>>>(perm, n, info, status);
  LS_CUDA(cudaGetLastError());
  return "";
}

std::string LargeSolver::syev32(cudaStream_t st, const float* A, float* Z, float* wtmp, double* w, int* perm, int n,
                                void* dwork, size_t dbytes, int* info, int* status) {
  std::string err = init();
  if (!err.empty()) return err;
  auto h = static_cast<cusolverDnHandle_t>(handle);
  auto p = static_cast<cusolverDnParams_t>(params);
  LS_CHECK(cusolverDnSetStream(h, st));
  LS_CUDA(cudaMemcpyAsync(Z, A, (size_t)n * n * sizeof(float), cudaMemcpyDeviceToDevice, st));
  void* hw = host.empty() ? nullptr : host.data();
  LS_CHECK(cusolverDnXsyevd(h, p, CUSOLVER_EIG_MODE_VECTOR, CUBLAS_FILL_MODE_LOWER, n, CUDA_R_32F, Z, n, CUDA_R_32F,
                            wtmp, CUDA_R_32F, dwork, dbytes, hw, host.size(), info));
  k_lib_syev32_post<<<grid_for(n), 256, 0, st>>>(perm, wtmp, w, n, info, status);
  LS_CUDA(cudaGetLastError());
  return "";
}

}  // namespace tb
