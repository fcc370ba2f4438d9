// Allocation-free generalized eigensolver (tb_sygvd_noalloc).
//
// Some callers of this library cannot let it allocate device memory: host
// frameworks that own all GPU memory through their own pool allocator and
// forbid libraries from calling cudaMalloc behind their back, latency-critical
// loops where cudaMalloc/cudaFree would synchronise the whole device, and
// processes that run under a fixed memory budget that must not grow at run
// time.  For them this entry point solves one H C = S C e problem with every
// intermediate in a statically sized device array that is part of the loaded
// module, using the same kernels as tb_sygvd_batch.
//
// Limits and sharing rules:
//  * n <= kNoAllocMaxN (256); larger n is rejected with TB_CAPACITY_EXCEEDED.
//  * The scratch (about 2 MiB) belongs to the library module, so every GPU that
//    loads the library holds it until the process exits.
//  * All calls on a device share the one array and it keeps the last call's
//    contents; each call rewrites everything it reads before reading it.
//    Calls whose GPU work overlaps (different streams, different host threads
//    without ordering) race on the array: serialise them.
//  * The first call on a device does its set-up: it raises the eigensolver
//    kernel's dynamic shared memory limit to what n = 256 needs (above the
//    48 KiB default from n = 237 on; setting a kernel attribute allocates
//    nothing) and looks up the array's device address (cudaGetSymbolAddress,
//    cached per device).  Make that first call before any stream capture
//    begins.
//  * The call is synchronous: it waits for its stream to read the status.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/tblite_b200.h"
#include "tb_common.cuh"
#include "tb_kernels.h"

namespace tb {

constexpr int kNoAllocMaxN = 256;
constexpr int kNoAllocTiles = ((kNoAllocMaxN + 63) / 64) * ((kNoAllocMaxN + 63) / 64);
constexpr long long kNoAllocN2 = (long long)kNoAllocMaxN * kNoAllocMaxN;
// misc region (in doubles): perm (n ints), status, active, ooff[2], moff[2], tiles
constexpr long long kMiscDoubles = kNoAllocMaxN / 2 + 8 + 2 * kNoAllocTiles + 8;
constexpr long long kScratchDoubles = 4 * kNoAllocN2 + kMiscDoubles;

// W (Cholesky factor, then GEMM temporary), X = L^-T, A (X^T H X, destroyed by
// the eigensolver), Z (eigenvector rows), then the misc region.
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

struct ScratchView {
  double *W, *X, *A, *Z;
  int* perm;
  int* status;
  int* active;
  int* ooff;
  long long* moff;
  int4* tiles;
};

__host__ __device__ inline ScratchView scratch_view(double* base) {
  ScratchView v;
  v.W = base;
  v.X = base + kNoAllocN2;
  v.A = base + 2 * kNoAllocN2;
  v.Z = base + 3 * kNoAllocN2;
  double* misc = base + 4 * kNoAllocN2;
  v.perm = reinterpret_cast<int*>(misc);
  int* ints = reinterpret_cast<int*>(misc + kNoAllocMaxN / 2);
  v.status = ints;
  v.active = ints + 1;
  v.ooff = ints + 2;                                                       // 2 ints
  v.moff = reinterpret_cast<long long*>(misc + kNoAllocMaxN / 2 + 4);      // 2 longs
  v.tiles = reinterpret_cast<int4*>(misc + kNoAllocMaxN / 2 + 8);          // 16 B aligned
  return v;
}

// Writes the one-matrix batch description and clears the status words, so no
// value of an earlier call is ever read.
__global__ void k_noalloc_init(double* base, int n) {
  const ScratchView v = scratch_view(base);
  const int nt = (n + 63) / 64;
  if (threadIdx.x == 0) {
    v.ooff[0] = 0;
    v.ooff[1] = n;
    v.moff[0] = 0;
    v.moff[1] = (long long)n * n;
    v.status[0] = kStOk;
    v.active[0] = 1;
  }
  for (int t = threadIdx.x; t < nt * nt; t += blockDim.x) v.tiles[t] = make_int4(0, t / nt, t % nt, 0);
}

}  // namespace tb

using namespace tb;

namespace {

std::mutex g_noalloc_mu;
double* g_noalloc_addr[64] = {nullptr};

tb_status noalloc_fail(tb_status st, const char* msg);

}  // namespace

extern const char* tb_noalloc_set_error(const char* msg);

extern "C" tb_status tb_sygvd_noalloc(int32_t n, const double* H, const double* S, double* w, double* C,
                                      void* stream) {
  if (n < 1 || n > kNoAllocMaxN)
    return noalloc_fail(TB_CAPACITY_EXCEEDED, "tb_sygvd_noalloc: n must be in 1..256 (static scratch limit)");
  if (!H || !S || !w || !C) return noalloc_fail(TB_BAD_INPUT, "tb_sygvd_noalloc: null pointer");
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return noalloc_fail(TB_CUDA_ERROR, cudaGetErrorString(e));
  if (dev < 0 || dev >= 64) return noalloc_fail(TB_CUDA_ERROR, "tb_sygvd_noalloc: device ordinal out of range");
  double* base = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[dev]) {
      // per-device set-up, with this device current: the eigensolver's shared
      // memory opt-in for the largest accepted n (raised only: the batched
      // paths may already have set a higher limit), then the scratch address
      // (cached last, so that a failed set-up is retried by the next call)
      cudaFuncAttributes fa;
      e = cudaFuncGetAttributes(&fa, (const void*)k_syev);
      const int need = (int)syev_smem_bytes(kNoAllocMaxN);
      if (e == cudaSuccess && fa.maxDynamicSharedSizeBytes < need)
        e = cudaFuncSetAttribute((const void*)k_syev, cudaFuncAttributeMaxDynamicSharedMemorySize, need);
      if (e != cudaSuccess) return noalloc_fail(TB_CUDA_ERROR, cudaGetErrorString(e));
      double* addr = nullptr;
      e = cudaGetSymbolAddress(reinterpret_cast<void**>(&addr), g_noalloc_scratch);
      if (e != cudaSuccess) return noalloc_fail(TB_CUDA_ERROR, cudaGetErrorString(e));
      g_noalloc_addr[dev] = addr;
    }
    base = g_noalloc_addr[dev];
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const ScratchView v = scratch_view(base);
  DevBatch B{};
  B.nmol = 1;
  B.ooff = v.ooff;
  B.moff = v.moff;
  const int nt = (n + 63) / 64, ntiles = nt * nt;
  k_noalloc_init<<<1, 64, 0, st>>>(base, n);
  k_cholesky<<<1, 256, 0, st>>>(B, S, v.W, v.status, nullptr);
  k_trinv<<<1, 256, 0, st>>>(B, v.W, v.X, v.status);
  // A = X^T H X (T = H X kept in W, whose Cholesky factor is no longer needed)
  k_gemm<<<ntiles, kGemmThreads, 0, st>>>(B, v.tiles, ntiles, H, 0, v.X, 0, nullptr, nullptr, nullptr, v.W, 1.0, 0.0,
                                 v.active, kGemmKUpToJ);
  k_gemm<<<ntiles, kGemmThreads, 0, st>>>(B, v.tiles, ntiles, v.X, 1, v.W, 0, nullptr, nullptr, nullptr, v.A, 1.0, 0.0,
                                 v.active, kGemmKUpToI | kGemmSym);
  k_syev<<<1, kEigThreads, syev_smem_bytes(n), st>>>(B, v.A, v.Z, v.W, w, v.perm, v.status, v.active);
  // C = X Z with the eigenvectors in ascending order
  k_gemm<<<ntiles, kGemmThreads, 0, st>>>(B, v.tiles, ntiles, v.X, 0, v.Z, 1, v.perm, nullptr, nullptr, C, 1.0, 0.0,
                                 v.active, kGemmKFromI);
  e = cudaGetLastError();
  if (e != cudaSuccess) return noalloc_fail(TB_CUDA_ERROR, cudaGetErrorString(e));
  int status = 0;
  e = cudaMemcpyAsync(&status, v.status, sizeof(int), cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return noalloc_fail(TB_CUDA_ERROR, cudaGetErrorString(e));
  if (status != kStOk) return noalloc_fail(static_cast<tb_status>(status), "tb_sygvd_noalloc: solver status");
  return TB_OK;
}

namespace {
tb_status noalloc_fail(tb_status st, const char* msg) {
  tb_noalloc_set_error(msg);
  return st;
}
}  // namespace
