// Split-precision batched GEMM on the Blackwell tensor cores (tcgen05).
//
// C_m = alpha op(A_m) diag(ks_m) op(B_m) + beta C_m for the contractions of
// the mixed-precision form (F' = X^T F X, C = X V, P = C f C^T), with the same
// arguments as k_gemm but a list of 128 x 128 tiles.  Operands are stored in
// FP64; each is split into TF32 hi + lo parts (hi = round(x), lo = round(x -
// hi)) and the product is formed as hi*hi + hi*lo + lo*hi with FP32
// accumulation ("TF32x3"), which keeps about FP32 accuracy.
//
// Per CTA (8 warps, one CTA per SM, persistent over the tile list):
//  * TMEM: a 128 x 128 FP32 accumulator (128 columns), allocated once;
//  * shared memory: two stages of A_hi, A_lo, B_hi, B_lo, each 128 rows x 32
//    K values in the canonical no-swizzle K-major layout of the tensor-core
//    operand descriptors: 8 x 16-byte core matrices, row r at (r % 8) * 16 +
//    (r / 8) * 1024 bytes, K chunk c (4 values) at c * 128 bytes;
//  * all 8 warps stage a K slab (FP64 loads, split, 16-byte shared stores), then one
//    thread issues 3 x 4 tcgen05.mma (M = 128, N = 128, K = 8 each) and
//    commits them to the stage's mbarrier; a stage is refilled only after its
//    mbarrier phase completes (bounded wait);
//  * epilogue: tcgen05.ld 32x32b (warp w reads TMEM lanes 32(w%4)..+31 = rows,
//    columns 64(w/4)..+63), FP64 stores.
// Every wait is bounded: on timeout the structure is marked failed (status)
// and the CTA leaves after releasing its TMEM.
#include <cuda_runtime.h>
#include <stdint.h>

#include "tb_common.cuh"
#include "tb_kernels.h"

namespace tb {

namespace {

constexpr int TM = 128, TN = 128, TK = 32;           // tile and K slab
constexpr int kOpBytes = TM * TK * 4;               // one TF32 operand slab: 16 KiB
constexpr int kStageBytes = 4 * kOpBytes;           // A_hi, A_lo, B_hi, B_lo
constexpr int kTmemCols = 128;
constexpr long long kWaitLimit = 1LL << 26;

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// operand descriptor: no swizzle, K-major, LBO = 128 B (next 4-value K chunk),
// SBO = 1024 B (next 8-row group), descriptor version 1
__device__ __forceinline__ uint64_t op_desc(uint32_t saddr) {
  return (uint64_t)((saddr & 0x3FFFF) >> 4) | ((uint64_t)(128 >> 4) << 16) | ((uint64_t)(1024 >> 4) << 32) |
         (1ull << 46);
}
// instruction descriptor: D F32, A/B TF32, both K-major, N = 128, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(TN >> 3) << 17) | ((uint32_t)(TM >> 4) << 24);

__device__ __forceinline__ uint32_t to_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return r;
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem_d),
      "l"(da), "l"(db), "r"(kIdesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
}

__device__ __forceinline__ void mma_commit(uint64_t* mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(mbar))
               : "memory");
}

// bounded wait for the given phase parity of an mbarrier
__device__ __forceinline__ bool mbar_wait(uint64_t* mbar, uint32_t parity) {
  const uint32_t a = smem_u32(mbar);
  for (long long it = 0; it < kWaitLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// One operand slab (128 rows x 32 K) of a 128 x 128 tile.  Row r of the slab
// is op(M)[rbase + r][k0 + k]: element M[row][k] when kmajor (row-major source,
// K contiguous), M[k][row] otherwise; rows go through perm (columns of op(B))
// and K through the diag(ks) scale when given.
__device__ __forceinline__ void stage_operand(unsigned char* s_hi, unsigned char* s_lo, const double* M, int kmajor,
                                              const int* perm, const double* kv, int n, int K, int rbase, int k0,
                                              int tid) {
  constexpr int kUnits = TM * (TK / 4) / kTcThreads;  // 4 units of 4 values per thread
  double x[kUnits][4];
  int off[kUnits];
  bool ok[kUnits];
#pragma unroll
  for (int q = 0; q < kUnits; ++q) {
    const int u = tid + kTcThreads * q;
    const int r = (u & 7) | ((u >> 6) << 3), c = (u >> 3) & 7;
    const int g = rbase + r;
    ok[q] = g < n;
    off[q] = (r & 7) * 16 + (r >> 3) * 1024 + c * 128;
    const int row = (ok[q] && perm) ? perm[g] : g;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int gk = k0 + 4 * c + j;
      double v = 0.0;
      if (ok[q] && gk < K) v = kmajor ? M[(long long)row * n + gk] : M[(long long)gk * n + row];
      x[q][j] = v;
    }
    if (kv) {
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int gk = k0 + 4 * c + j;
        if (gk < K) x[q][j] *= kv[gk];
      }
    }
  }
#pragma unroll
  for (int q = 0; q < kUnits; ++q) {
    if (!ok[q]) continue;
    uint32_t h[4], l[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const float f = (float)x[q][j];
      h[j] = to_tf32(f);
      l[j] = to_tf32(f - __uint_as_float(h[j]));
    }
    *reinterpret_cast<uint4*>(s_hi + off[q]) = make_uint4(h[0], h[1], h[2], h[3]);
    *reinterpret_cast<uint4*>(s_lo + off[q]) = make_uint4(l[0], l[1], l[2], l[3]);
  }
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace

__global__ void __launch_bounds__(kTcThreads, 1) k_gemm_tc(DevBatch B, const int4* __restrict__ tiles, int ntiles,
                                                    const double* __restrict__ Ab, int ta,
                                                    const double* __restrict__ Bb, int tb_,
                                                    const int* __restrict__ perm, const double* __restrict__ ks,
                                                    const int* __restrict__ kdim, double* __restrict__ Cb,
                                                    double alpha, double beta, const int* __restrict__ active,
                                                    int* __restrict__ status) {
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t tmem_base;
  __shared__ int abort_flag;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;  // kTcThreads = 8 warps

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&mbar[0])), "r"(1));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(&mbar[1])), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    abort_flag = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base;
  uint32_t uses[2] = {0, 0};  // commits issued per stage (the last one's phase parity = (uses - 1) & 1)
  int cur = -1;               // structure of the tile in work

  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int4 tl = tiles[t];
    const int m = tl.x;
    if (active && !active[m]) continue;
    cur = m;
    const int n = B.ooff[m + 1] - B.ooff[m];
    const int K = kdim ? min(max(kdim[m], 0), n) : n;  // never outside [0, n], whatever kdim holds
    const long long mo = B.moff[m];
    const long long vo = B.ooff[m];
    const double* A = Ab + mo;
    const double* Bm = Bb + mo;
    const int* pm = perm ? perm + vo : nullptr;
    const double* kv = ks ? ks + vo : nullptr;
    const int i0 = tl.y * TM, j0 = tl.z * TN;
    const int nk = (K + TK - 1) / TK;
    for (int kt = 0; kt < nk; ++kt) {
      const int st = kt & 1;
      // the stage's previous MMAs must have finished reading it
      if (uses[st] > 0) {
        // the stage's last commit must have completed before it is refilled
        if (!mbar_wait(&mbar[st], (uses[st] - 1) & 1)) atomicExch(&abort_flag, 1);
      }
      unsigned char* sA_hi = tc_smem + st * kStageBytes;
      unsigned char* sA_lo = sA_hi + kOpBytes;
      unsigned char* sB_hi = sA_lo + kOpBytes;
      unsigned char* sB_lo = sB_hi + kOpBytes;
      const int k0 = kt * TK;
      // Stage op(A)[i0 + r][k0 + k] and op(B)[k0 + k][j0 + r] in units of one
      // core-matrix row (row r, 4 consecutive K values = 16 bytes).  Unit u:
      // r % 8 = u bits 0-2, K chunk c = bits 3-5, r / 8 = bits 6-9, so the 8
      // lanes of a quarter-warp store 128 contiguous bytes.  Rows past n are
      // skipped (they only reach output rows or columns that are not stored);
      // K past the structure's K is zero.  Loads first, then split and store.
      // op(A) rows are K-contiguous unless A is transposed; op(B)^T rows unless B is not
      stage_operand(sA_hi, sA_lo, A, !ta, nullptr, kv, n, K, i0, k0, tid);
      stage_operand(sB_hi, sB_lo, Bm, tb_, pm, nullptr, n, K, j0, k0, tid);
      // generic-proxy shared stores must be visible to the tensor core's async proxy
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (abort_flag) break;
      if (tid == 0) {
#pragma unroll
        for (int s = 0; s < TK / 8; ++s) {
          const uint32_t kb = s * 256;  // two 4-value chunks per K = 8 step
          const uint64_t dah = op_desc(smem_u32(sA_hi) + kb), dal = op_desc(smem_u32(sA_lo) + kb);
          const uint64_t dbh = op_desc(smem_u32(sB_hi) + kb), dbl = op_desc(smem_u32(sB_lo) + kb);
          mma_tf32(tmem, dah, dbh, (kt > 0 || s > 0) ? 1u : 0u);
          mma_tf32(tmem, dah, dbl, 1u);
          mma_tf32(tmem, dal, dbh, 1u);
        }
        mma_commit(&mbar[st]);
      }
      ++uses[st];
    }
    __syncthreads();
    if (abort_flag) break;
    // wait for the last stage's MMAs (they complete in order); K = 0 gives C = beta C
    if (nk > 0) {
      const int st = (nk - 1) & 1;
      if (!mbar_wait(&mbar[st], (uses[st] - 1) & 1)) atomicExch(&abort_flag, 1);
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    __syncthreads();
    if (abort_flag) break;
    // epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 (its rows) and
    // columns 64 (w / 4) .. + 63, 16 per load
    const int quad = warp & 3, half = warp >> 2;
    const int gi = i0 + 32 * quad + lane;
#pragma unroll 1
    for (int c0 = 64 * half; c0 < 64 * half + 64; c0 += 16) {
      float v[16];
      if (nk > 0) {
        tmem_ld16(tmem + ((uint32_t)(32 * quad) << 16) + (uint32_t)c0, v);
      } else {
#pragma unroll
        for (int c = 0; c < 16; ++c) v[c] = 0.0f;
      }
      if (gi < n) {
#pragma unroll
        for (int c = 0; c < 16; ++c) {
          const int gj = j0 + c0 + c;
          if (gj < n) {
            double* p = Cb + mo + (long long)gi * n + gj;
            *p = beta == 0.0 ? alpha * (double)v[c] : alpha * (double)v[c] + beta * (*p);
          }
        }
      }
    }
    // the next tile's first MMA overwrites the accumulator: all reads done first
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  }
  // a wait ran out: the structure of the tile in work is marked failed
  if (abort_flag && tid == 0 && status && cur >= 0) status[cur] = kStEigenFailed;
  // let any MMAs still in flight finish before the accumulator is released (bounded)
  for (int st = 0; st < 2; ++st)
    if (uses[st] > 0) mbar_wait(&mbar[st], (uses[st] - 1) & 1);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTmemCols));
}

size_t gemm_tc_smem_bytes() { return 2 * (size_t)kStageBytes + 1024; }

}  // namespace tb
