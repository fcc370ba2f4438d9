// Batched FP64 dense linear algebra for uneven structure sizes:
//  * k_cholesky / k_trinv: S = L L^T and X = L^-T (once per structure);
//  * k_gemm: C = alpha op(A) diag(ks) op(B) + beta C over a tile list;
//  * k_syev: symmetric eigenproblem, one CTA per structure (Householder
//    tridiagonalisation, explicit Q, implicit QL with the rotations of each
//    sweep applied to the eigenvector rows by all threads, rank-based sort).
// Together these give sygvd (itype 1, jobz 'V'; reference src/lapack/sygvd.h:4-23):
// H C = S C e  <=>  (X^T H X) Z = Z e, C = X Z.
#include "tb_common.cuh"
#include "tb_kernels.h"

namespace tb {

// ------------------------------------------------------------ Cholesky
// Left-looking Cholesky of the structure's overlap S (row-major), result
// stored column-major in W (W[k][i] = L[i][k], i >= k), kFactorGroup columns
// at a time: every row i of the group's columns is first updated with all
// finished columns k < j0 (each W[k][i] read once per group, the group's
// entries W[k][j0..] broadcast), then the group is finished column by column
// with the in-group terms.  Reads of the finished part drop by the group size
// against a column-at-a-time walk.  The group's entries of the finished
// columns, which every row needs, are staged in shared memory kFactorChunk
// columns at a time; the accumulation order is that of a plain loop over k.
constexpr int kFactorGroup = 16;
constexpr int kFactorChunk = 128;  // values of k staged in shared memory per round

__global__ void k_cholesky(DevBatch B, const double* __restrict__ S, double* __restrict__ W,
                           int* __restrict__ status, const int* __restrict__ active) {
  constexpr int G = kFactorGroup, KC = kFactorChunk;
  __shared__ __align__(16) double ws[KC][G];  // ws[k - kc0][q] = W[k][j0 + q] = L[j0 + q][k]
  const int m = B.order ? B.order[blockIdx.x] : blockIdx.x;
  if (active && !active[m]) return;
  const int n = B.ooff[m + 1] - B.ooff[m];
  if (on_library(B, n)) return;
  const long long mo = B.moff[m];
  const double* s = S + mo;
  double* w = W + mo;
  const int tid = threadIdx.x, nt = blockDim.x;
  __shared__ double ljj;
  __shared__ int bad;
  if (tid == 0) bad = 0;
  __syncthreads();
  for (int j0 = 0; j0 < n; j0 += G) {
    const int gq = min(G, n - j0);
    for (int i0 = j0; i0 < n; i0 += nt) {
      const int i = i0 + tid;  // threads past the last row still stage and wait
      double acc[G];
#pragma unroll
      for (int q = 0; q < G; ++q) acc[q] = (q < gq && i < n) ? s[(long long)(j0 + q) * n + i] : 0.0;
      for (int kc0 = 0; kc0 < j0; kc0 += KC) {
        const int kn = min(KC, j0 - kc0);
        __syncthreads();  // the previous chunk has been read
        for (int e = tid; e < kn * G; e += nt) {
          const int kk = e / G, q = e - kk * G;
          ws[kk][q] = q < gq ? w[(long long)(kc0 + kk) * n + j0 + q] : 0.0;
        }
        __syncthreads();
        if (i < n)
          for (int kk = 0; kk < kn; ++kk) {
            const double a = w[(long long)(kc0 + kk) * n + i];
#pragma unroll
            for (int q = 0; q < G; ++q)
              if (q < gq) acc[q] -= a * ws[kk][q];
          }
      }
      if (i < n) {
#pragma unroll
        for (int q = 0; q < G; ++q)
          if (q < gq) w[(long long)(j0 + q) * n + i] = acc[q];
      }
    }
    __syncthreads();
    for (int q = 0; q < gq; ++q) {
      const int j = j0 + q;
      if (tid == 0) {
        double d = w[(long long)j * n + j];
        for (int p = 0; p < q; ++p) {
          const double l = w[(long long)(j0 + p) * n + j];
          d -= l * l;
        }
        if (!(d > 0.0)) { bad = 1; ljj = 1.0; } else ljj = sqrt(d);
        w[(long long)j * n + j] = ljj;
      }
      __syncthreads();
      if (bad) break;
      const double inv = 1.0 / ljj;
      for (int i = j + 1 + tid; i < n; i += nt) {
        double t = w[(long long)j * n + i];
        for (int p = 0; p < q; ++p) t -= w[(long long)(j0 + p) * n + i] * w[(long long)(j0 + p) * n + j];
        w[(long long)j * n + i] = t * inv;
      }
      __syncthreads();
    }
    if (bad) break;
  }
  if (tid == 0 && bad) status[m] = kStNotSpd;
}

// X = L^-T (upper triangular, row-major): column c solves L^T x = e_c by
// backward substitution, kFactorGroup rows at a time from the bottom: the
// group's rows are first reduced with every finished row below it (each
// X[k][c] read once per group), then solved upwards inside the group.  Each
// thread owns a column; the group's rows of W (the L entries every column
// needs) are staged in shared memory kFactorChunk values of k at a time, so
// the inner loop reads them at shared-memory rather than L2 latency.  The
// accumulation order is that of a plain loop over k, so X does not depend on
// the staging.
__global__ void k_trinv(DevBatch B, const double* __restrict__ W, double* __restrict__ X,
                        const int* __restrict__ status) {
  constexpr int G = kFactorGroup, KC = kFactorChunk;
  __shared__ double ws[G][KC];  // ws[q][k - kc0] = W[r1 - q][k]
  const int m = B.order ? B.order[blockIdx.x] : blockIdx.x;
  if (status[m] != kStOk) return;
  const int n = B.ooff[m + 1] - B.ooff[m];
  if (on_library(B, n)) return;
  const long long mo = B.moff[m];
  const double* w = W + mo;
  double* x = X + mo;
  for (int c0 = 0; c0 < n; c0 += blockDim.x) {
    const int c = c0 + threadIdx.x;  // threads past the last column still stage and wait
    const int chi = min(n, c0 + (int)blockDim.x) - 1;  // the round's largest column
    for (int r1 = n - 1; r1 >= 0; r1 -= G) {
      const int gq = min(G, r1 + 1);
      double acc[G];
#pragma unroll
      for (int q = 0; q < G; ++q) acc[q] = (q < gq && r1 - q == c) ? 1.0 : 0.0;
      for (int kc0 = r1 + 1; kc0 <= chi; kc0 += KC) {
        const int kn = min(KC, chi + 1 - kc0);
        __syncthreads();  // the previous chunk has been read
        for (int e = threadIdx.x; e < gq * kn; e += blockDim.x) {
          const int q = e / kn, kk = e - q * kn;
          ws[q][kk] = w[(long long)(r1 - q) * n + kc0 + kk];  // W[r][k] = L[k][r]
        }
        __syncthreads();
        const int kend = c < n ? min(kn, c + 1 - kc0) : 0;  // X[k][c] = 0 for k > c
        for (int kk = 0; kk < kend; ++kk) {
          const double xk = x[(long long)(kc0 + kk) * n + c];
#pragma unroll
          for (int q = 0; q < G; ++q)
            if (q < gq) acc[q] -= ws[q][kk] * xk;
        }
      }
      if (c >= n) continue;
      double xg[G];
#pragma unroll
      for (int q = 0; q < G; ++q) {
        if (q >= gq) break;
        const int r = r1 - q;
        double t = acc[q];
        for (int p = 0; p < q; ++p) t -= w[(long long)r * n + (r1 - p)] * xg[p];
        xg[q] = r > c ? 0.0 : t / w[(long long)r * n + r];
      }
#pragma unroll
      for (int q = 0; q < G; ++q)
        if (q < gq) x[(long long)(r1 - q) * n + c] = xg[q];
    }
  }
}

// ------------------------------------------------------------ batched GEMM
// C_m = alpha * op(A_m) * diag(ks_m) * op(B_m) + beta * C_m for every tile in
// the list (structure, tile row, tile col).  Square n_m x n_m operands with
// leading dimension n_m at offset moff[m]; K = kdim[m] if kdim != NULL.
// op(B) may gather its columns through perm (eigenvector reordering).
// `shape` skips known zeros and redundant tiles: kGemmKUpToJ (op(B) upper
// triangular: only k < the tile's last column), kGemmKUpToI (op(A) lower
// triangular: k < its last row), kGemmKFromI (op(A) upper triangular: k >=
// its first row), kGemmSym (C symmetric: tiles below the diagonal are
// skipped, and each element of the upper triangle is computed once and also
// written to its mirror).
// TILE x TILE tiles (64 or 32) on the FP64 tensor instruction
// mma.sync.m8n8k4.f64: four warps, each owning a quarter of the tile as
// (TILE/16) x (TILE/16) fragments of 8 x 8.  K slabs of 16 are staged by
// cp.async in a two-stage ring (zero fill past the matrix edge); the shared
// tiles are padded by 4 doubles so the 64-bit fragment loads of a half-warp
// hit 16 distinct bank pairs.  Every output element accumulates over k in the
// same order (slabs starting at multiples of 16, then the four k-steps of the
// instruction) whatever the tile; the k ranges that only one tile size skips
// hold exact zeros of the triangular operand, which leave a sum unchanged.
// So the two tile sizes give the same bits, and the autotuner picks the tile
// per structure size (k_gemm: 64, k_gemm32: 32).
constexpr int GK = 16;
static_assert(kGemmThreads == 128, "k_gemm assumes four warps");

namespace {
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, bool valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  const int n = valid ? 8 : 0;  // bytes read; the rest of the 8 is zero-filled
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }
// D = A B + D for one 8 x 8 x 4 step.  Lane l = 4 g + t holds A[g][t], B[t][g]
// and D[g][2t], D[g][2t+1].
__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

template <int GT>
__device__ __forceinline__ void gemm_body(const DevBatch& B, const int4* __restrict__ tiles, int ntiles,
                                          const double* __restrict__ Ab, int ta, const double* __restrict__ Bb,
                                          int tb_, const int* __restrict__ perm, const double* __restrict__ ks,
                                          const int* __restrict__ kdim, double* __restrict__ Cb, double alpha,
                                          double beta, const int* __restrict__ active, int shape) {
  constexpr int GP = GT + 4, FX = GT / 16;  // padded row; fragments per warp and dimension
  constexpr int RA = GT / 8;                // slab elements of op(A) (and of op(B)) per thread
  constexpr int TSH = GT == 64 ? 6 : 5;     // log2(GT)
  __shared__ __align__(16) double As[2][GK][GP];
  __shared__ __align__(16) double Bs[2][GK][GP];
  __shared__ __align__(16) double Ks[2][GK];
  __shared__ int colS[GT];  // columns of op(B) for this tile (through perm)
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, tg = lane & 3;                          // fragment coordinates
  const int wr = (warp >> 1) * (GT / 2), wc = (warp & 1) * (GT / 2);  // this warp's quarter of the tile
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int4 tl = tiles[t];
    const int m = tl.x;
    if (active && !active[m]) continue;
    if ((shape & kGemmSym) && tl.z < tl.y) continue;
    const int n = B.ooff[m + 1] - B.ooff[m];
    // the reduction length never leaves [0, n], whatever kdim holds
    const int K = kdim ? min(max(kdim[m], 0), n) : n;
    const long long mo = B.moff[m];
    const long long vo = B.ooff[m];
    const double* A = Ab + mo;
    const double* Bm = Bb + mo;
    const int* pm = perm ? perm + vo : nullptr;
    const double* kv = ks ? ks + vo : nullptr;
    const int i0 = tl.y * GT, j0 = tl.z * GT;
    int klo = 0, khi = K;
    if (shape & kGemmKUpToJ) khi = min(khi, j0 + GT);
    if (shape & kGemmKUpToI) khi = min(khi, i0 + GT);
    if (shape & kGemmKFromI) klo = min(i0, K);
    double acc[FX][FX][2];
#pragma unroll
    for (int a = 0; a < FX; ++a)
#pragma unroll
      for (int b = 0; b < FX; ++b) acc[a][b][0] = acc[a][b][1] = 0.0;
    __syncthreads();  // colS and the ring of the previous tile are free
    if (tid < GT) colS[tid] = pm ? (j0 + tid < n ? pm[j0 + tid] : 0) : j0 + tid;
    __syncthreads();
    // Element r of a slab for this thread:
    //   op(A) not transposed: kk = tid & 15, ii = (tid >> 4) + 8 r;  transposed: ii = tid & (GT-1), kk = (tid >> log2 GT) + (128/GT) r
    //   op(B) not transposed: jj = tid & (GT-1), kb = (tid >> log2 GT) + (128/GT) r;  transposed: kb = tid & 15, jj = (tid >> 4) + 8 r
    const int lo16 = tid & 15, hi8 = tid >> 4, loT = tid & (GT - 1), hiT = tid >> TSH;
    constexpr int SK = kGemmThreads / GT;  // k step of the transposed loads
    auto issue = [&](int buf, int k0) {
      if (!ta) {
        const int gk = k0 + lo16;
#pragma unroll
        for (int r = 0; r < RA; ++r) {
          const int gi = i0 + hi8 + 8 * r;
          const bool v = gi < n && gk < K;
          cp_async8(&As[buf][lo16][hi8 + 8 * r], v ? A + (long long)gi * n + gk : A, v);
        }
      } else {
        const int gi = i0 + loT;
#pragma unroll
        for (int r = 0; r < RA; ++r) {
          const int gk = k0 + hiT + SK * r;
          const bool v = gi < n && gk < K;
          cp_async8(&As[buf][hiT + SK * r][loT], v ? A + (long long)gk * n + gi : A, v);
        }
      }
      if (!tb_) {
        const bool vj = j0 + loT < n;
        const int col = colS[loT];
#pragma unroll
        for (int r = 0; r < RA; ++r) {
          const int gk = k0 + hiT + SK * r;
          const bool v = vj && gk < K;
          cp_async8(&Bs[buf][hiT + SK * r][loT], v ? Bm + (long long)gk * n + col : Bm, v);
        }
      } else {
        const int gk = k0 + lo16;
#pragma unroll
        for (int r = 0; r < RA; ++r) {
          const int jj = hi8 + 8 * r;
          const bool v = j0 + jj < n && gk < K;
          cp_async8(&Bs[buf][lo16][jj], v ? Bm + (long long)colS[jj] * n + gk : Bm, v);
        }
      }
      if (kv && tid < GK) cp_async8(&Ks[buf][tid], k0 + tid < K ? kv + k0 + tid : kv, k0 + tid < K);
      cp_async_commit();
    };
    const int nk = khi > klo ? (khi - klo + GK - 1) / GK : 0;
    if (nk > 0) issue(0, klo);
    for (int kt = 0; kt < nk; ++kt) {
      const int cur = kt & 1;
      if (kt + 1 < nk) {
        issue(cur ^ 1, klo + (kt + 1) * GK);
        cp_async_wait<1>();
      } else {
        cp_async_wait<0>();
      }
      __syncthreads();
      if (kv) {  // diag(ks) between the factors: scale the slab of op(B) once
        for (int e = tid; e < GK * GT; e += kGemmThreads) Bs[cur][e / GT][e % GT] *= Ks[cur][e / GT];
        __syncthreads();
      }
#pragma unroll
      for (int k4 = 0; k4 < GK; k4 += 4) {
        double af[FX], bf[FX];
#pragma unroll
        for (int x = 0; x < FX; ++x) af[x] = As[cur][k4 + tg][wr + 8 * x + g];
#pragma unroll
        for (int y = 0; y < FX; ++y) bf[y] = Bs[cur][k4 + tg][wc + 8 * y + g];
#pragma unroll
        for (int x = 0; x < FX; ++x)
#pragma unroll
          for (int y = 0; y < FX; ++y) dmma(acc[x][y][0], acc[x][y][1], af[x], bf[y]);
      }
      __syncthreads();  // buffer cur is refilled two slabs later
    }
#pragma unroll
    for (int x = 0; x < FX; ++x) {
      const int gi = i0 + wr + 8 * x + g;
      if (gi >= n) continue;
#pragma unroll
      for (int y = 0; y < FX; ++y) {
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int gj = j0 + wc + 8 * y + 2 * tg + h;
          if (gj >= n) continue;
          // symmetric result: the upper triangle is computed and mirrored, so
          // no element depends on which tile it fell in
          if ((shape & kGemmSym) && gi > gj) continue;
          if (!TB_GUARD(8, (long long)gi * n + gj, 0, (long long)n * n)) continue;
          double* c = Cb + mo + (long long)gi * n + gj;
          const double r = beta == 0.0 ? alpha * acc[x][y][h] : alpha * acc[x][y][h] + beta * (*c);
          *c = r;
          if ((shape & kGemmSym) && gi != gj) Cb[mo + (long long)gj * n + gi] = r;
        }
      }
    }
  }
}
}  // namespace

__global__ void __launch_bounds__(kGemmThreads) k_gemm(DevBatch B, const int4* __restrict__ tiles, int ntiles,
                                                       const double* __restrict__ Ab, int ta,
                                                       const double* __restrict__ Bb, int tb_,
                                                       const int* __restrict__ perm, const double* __restrict__ ks,
                                                       const int* __restrict__ kdim, double* __restrict__ Cb,
                                                       double alpha, double beta, const int* __restrict__ active,
                                                       int shape) {
  gemm_body<64>(B, tiles, ntiles, Ab, ta, Bb, tb_, perm, ks, kdim, Cb, alpha, beta, active, shape);
}

__global__ void __launch_bounds__(kGemmThreads) k_gemm32(DevBatch B, const int4* __restrict__ tiles, int ntiles,
                                                         const double* __restrict__ Ab, int ta,
                                                         const double* __restrict__ Bb, int tb_,
                                                         const int* __restrict__ perm, const double* __restrict__ ks,
                                                         const int* __restrict__ kdim, double* __restrict__ Cb,
                                                         double alpha, double beta, const int* __restrict__ active,
                                                         int shape) {
  gemm_body<32>(B, tiles, ntiles, Ab, ta, Bb, tb_, perm, ks, kdim, Cb, alpha, beta, active, shape);
}

// ------------------------------------------------------------ eigensolver
// Symmetric eigenproblem of A (n x n, row-major, overwritten) for every
// active structure, one CTA of 256 threads per structure: w ascending,
// eigenvector j = row perm[j] of Zc (n x n, one eigenvector per row).
//
//  1. Householder tridiagonalisation in panels (tridiagonalise): within a
//     panel the trailing block keeps its value from the panel start, each
//     step forms its product with one read-only walk and corrects it with the
//     panel's pairs; the panel-closing walk applies the rank-2 width update
//     fused with the next product.  Walks read row segments (colwalk); with
//     a scratch matrix (FP64) they read only the upper triangle (symwalk,
//     panel_walk_tc_sym, the latter on the FP64 tensor instruction).
//     Reflector k is kept in row k of A.
//  2. Zc = Q^T accumulated backwards in compact-WY blocks of kQBlock
//     reflectors (form_q; FP64 with a scratch matrix: formq_block_tc, 64-row
//     tiles on the FP64 tensor instruction).
//  3. Tridiagonal eigenproblem: divide and conquer (dc_solve) for FP64
//     structures of kDcMin+ rows with a scratch matrix, else implicit QL
//     with Wilkinson shift (warp 0 runs the rotation chain, warps 1.. apply
//     sweeps to Zc through a kRing-slot shared-memory ring; every wait is
//     bounded, on timeout the structure is marked failed).
//  4. Ascending order by rank (ties by index).
namespace {

// Tridiagonalisation panel: reflectors per panel (2 panel n <= ring) and, for
// the FP32 column form of the panel-closing walk, rows per load batch.  FP64
// moves twice the bytes per element, so its walks are traffic-bound and wide
// panels pay (its panel-closing walk is panel_walk_tc / panel_walk_tc_sym); in
// FP32 a panel of one (each step's update fused with the next product) is as fast.
template <typename T> struct PanelCfg;
template <> struct PanelCfg<double> { static constexpr int width = 8; };
template <> struct PanelCfg<float> { static constexpr int width = 1, batch = 12; };
// Read-only Householder walk (colwalk): the warps form kWalkRowGroups row
// groups (interleaved rows) times nw / kWalkRowGroups column groups; a lane
// holds `cols` columns (32 apart) of its group's strip and loads `rows` rows
// of them before using any, so a warp reads whole row segments (contiguous
// for DRAM) with cols * rows loads in flight per lane.
constexpr int kWalkRowGroups = 4;
template <typename T> struct WalkCfg { static constexpr int cols = 3, rows = 4; };
static_assert(PanelCfg<double>::width <= kRing && PanelCfg<float>::width <= kRing, "panel exceeds the ring");
constexpr int kQBlock = 16;     // reflectors per compact-WY block of the Q accumulation
constexpr int kWaveK = 4;            // QL sweeps applied per pass over Zc
constexpr int kWin = 2 * kWaveK;     // rows of Zc in flight per column
constexpr long long kSpinLimit = 1LL << 24;

template <typename T> struct Eps;
template <> struct Eps<double> { static constexpr double v = 2.220446049250313e-16; };
template <> struct Eps<float> { static constexpr float v = 1.1920929e-07f; };
__device__ inline double tb_sqrt(double x) { return sqrt(x); }
__device__ inline float tb_sqrt(float x) { return sqrtf(x); }
__device__ inline double tb_abs(double x) { return fabs(x); }
__device__ inline float tb_abs(float x) { return fabsf(x); }
// one Newton step y(3 - x y^2)/2 on the hardware estimate keeps Givens pairs orthogonal to ~1 ulp
__device__ inline float tb_rsqrt(float x) {
  const float y = rsqrtf(x);
  return y * (1.5f - 0.5f * x * y * y);
}

// reciprocal square root on the QL rotation chain (FP32: one Newton step on the estimate)
__device__ inline double chain_rsqrt(double x) { return rsqrt(x); }

// 1/x for the divide-and-conquer inner loops: the hardware reciprocal
// estimate (rcp.approx.ftz.f64) refined by two Newton-Raphson steps for
// f(r) = 1/r - x, r <- r + r (1 - x r), each squaring the relative error;
// within a few units in the last place, not correctly rounded.  x = 0 gives
// inf and |x| = inf gives 0, as 1/x does.  FP32 keeps the division.
__device__ inline double dc_rcp(double x) {
  double r;
  asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(x));
  if (r == 0.0 || isinf(r)) return r;
  double e = fma(-x, r, 1.0);
  r = fma(r, e, r);
  e = fma(-x, r, 1.0);
  return fma(r, e, r);
}
__device__ inline float dc_rcp(float x) { return 1.0f / x; }
__device__ inline float chain_rsqrt(float x) { return tb_rsqrt(x); }

template <typename T>
__device__ inline T block_sum_syev(T v, T* red) { return block_sum(v, red); }

// Householder reflector of row k: x = A[k][k+1..n-1] -> tau[k], e[k] and v
// (v[0] = 1), written to `v` and back into row k.
template <typename T>
__device__ void reflector(T* A, int n, int k, T* v, T* tau, T* e, T* red, T* sh) {
  const int tid = threadIdx.x, nt = blockDim.x;
  const int mm = n - k - 1;
  T* rowk = A + (long long)k * n + k + 1;
  T part = T(0);
  for (int i = 1 + tid; i < mm; i += nt) part += rowk[i] * rowk[i];
  const T sigma = block_sum_syev(part, red);
  if (tid == 0) {
    const T alpha = rowk[0];
    if (sigma == T(0)) {
      tau[k] = T(0); e[k] = alpha; sh[0] = T(0); sh[1] = T(0);
    } else {
      const T r = tb_sqrt(alpha * alpha + sigma);
      const T beta = alpha <= T(0) ? r : -r;
      tau[k] = (beta - alpha) / beta;
      e[k] = beta;
      sh[0] = tau[k];
      sh[1] = T(1) / (alpha - beta);
    }
  }
  __syncthreads();
  const T scal = sh[1];
  const bool refl = sh[0] != T(0);
  for (int i = tid; i < mm; i += nt) {
    const T x = i == 0 ? T(1) : (refl ? rowk[i] * scal : T(0));
    v[i] = x;
    if (refl) rowk[i] = x;
  }
  __syncthreads();
}

// Rows of a walk over an nm-column block are split in two halves (separate
// threads, partial sums added at the end) when that shortens the slowest
// thread's walk by more than an eighth: it walks ceil(nm/nt) whole columns,
// or ceil(2nm/nt) halves.  True for nm <= nt/2 (idle warps otherwise) and for
// the ranges of nm where a last partial round of whole columns would run.
__device__ inline bool walk_split(int nm, int nt) {
  const int whole = (nm + nt - 1) / nt * nm, halves = (2 * nm + nt - 1) / nt * ((nm + 1) >> 1);
  return 8 * halves < 7 * whole;
}

// Read-only walk over the square block r0..r0+nm-1 (rows and columns) of a
// row-major matrix M: out_c = scale * sum_r M[r][c] x_{r-r0}.  Row group g
// (warps g, g + kWalkRowGroups, ...) sums rows g, g + kWalkRowGroups, ... into
// its own partial vector (group 0: out, groups 1..3: p1, p2, p3, nm entries
// each, distinct from x and out); the partials are added at the end in a fixed
// order, so the result is deterministic.  Needs a multiple of kWalkRowGroups
// warps.  Kept out of line (as is panel_walk) so that its load registers are
// allocated apart from the rest of the eigensolver.
template <typename T>
__device__ __noinline__ void colwalk(const T* M, int n, int r0, int nm, const T* x, T* out, T scale, T* p1, T* p2,
                                     T* p3) {
  constexpr int kJ = WalkCfg<T>::cols, kR = WalkCfg<T>::rows, kG = kWalkRowGroups;
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5;
  const int ncg = (nt >> 5) / kG, rg = warp % kG, cg = warp / kG;
  const int strip = 32 * kJ * ncg;  // columns per pass
  T* mine = rg == 0 ? out : (rg == 1 ? p1 : (rg == 2 ? p2 : p3));
  const T* Mb = M + (long long)r0 * n + r0;
  for (int c0 = 0; c0 < nm; c0 += strip) {
    const int cb = c0 + cg * 32 * kJ + lane;
    T acc[kJ];
#pragma unroll
    for (int j = 0; j < kJ; ++j) acc[j] = T(0);
    for (int rb = rg; rb < nm; rb += kG * kR) {
      T q[kR][kJ];
#pragma unroll
      for (int u = 0; u < kR; ++u)
#pragma unroll
        for (int j = 0; j < kJ; ++j) {
          const int r = rb + kG * u, c = cb + 32 * j;
          q[u][j] = (r < nm && c < nm) ? Mb[(long long)r * n + c] : T(0);
        }
#pragma unroll
      for (int u = 0; u < kR; ++u) {
        const int r = rb + kG * u;
        const T xr = r < nm ? x[r] : T(0);
#pragma unroll
        for (int j = 0; j < kJ; ++j) acc[j] += q[u][j] * xr;
      }
    }
#pragma unroll
    for (int j = 0; j < kJ; ++j) {
      const int c = cb + 32 * j;
      if (c < nm) mine[c] = acc[j];
    }
  }
  __syncthreads();
  for (int c = tid; c < nm; c += nt) out[c] = scale * (((out[c] + p1[c]) + p2[c]) + p3[c]);
}

// The same product as colwalk from the upper triangle of the block only
// (half the bytes): with U the upper triangle including the diagonal,
// out = scale (U^T x + (U - diag) x).  Warp w takes rows w, w + 8, ...: for
// each strip of 32 kSymCols columns a lane loads the upper part of kSymRows
// of its rows at a time; the column products go to the warp's own vector
// gp[w][.] (global scratch, 8 nm entries), the row products are reduced
// across the warp and added to out[r] (the row's owner warp only), then
// out_c = scale (out_c + sum_w gp[w][c]) in a fixed order.  FP64, 8 warps.
constexpr int kSymCols = 3, kSymRows = 4;
constexpr int kSymMin = 96;  // structures of more AOs take the upper-triangle walks (scratch of 8n <= n^2)
__device__ __noinline__ void symwalk(const double* M, int n, int r0, int nm, const double* x, double* out, double scale,
                                     double* gp) {
  static_assert(kSymRows == 4, "the row reduction below pairs four rows");
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5;
  const double* Mb = M + (long long)r0 * n + r0;
  for (int c = tid; c < nm; c += nt) out[c] = 0.0;
  __syncthreads();
  for (int cs = 0; cs < nm; cs += 32 * kSymCols) {
    const int ce = min(cs + 32 * kSymCols, nm);
    double xs[kSymCols], acc[kSymCols];
#pragma unroll
    for (int j = 0; j < kSymCols; ++j) {
      const int c = cs + lane + 32 * j;
      xs[j] = c < nm ? x[c] : 0.0;
      acc[j] = 0.0;
    }
    for (int rb = warp; rb < ce; rb += 8 * kSymRows) {
      double a[kSymRows][kSymCols];
#pragma unroll
      for (int u = 0; u < kSymRows; ++u)
#pragma unroll
        for (int j = 0; j < kSymCols; ++j) {
          const int r = rb + 8 * u, c = cs + lane + 32 * j;
          a[u][j] = (r < ce && c >= r && c < nm) ? Mb[(long long)r * n + c] : 0.0;
        }
      double v[kSymRows];
#pragma unroll
      for (int u = 0; u < kSymRows; ++u) {
        const int r = rb + 8 * u;
        const double xr = r < nm ? x[r] : 0.0;
        v[u] = 0.0;
#pragma unroll
        for (int j = 0; j < kSymCols; ++j) {
          const int c = cs + lane + 32 * j;
          acc[j] += a[u][j] * xr;
          if (c > r) v[u] += a[u][j] * xs[j];
        }
      }
      // the four row sums across the warp: halves exchange pairs (xor 16),
      // quarters exchange one (xor 8), then a butterfly over the last 3 bits;
      // lane 8u ends with the total of row u
      const bool h16 = lane & 16, h8 = lane & 8;
      double k0 = h16 ? v[2] : v[0], k1 = h16 ? v[3] : v[1];
      k0 += __shfl_xor_sync(0xffffffffu, h16 ? v[0] : v[2], 16);
      k1 += __shfl_xor_sync(0xffffffffu, h16 ? v[1] : v[3], 16);
      double k = h8 ? k1 : k0;
      k += __shfl_xor_sync(0xffffffffu, h8 ? k0 : k1, 8);
      k += __shfl_xor_sync(0xffffffffu, k, 4);
      k += __shfl_xor_sync(0xffffffffu, k, 2);
      k += __shfl_xor_sync(0xffffffffu, k, 1);
      if ((lane & 7) == 0) {
        const int r = rb + 8 * (lane >> 3);
        if (r < ce) out[r] += k;
      }
    }
#pragma unroll
    for (int j = 0; j < kSymCols; ++j) {
      const int c = cs + lane + 32 * j;
      if (c < nm) gp[(long long)warp * nm + c] = acc[j];
    }
  }
  __syncthreads();
  for (int c = tid; c < nm; c += nt) {
    double t = out[c];
#pragma unroll
    for (int w = 0; w < 8; ++w) t += gp[(long long)w * nm + c];
    out[c] = scale * t;
  }
}

// Closing walk of a tridiagonalisation panel over rows and columns
// r0..r0+nm-1 (both relative to the matrix origin, the block is square):
// M -= sum_i PV_i PW_i^T + PW_i PV_i^T over the panel's pairs (absolute
// index), and out_c = scale * sum_r M_new[r][c] x_{r-r0}.  One thread per
// column (or column half, see walk_split) keeps its column's pair entries in
// registers.
template <typename T>
__device__ __noinline__ void panel_walk(T* M, int n, int r0, int nm, const T* PV, const T* PW, const T* x, T* out,
                                        T scale, T* part) {
  constexpr int kPanel = PanelCfg<T>::width, kPanelBatch = PanelCfg<T>::batch;
  const int tid = threadIdx.x, nt = blockDim.x;
  const bool split = walk_split(nm, nt);
  const int half = split ? (nm + 1) >> 1 : nm, nunit = split ? 2 * nm : nm;
  for (int un = tid; un < nunit; un += nt) {
    const int h = un >= nm, jj = h ? un - nm : un;
    const int rb = h ? half : 0, re = h ? nm : half;
    const int c = r0 + jj;
    T vc[kPanel], wc[kPanel];
#pragma unroll
    for (int i = 0; i < kPanel; ++i) {
      vc[i] = PV[(long long)i * n + c];
      wc[i] = PW[(long long)i * n + c];
    }
    T acc = T(0);
    for (int i0 = rb; i0 < re; i0 += kPanelBatch) {
      T q[kPanelBatch];
#pragma unroll
      for (int u = 0; u < kPanelBatch; ++u)
        q[u] = (i0 + u < re) ? M[(long long)(r0 + i0 + u) * n + c] : T(0);
#pragma unroll
      for (int u = 0; u < kPanelBatch; ++u) {
        if (i0 + u < re) {
          const int rr = r0 + i0 + u;
          T y = q[u];
#pragma unroll
          for (int i = 0; i < kPanel; ++i) y -= PV[(long long)i * n + rr] * wc[i] + PW[(long long)i * n + rr] * vc[i];
          M[(long long)rr * n + c] = y;
          acc += y * x[i0 + u];
        }
      }
    }
    if (h) part[jj] = acc;
    else out[jj] = split ? acc : scale * acc;
  }
  if (split) {
    __syncthreads();
    for (int jj = tid; jj < nm; jj += nt) out[jj] = scale * (out[jj] + part[jj]);
  }
}

// FP64 panel-closing walk on the tensor instruction (mma.sync m8n8k4), same
// result as panel_walk up to rounding: with the panel's 8 pairs as
// K = [PV; PW] (16 x n) and L = [PW; PV], the block is updated as
// M -= K^T L over 16 x 32 tiles per warp (accumulators initialised from M,
// stored back), and out_c = scale * sum_r M_new[r][c] x_{r-r0} is formed from
// the same fragments.  Warps as in colwalk: kWalkRowGroups groups of
// interleaved 16-row tiles times nw / kWalkRowGroups column groups; the row
// groups' partial sums go through out, p1, p2, p3 (nm entries each).
__device__ __noinline__ void panel_walk_tc(double* M, int n, int r0, int nm, const double* PV, const double* PW,
                                           const double* x, double* out, double scale, double* p1, double* p2,
                                           double* p3) {
  static_assert(PanelCfg<double>::width == 8, "two panel halves of four k-steps");
  constexpr int kG = kWalkRowGroups;
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, t = lane & 3;
  const int ncg = (nt >> 5) / kG, rg = warp % kG, cg = warp / kG;
  double* mine = rg == 0 ? out : (rg == 1 ? p1 : (rg == 2 ? p2 : p3));
  double* Mb = M + (long long)r0 * n + r0;
  for (int c0 = 0; c0 < nm; c0 += 32 * ncg) {
    const int cw = c0 + 32 * cg;  // this warp's first column (relative)
    for (int rt = 16 * rg; rt < nm; rt += 16 * kG) {
      double d[2][4][2];
#pragma unroll
      for (int xx = 0; xx < 2; ++xx)
#pragma unroll
        for (int y = 0; y < 4; ++y)
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int r = rt + 8 * xx + g, c = cw + 8 * y + 2 * t + h;
            d[xx][y][h] = (r < nm && c < nm) ? Mb[(long long)r * n + c] : 0.0;
          }
#pragma unroll
      for (int ks = 0; ks < 4; ++ks) {
        const int k = 4 * (ks & 1) + t;                                 // pair index
        const double* Kr = (ks < 2 ? PV : PW) + (long long)k * n + r0;  // row side
        const double* Lc = (ks < 2 ? PW : PV) + (long long)k * n + r0;  // column side
        double a[2], b[4];
#pragma unroll
        for (int xx = 0; xx < 2; ++xx) {
          const int r = rt + 8 * xx + g;
          a[xx] = r < nm ? -Kr[r] : 0.0;
        }
#pragma unroll
        for (int y = 0; y < 4; ++y) {
          const int c = cw + 8 * y + g;
          b[y] = c < nm ? Lc[c] : 0.0;
        }
#pragma unroll
        for (int xx = 0; xx < 2; ++xx)
#pragma unroll
          for (int y = 0; y < 4; ++y) dmma(d[xx][y][0], d[xx][y][1], a[xx], b[y]);
      }
      const double x0 = rt + g < nm ? x[rt + g] : 0.0, x1 = rt + 8 + g < nm ? x[rt + 8 + g] : 0.0;
#pragma unroll
      for (int xx = 0; xx < 2; ++xx)
#pragma unroll
        for (int y = 0; y < 4; ++y)
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int r = rt + 8 * xx + g, c = cw + 8 * y + 2 * t + h;
            if (r < nm && c < nm) Mb[(long long)r * n + c] = d[xx][y][h];
          }
      // this tile's column sums over its 16 rows (the eight row lanes g are
      // lanes t, t + 4, ..., t + 28), added to the warp's own entries of `mine`
#pragma unroll
      for (int y = 0; y < 4; ++y)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          double v = d[0][y][h] * x0 + d[1][y][h] * x1;
          v += __shfl_xor_sync(0xffffffffu, v, 4);
          v += __shfl_xor_sync(0xffffffffu, v, 8);
          v += __shfl_xor_sync(0xffffffffu, v, 16);
          const int c = cw + 8 * y + 2 * t + h;
          if (g == 0 && c < nm) mine[c] = rt == 16 * rg ? v : mine[c] + v;
        }
    }
    if (16 * rg >= nm)  // a row group without rows still owns its partial entries
      for (int c = cw + lane; c < cw + 32 && c < nm; c += 32) mine[c] = 0.0;
  }
  __syncthreads();
  for (int c = tid; c < nm; c += nt) out[c] = scale * (((out[c] + p1[c]) + p2[c]) + p3[c]);
}

// panel_walk_tc on the upper triangle of the block only (as symwalk for
// colwalk): tiles wholly below the diagonal are skipped, entries below it are
// neither read nor written.  Column products (entries on and above the
// diagonal) and row products (above it) of warp w accumulate in gp[w][.]
// (global scratch, 8 nm entries); out_c = scale sum_w gp[w][c].  Warp tiles
// of 16 x 8 kNY (kNY column fragments): 16 columns measured 5% faster than 32
// in the batch (fewer registers, no stack traffic in the tile loop).
template <int kNY>
__device__ __noinline__ void panel_walk_tc_sym(double* M, int n, int r0, int nm, const double* PV, const double* PW,
                                               const double* x, double* out, double scale, double* gp) {
  constexpr int kG = kWalkRowGroups;
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, t = lane & 3;
  const int ncg = (nt >> 5) / kG, rg = warp % kG, cg = warp / kG;
  double* mine = gp + (long long)warp * nm;
  for (int c = lane; c < nm; c += 32) mine[c] = 0.0;
  __syncwarp();
  double* Mb = M + (long long)r0 * n + r0;
  for (int c0 = 0; c0 < nm; c0 += 8 * kNY * ncg) {
    const int cw = c0 + 8 * kNY * cg;  // this warp's first column (relative)
    if (cw >= nm) continue;
    const int rend = min(nm, cw + 8 * kNY);  // rows with an entry on or above the diagonal in these columns
    for (int rt = 16 * rg; rt < rend; rt += 16 * kG) {
      double d[2][kNY][2];
#pragma unroll
      for (int xx = 0; xx < 2; ++xx)
#pragma unroll
        for (int y = 0; y < kNY; ++y)
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int r = rt + 8 * xx + g, c = cw + 8 * y + 2 * t + h;
            d[xx][y][h] = (r < nm && c < nm && c >= r) ? Mb[(long long)r * n + c] : 0.0;
          }
#pragma unroll
      for (int ks = 0; ks < 4; ++ks) {
        const int k = 4 * (ks & 1) + t;
        const double* Kr = (ks < 2 ? PV : PW) + (long long)k * n + r0;
        const double* Lc = (ks < 2 ? PW : PV) + (long long)k * n + r0;
        double a[2], b[kNY];
#pragma unroll
        for (int xx = 0; xx < 2; ++xx) {
          const int r = rt + 8 * xx + g;
          a[xx] = r < nm ? -Kr[r] : 0.0;
        }
#pragma unroll
        for (int y = 0; y < kNY; ++y) {
          const int c = cw + 8 * y + g;
          b[y] = c < nm ? Lc[c] : 0.0;
        }
#pragma unroll
        for (int xx = 0; xx < 2; ++xx)
#pragma unroll
          for (int y = 0; y < kNY; ++y) dmma(d[xx][y][0], d[xx][y][1], a[xx], b[y]);
      }
      // store the upper entries and drop the others from the products below
#pragma unroll
      for (int xx = 0; xx < 2; ++xx)
#pragma unroll
        for (int y = 0; y < kNY; ++y)
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const int r = rt + 8 * xx + g, c = cw + 8 * y + 2 * t + h;
            if (r < nm && c < nm && c >= r) Mb[(long long)r * n + c] = d[xx][y][h];
            else d[xx][y][h] = 0.0;
          }
      const double x0 = rt + g < nm ? x[rt + g] : 0.0, x1 = rt + 8 + g < nm ? x[rt + 8 + g] : 0.0;
      // row products (strictly above the diagonal) over this tile's columns
      double rp0 = 0.0, rp1 = 0.0;
#pragma unroll
      for (int y = 0; y < kNY; ++y)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int c = cw + 8 * y + 2 * t + h;
          const double xc = c < nm ? x[c] : 0.0;
          if (c > rt + g) rp0 += d[0][y][h] * xc;
          if (c > rt + 8 + g) rp1 += d[1][y][h] * xc;
        }
      // column products over the tile's 16 rows (row lanes g: lanes t + 4g)
#pragma unroll
      for (int y = 0; y < kNY; ++y)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          double v = d[0][y][h] * x0 + d[1][y][h] * x1;
          v += __shfl_xor_sync(0xffffffffu, v, 4);
          v += __shfl_xor_sync(0xffffffffu, v, 8);
          v += __shfl_xor_sync(0xffffffffu, v, 16);
          const int c = cw + 8 * y + 2 * t + h;
          if (g == 0 && c < nm) mine[c] += v;
        }
      __syncwarp();
      rp0 += __shfl_xor_sync(0xffffffffu, rp0, 1);
      rp0 += __shfl_xor_sync(0xffffffffu, rp0, 2);
      rp1 += __shfl_xor_sync(0xffffffffu, rp1, 1);
      rp1 += __shfl_xor_sync(0xffffffffu, rp1, 2);
      if (t == 0) {
        if (rt + g < nm) mine[rt + g] += rp0;
        if (rt + 8 + g < nm) mine[rt + 8 + g] += rp1;
      }
      __syncwarp();
    }
  }
  __syncthreads();
  for (int c = tid; c < nm; c += nt) {
    double v = 0.0;
    for (int w = 0; w < (nt >> 5); ++w) v += gp[(long long)w * nm + c];
    out[c] = scale * v;
  }
}

// One compact-WY block of the Q accumulation on the FP64 tensor instruction
// (mma.sync.m8n8k4): with Zb the rows and columns c0..n-1 of Z (m x m) and Vs
// the block's reflectors (kQBlock x m, shared memory), for each tile of 64
// rows of Zb in turn
//   Wm = Zt Vs^T    (64 x kQBlock; warp w rows 8w..8w+7, slabs of 64 x 8
//                    staged in shared memory and prefetched into registers),
//   Wt = Wm T^T     (64 x kQBlock, four entries per thread),
//   Zt -= Wt Vs     (64 x 64 tiles, each warp 16 x 32 as 2 x 4 fragments,
//                    accumulators initialised with Zt),
// so that a tile is read again by the update while it is still in L2.  Same
// arithmetic as Zc <- Zc - (Zc V) T^T V^T row by row.  Wm and Wt go through
// the global scratch Wq (2 x 64 x kQBlock); stage: 512 nsub elements of
// shared memory (nsub <= kFqSubMax sub-slabs of 8 columns per barrier pair).
// 256 threads.
constexpr int kFqSubMax = 4;  // 8-column sub-slabs staged per barrier pair (at most)
template <typename T, int nsub>
__device__ __noinline__ void formq_block_tc(T* Z, int n, int c0, int m, const T* Vs, const T (*Ts)[kQBlock], T* Wq,
                                            T* stage) {
  if constexpr (sizeof(T) == 8) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, g = lane >> 2, tg = lane & 3;
    T* Zb = Z + (long long)c0 * n + c0;
    T* Wm = Wq;                   // 64 x kQBlock
    T* Wt = Wq + 64 * kQBlock;    // 64 x kQBlock
    const int wrow = (warp >> 1) * 16, wcol = (warp & 1) * 32;
    for (int rt = 0; rt < m; rt += 64) {
      // Wm = Zt Vs^T
      // slabs of nsub x 8 columns per barrier pair (sub-slab j: 64 x 8 at stage + 512 j)
      double a0[2] = {0.0, 0.0}, a1[2] = {0.0, 0.0};
      double pf[2 * nsub];
#pragma unroll
      for (int u = 0; u < 2 * nsub; ++u) {
        const int x = tid + 256 * u, r = rt + ((x & 511) >> 3), c = 8 * (x >> 9) + (x & 7);
        pf[u] = (r < m && c < m) ? Zb[(long long)r * n + c] : 0.0;
      }
      for (int k0 = 0; k0 < m; k0 += 8 * nsub) {
#pragma unroll
        for (int u = 0; u < 2 * nsub; ++u) stage[tid + 256 * u] = pf[u];
        __syncthreads();
        if (k0 + 8 * nsub < m)
#pragma unroll
          for (int u = 0; u < 2 * nsub; ++u) {
            const int x = tid + 256 * u, r = rt + ((x & 511) >> 3), c = k0 + 8 * nsub + 8 * (x >> 9) + (x & 7);
            pf[u] = (r < m && c < m) ? Zb[(long long)r * n + c] : 0.0;
          }
#pragma unroll
        for (int j = 0; j < nsub; ++j) {
#pragma unroll
          for (int k4 = 0; k4 < 8; k4 += 4) {
            const int kk = k0 + 8 * j + k4 + tg;
            const double af = stage[512 * j + (8 * warp + g) * 8 + k4 + tg];
#pragma unroll
            for (int y = 0; y < 2; ++y) {
              const double bf = kk < m ? Vs[(8 * y + g) * m + kk] : 0.0;
              dmma(a0[y], a1[y], af, bf);
            }
          }
        }
        __syncthreads();
      }
#pragma unroll
      for (int y = 0; y < 2; ++y) {
        Wm[(8 * warp + g) * kQBlock + 8 * y + 2 * tg] = a0[y];
        Wm[(8 * warp + g) * kQBlock + 8 * y + 2 * tg + 1] = a1[y];
      }
      __syncthreads();
      // Wt = Wm T^T: entry (r, i) = sum_q Wm[r][q] T[i][q]
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int x = tid + 256 * u, r = x >> 4, i = x & (kQBlock - 1);
        double sum = 0.0;
#pragma unroll
        for (int q = 0; q < kQBlock; ++q) sum += Wm[r * kQBlock + q] * Ts[i][q];
        Wt[x] = sum;
      }
      __syncthreads();
      // Zt -= Wt Vs
      for (int ct = 0; ct < m; ct += 64) {
        double d0[2][4], d1[2][4];
#pragma unroll
        for (int x = 0; x < 2; ++x)
#pragma unroll
          for (int y = 0; y < 4; ++y) {
            const int r = rt + wrow + 8 * x + g, c = ct + wcol + 8 * y + 2 * tg;
            d0[x][y] = (r < m && c < m) ? Zb[(long long)r * n + c] : 0.0;
            d1[x][y] = (r < m && c + 1 < m) ? Zb[(long long)r * n + c + 1] : 0.0;
          }
#pragma unroll
        for (int k4 = 0; k4 < kQBlock; k4 += 4) {
          double af[2], bf[4];
#pragma unroll
          for (int x = 0; x < 2; ++x) af[x] = -Wt[(wrow + 8 * x + g) * kQBlock + k4 + tg];
#pragma unroll
          for (int y = 0; y < 4; ++y) {
            const int c = ct + wcol + 8 * y + g;
            bf[y] = c < m ? Vs[(k4 + tg) * m + c] : 0.0;
          }
#pragma unroll
          for (int x = 0; x < 2; ++x)
#pragma unroll
            for (int y = 0; y < 4; ++y) dmma(d0[x][y], d1[x][y], af[x], bf[y]);
        }
#pragma unroll
        for (int x = 0; x < 2; ++x)
#pragma unroll
          for (int y = 0; y < 4; ++y) {
            const int r = rt + wrow + 8 * x + g, c = ct + wcol + 8 * y + 2 * tg;
            if (r < m && c < m) Zb[(long long)r * n + c] = d0[x][y];
            if (r < m && c + 1 < m) Zb[(long long)r * n + c + 1] = d1[x][y];
          }
      }
      __syncthreads();  // Wm and Wt are rewritten by the next tile
    }
  }
}

// ------------------------------------------------ divide and conquer (Cuppen)
// Tridiagonal T (d, e) = diag(T_left, T_right) + rho v v^T torn at every node
// of a halving tree down to 1 x 1 leaves; the eigenvector matrix G of each
// node (rows = eigenvectors in T's index space, an m x m diagonal block of an
// n x n buffer) is built bottom-up by rank-one merges:
//  * z = [last column of G_left ; sign(e) * first column of G_right], unit
//    norm, rho' = |e| |z|^2; eigenvalues sorted;
//  * deflation (tolerance 8 eps max(|delta|max, rho')): entries with rho'|z_i|
//    below it keep their eigenpair; adjacent close pairs are rotated so that
//    one z entry vanishes (LAPACK dlaed2's two tests);
//  * roots of the secular equation 1 + rho' sum z_i^2 / (delta_i - lambda) = 0
//    by bracketed two-pole rational interpolation (Bunch, Nielsen and Sorensen
//    1978), each root kept as (nearest pole, offset) so that delta_i - lambda
//    keeps full relative accuracy;
//  * z recomputed from the roots (Gu and Eisenstat 1994) so the eigenvectors
//    w_j = z_i / (delta_i - lambda_j) are orthogonal to working accuracy;
//  * G_node = W G_children as a tiled product with W generated on the fly.
// Finally Zc <- G Zc (Zc = Q^T), and the eigenvalues are left in d.
// kDcMin, kDcK, kDcBs, kDcTileElems and dc_ws_elems (tb_kernels.h): the
// workspace starts at tau and runs to the end of the dynamic shared memory,
// which syev_smem_bytes sizes so that every structure of kDcMin+ rows has it.

// Root j of 1 + rho sum_i z_i^2 / (dl_i - lambda) = 0 (dl strictly ascending,
// rho > 0): lambda = dl[*o] + *tau.
template <typename T>
__device__ void secular_root(int j, int k, const T* dl, const T* z, T rho, int* o_out, T* tau_out) {
  const T eps = Eps<T>::v;
  int o;
  T lo, hi;
  if (j < k - 1) {
    const T mid = T(0.5) * (dl[j + 1] - dl[j]);
    T f = T(1);
    for (int i = 0; i < k; ++i) f += rho * z[i] * z[i] * dc_rcp((dl[i] - dl[j]) - mid);
    if (f >= T(0)) { o = j; lo = T(0); hi = mid; }
    else { o = j + 1; lo = -mid; hi = T(0); }
  } else {
    T s = T(0);
    for (int i = 0; i < k; ++i) s += z[i] * z[i];
    o = k - 1; lo = T(0); hi = rho * s;
  }
  const T base = dl[o];
  T tau = T(0.5) * (lo + hi);
  for (int it = 0; it < 100; ++it) {
    T psi = T(0), phi = T(0), dpsi = T(0), dphi = T(0);
    for (int i = 0; i < k; ++i) {
      const T r = dc_rcp((dl[i] - base) - tau);
      const T q = z[i] * z[i] * r;
      if (i <= j) { psi += q; dpsi += q * r; }
      else { phi += q; dphi += q * r; }
    }
    psi *= rho; phi *= rho; dpsi *= rho; dphi *= rho;
    const T f = T(1) + psi + phi;
    const T err = eps * (T(8) * (tb_abs(psi) + tb_abs(phi)) + T(3) + tb_abs(tau) * (dpsi + dphi));
    if (tb_abs(f) <= err) break;
    if (f < T(0)) lo = tau; else hi = tau;
    if (hi - lo <= T(2) * eps * fmax(tb_abs(lo), tb_abs(hi))) break;
    const T a = (dl[j] - base) - tau;
    T eta = T(0);
    bool ok = false;
    if (j < k - 1) {  // psi ~ c1 + s1/(a - eta), phi ~ c2 + s2/(b - eta)
      const T b = (dl[j + 1] - base) - tau;
      const T s1 = dpsi * a * a, c1 = psi - dpsi * a, s2 = dphi * b * b, c2 = phi - dphi * b;
      const T C = T(1) + c1 + c2;
      const T Bq = C * (a + b) + s1 + s2;
      const T sq = tb_sqrt(fmax(Bq * Bq - T(4) * C * a * b * f, T(0)));
      const T q = Bq >= T(0) ? T(0.5) * (Bq + sq) : T(0.5) * (Bq - sq);
      if (q != T(0)) { eta = a * b * f / q; ok = eta > a && eta < b; }
      if (!ok && C != T(0)) { eta = q / C; ok = eta > a && eta < b; }
    } else {
      const T s1 = dpsi * a * a, C = T(1) + psi - dpsi * a;
      if (C > T(0)) { eta = a + s1 / C; ok = true; }
    }
    T tn = tau + eta;
    if (!ok || !(tn > lo && tn < hi)) tn = T(0.5) * (lo + hi);
    tau = tn;
  }
  *o_out = o;
  *tau_out = tau;
}

// Out[(r0 + j) ld + c0 + c] = sum_i gen(j, i) In[(srow ? srow[i] : i) ld + c0 + c]
// for j < nrow, c < ncol, i < kdim: 64 x 64 output tiles, slabs of kDcK
// staged in shared memory (Wt: 64 x kDcK, Bt: kDcK x 64 with padded rows).
// The next slab (its loads and generated entries) is fetched into registers
// while the current one is multiplied.  FP64: on the FP64 tensor instruction
// mma.sync.m8n8k4 (each warp a 16 x 32 block as 2 x 4 fragments of 8 x 8);
// FP32: 4 x 4 outputs per thread.
template <typename T, typename Gen>
__device__ void dc_gemm(int nrow, int kdim, int ncol, Gen gen, const T* In, const int* srow, T* Out, int r0, int c0,
                        int ld, T* Wt, T* Bt) {
  constexpr bool kTensor = sizeof(T) == 8;
  const int tid = threadIdx.x, ty = tid >> 4, tx = tid & 15;
  const int lane = tid & 31, warp = tid >> 5, g = lane >> 2, tg = lane & 3;
  const int wrow = (warp >> 1) * 16, wcol = (warp & 1) * 32;  // this warp's block of the tile (FP64)
  for (int j0 = 0; j0 < nrow; j0 += 64) {
    for (int cb = 0; cb < ncol; cb += 64) {
      T acc[4][4];  // FP32: outputs; FP64: acc[x][2y + h] of fragment (x, y) for x < 2, y < 4
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] = T(0);
      T acc2[2][4];  // FP64: second half of the fragments' outputs
#pragma unroll
      for (int a = 0; a < 2; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc2[a][b] = T(0);
      constexpr int kPer = 64 * kDcK / kEigThreads;  // slab entries per thread
      T wr[kPer], br[kPer];
      auto fetch = [&](int i0) {
#pragma unroll
        for (int u = 0; u < kPer; ++u) {
          const int x = tid + u * kEigThreads;
          const int jj = x / kDcK, kk = x - jj * kDcK, j = j0 + jj, i = i0 + kk;
          wr[u] = (j < nrow && i < kdim) ? gen(j, i) : T(0);
          const int kb = x >> 6, cc = x & 63, ib = i0 + kb;
          br[u] = (ib < kdim && cb + cc < ncol) ? In[(long long)(srow ? srow[ib] : ib) * ld + c0 + cb + cc] : T(0);
        }
      };
      fetch(0);
      for (int i0 = 0; i0 < kdim; i0 += kDcK) {
#pragma unroll
        for (int u = 0; u < kPer; ++u) {
          const int x = tid + u * kEigThreads;
          Wt[x] = wr[u];
          Bt[(x >> 6) * kDcBs + (x & 63)] = br[u];
        }
        __syncthreads();
        if (i0 + kDcK < kdim) fetch(i0 + kDcK);
        if constexpr (kTensor) {
#pragma unroll
          for (int k4 = 0; k4 < kDcK; k4 += 4) {
            double af[2], bf[4];
#pragma unroll
            for (int x = 0; x < 2; ++x) af[x] = Wt[(wrow + 8 * x + g) * kDcK + k4 + tg];
#pragma unroll
            for (int y = 0; y < 4; ++y) bf[y] = Bt[(k4 + tg) * kDcBs + wcol + 8 * y + g];
#pragma unroll
            for (int x = 0; x < 2; ++x)
#pragma unroll
              for (int y = 0; y < 4; ++y) dmma(acc[x][y], acc2[x][y], af[x], bf[y]);
          }
        } else {
#pragma unroll
          for (int kk = 0; kk < kDcK; ++kk) {
            T av[4], bv[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) av[a] = Wt[(ty * 4 + a) * kDcK + kk];
#pragma unroll
            for (int b = 0; b < 4; ++b) bv[b] = Bt[kk * kDcBs + tx + 16 * b];
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
              for (int b = 0; b < 4; ++b) acc[a][b] += av[a] * bv[b];
          }
        }
        __syncthreads();
      }
      if constexpr (kTensor) {  // fragment (x, y): rows wrow + 8x + g, columns wcol + 8y + 2 tg + {0, 1}
#pragma unroll
        for (int x = 0; x < 2; ++x) {
          const int j = j0 + wrow + 8 * x + g;
          if (j >= nrow) continue;
#pragma unroll
          for (int y = 0; y < 4; ++y) {
            const int c = cb + wcol + 8 * y + 2 * tg;
            if (c < ncol) Out[(long long)(r0 + j) * ld + c0 + c] = acc[x][y];
            if (c + 1 < ncol) Out[(long long)(r0 + j) * ld + c0 + c + 1] = acc2[x][y];
          }
        }
      } else {
#pragma unroll
        for (int a = 0; a < 4; ++a) {
          const int j = j0 + ty * 4 + a;
          if (j >= nrow) continue;
#pragma unroll
          for (int b = 0; b < 4; ++b) {
            const int c = cb + tx + 16 * b;
            if (c < ncol) Out[(long long)(r0 + j) * ld + c0 + c] = acc[a][b];
          }
        }
      }
    }
  }
}

// One merge of the node [lo, hi) torn at t: children's G blocks in Gi (the
// node's diagonal block), eigenvalues in d[lo, hi).  The rows lo..hi-1 of V
// (columns vc0 .. vc0+vcols-1; V = Gi itself, or the children's eigenvectors
// already applied to Zc) are combined into the same rows of Out and the
// merged eigenvalues written to d[lo, hi).  V is overwritten.  ws:
// dc_ws_elems(hi - lo) T.
template <typename T>
__device__ void dc_merge(T* d, const T* e, int n, int lo, int t, int hi, T* Gi, T* V, int vc0, int vcols, T* Out,
                         T* ws, T* red) {
  const int tid = threadIdx.x, nt = blockDim.x;
  const int m = hi - lo;
  T* delta = ws;          // m: sorted eigenvalues (rotated pairs updated)
  T* zs = delta + m;      // m: sorted z (unit norm)
  T* dl = zs + m;         // k: non-deflated delta
  T* zl = dl + m;         // k: their z, then the recomputed z
  T* tv = zl + m;         // k: root offsets
  T* inrm = tv + m;       // k: 1 / |w_j|
  T* rc = inrm + m;       // rotations: cosine
  T* rsn = rc + m;        //            sine
  T* Wt = rsn + m;
  T* Bt = Wt + 64 * kDcK;
  int* rowof = reinterpret_cast<int*>(Wt + kDcTileElems);  // m: row of sorted entry s
  int* flg = rowof + m;   // m: deflated
  int* ndl = flg + m;     // m: sorted index of the k non-deflated, then of the deflated
  int* rp = ndl + m;      // rotations: rows
  int* rq = rp + m;
  int* ori = rq + m;      // k: root origin (index into dl)
  int* srow = ori + m;    // k: row of non-deflated entry
  __shared__ int s_k, s_nrot;
  __shared__ T s_rho;
  const T ev = e[t - 1];
  const T rho = tb_abs(ev), sg = ev >= T(0) ? T(1) : T(-1);
  // children's blocks are diagonal sub-blocks: clear the rest of the node's block
  if (V == Gi)
    for (int r = lo + (tid >> 5); r < hi; r += nt >> 5)
      for (int c = (r < t ? t : lo) + (tid & 31); c < (r < t ? hi : t); c += 32) Gi[(long long)r * n + c] = T(0);
  // z and its norm
  T part = T(0);
  for (int r = lo + tid; r < hi; r += nt) {
    const T z = r < t ? Gi[(long long)r * n + t - 1] : sg * Gi[(long long)r * n + t];
    part += z * z;
  }
  const T zz = block_sum(part, red);  // synchronises
  const T zsc = T(1) / tb_sqrt(zz), rhop = rho * zz;
  // rank sort of the eigenvalues (ties by index)
  for (int r = lo + tid; r < hi; r += nt) {
    const T dr = d[r];
    int rank = 0;
    for (int q = lo; q < hi; ++q) {
      const T dq = d[q];
      rank += (dq < dr || (dq == dr && q < r)) ? 1 : 0;
    }
    rowof[rank] = r;
    delta[rank] = dr;
    zs[rank] = (r < t ? Gi[(long long)r * n + t - 1] : sg * Gi[(long long)r * n + t]) * zsc;
  }
  __syncthreads();
  if (tid < 32) {  // deflation scan (lane 0, in order) and compaction (warp ballots), warp 0
    const int lane = tid;
    T dmax = T(0);
    for (int s = lane; s < m; s += 32) dmax = fmax(dmax, tb_abs(delta[s]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) dmax = fmax(dmax, __shfl_xor_sync(0xffffffffu, dmax, o));
    const T tol = T(8) * Eps<T>::v * fmax(dmax, rhop);
    for (int s = lane; s < m; s += 32) flg[s] = rhop * tb_abs(zs[s]) <= tol ? 1 : 0;
    __syncwarp();
    if (lane == 0) {
      // close pair (prev, s): the rotation zeroing z_prev (c = z_s / tau, sn = -z_prev / tau,
      // tau = |(z_prev, z_s)|) deflates when |(d_s - d_prev) c sn| <= tol, tested as
      // |d_s - d_prev| |z_prev z_s| <= tol tau^2 without the square root
      int nrot = 0, prev = -1;
      for (int s = 0; s < m; ++s) {
        if (flg[s]) continue;
        if (prev >= 0) {
          const T za = zs[prev], zb = zs[s], t2 = za * za + zb * zb;
          if (tb_abs(delta[s] - delta[prev]) * tb_abs(za * zb) <= tol * t2) {
            const T tau = tb_sqrt(t2);
            const T c = zb / tau, sn = -za / tau;
            rp[nrot] = rowof[prev]; rq[nrot] = rowof[s]; rc[nrot] = c; rsn[nrot] = sn; ++nrot;
            zs[s] = tau; zs[prev] = T(0);
            const T dp = delta[prev], ds = delta[s];
            delta[prev] = dp * c * c + ds * sn * sn;
            delta[s] = dp * sn * sn + ds * c * c;
            flg[prev] = 1;
          }
        }
        prev = s;
      }
      s_nrot = nrot;
    }
    __syncwarp();
    // non-deflated entries first, then the deflated ones, each in order
    int k = 0;
    for (int s0 = 0; s0 < m; s0 += 32) {
      const int s = s0 + lane;
      const bool keep = s < m && !flg[s];
      const unsigned bal = __ballot_sync(0xffffffffu, keep);
      if (keep) {
        const int pos = k + __popc(bal & ((1u << lane) - 1u));
        ndl[pos] = s; dl[pos] = delta[s]; zl[pos] = zs[s]; srow[pos] = rowof[s];
      }
      k += __popc(bal);
    }
    int q = k;
    for (int s0 = 0; s0 < m; s0 += 32) {
      const int s = s0 + lane;
      const bool defl = s < m && flg[s];
      const unsigned bal = __ballot_sync(0xffffffffu, defl);
      if (defl) ndl[q + __popc(bal & ((1u << lane) - 1u))] = s;
      q += __popc(bal);
    }
    if (lane == 0) { s_k = k; s_rho = rhop; }
  }
  __syncthreads();
  const int k = s_k, nrot = s_nrot;
  // close-pair rotations on the rows, one thread per column, in order
  for (int c = vc0 + tid; c < vc0 + vcols; c += nt)
    for (int q = 0; q < nrot; ++q) {
      T* pa = V + (long long)rp[q] * n + c;
      T* pb = V + (long long)rq[q] * n + c;
      const T a = *pa, b = *pb;
      *pa = rc[q] * a + rsn[q] * b;
      *pb = rc[q] * b - rsn[q] * a;
    }
  for (int j = tid; j < k; j += nt) secular_root(j, k, dl, zl, s_rho, ori + j, tv + j);
  __syncthreads();
  for (int i = tid; i < k; i += nt) {  // Gu-Eisenstat: every ratio in (0, 1]
    const T di = dl[i];
    T prod = ((dl[ori[k - 1]] - di) + tv[k - 1]) / s_rho;
    for (int j = 0; j < i; ++j) prod *= ((dl[ori[j]] - di) + tv[j]) * dc_rcp(dl[j] - di);
    for (int j = i + 1; j < k; ++j) prod *= ((dl[ori[j - 1]] - di) + tv[j - 1]) * dc_rcp(dl[j] - di);
    zl[i] = copysign(tb_sqrt(fmax(prod, T(0))), zl[i]);
  }
  __syncthreads();
  for (int j = tid; j < k; j += nt) {
    const T bj = dl[ori[j]], tj = tv[j];
    T s = T(0);
    for (int i = 0; i < k; ++i) {
      const T w = zl[i] * dc_rcp((dl[i] - bj) - tj);
      s += w * w;
    }
    inrm[j] = T(1) / tb_sqrt(s);
  }
  __syncthreads();
  // roots: Out rows lo .. lo+k-1; deflated: rows lo+k .. hi-1 copied
  auto wgen = [&](int j, int i) { return zl[i] * dc_rcp((dl[i] - dl[ori[j]]) - tv[j]) * inrm[j]; };
  // W formed once (row stride n) instead of once per 64-column tile of the
  // product, where Gi has a free k x k block: at the root all of Gi is free
  // once z has been read; below it, rows lo.. of Gi beside the node's block
  // (columns hi.. or ..lo) belong to no node of this level
  T* Wb = nullptr;
  if (V != Gi) Wb = Gi;
  else if (hi + k <= n) Wb = Gi + (long long)lo * n + hi;
  else if (lo >= k) Wb = Gi + (long long)lo * n + (lo - k);
  if (Wb) {
    for (int j = tid >> 5; j < k; j += nt >> 5)
      for (int i = tid & 31; i < k; i += 32) Wb[(long long)j * n + i] = wgen(j, i);
    __syncthreads();
    dc_gemm<T>(k, k, vcols, [&](int j, int i) { return Wb[(long long)j * n + i]; }, V, srow, Out, lo, vc0, n, Wt, Bt);
  } else {
    dc_gemm<T>(k, k, vcols, wgen, V, srow, Out, lo, vc0, n, Wt, Bt);
  }
  for (int q = tid >> 5; q < m - k; q += nt >> 5) {
    const T* src = V + (long long)rowof[ndl[k + q]] * n;
    T* dst = Out + (long long)(lo + k + q) * n;
    for (int c = vc0 + (tid & 31); c < vc0 + vcols; c += 32) dst[c] = src[c];
  }
  __syncthreads();
  for (int j = tid; j < m; j += nt) d[lo + j] = j < k ? dl[ori[j]] + tv[j] : delta[ndl[j]];
  __syncthreads();
}

constexpr int kDcLeaf = 24;  // leaves of the merge tree: at most this many rows, solved by one warp

// Leaf [lo, lo+s) of the tree (s <= kDcLeaf) by one warp: implicit QL with
// Wilkinson shifts (the same sweep as the k_syev producer) on lane 0 over
// d[lo..] and a private copy of the leaf's off-diagonal, each sweep's
// rotations then applied by lanes (one per column) to the rows of the leaf's
// eigenvector block U in shared memory; U is written to G's diagonal block.
// Returns false if an eigenvalue took more than 60 sweeps.
constexpr int kDcLeafWs = kDcLeaf * kDcLeaf + 3 * kDcLeaf;  // per leaf warp: U, off-diagonal, rotations
static_assert(kDcLeafWs <= dc_ws_elems<double>(kDcMin), "leaf workspace exceeds the divide-and-conquer workspace");

template <typename T>
__device__ bool dc_leaf(T* d, const T* e, int lo, int s, T* U, T* le, T* rcs, T* G, int n) {
  const int lane = threadIdx.x & 31;
  const T eps = Eps<T>::v;
  for (int x = lane; x < s * s; x += 32) U[x] = (x / s == x % s) ? T(1) : T(0);
  for (int i = lane; i < s; i += 32) le[i] = i < s - 1 ? e[lo + i] : T(0);
  __syncwarp();
  T* dd = d + lo;
  bool ok = true;
  for (int l = 0; l < s && ok; ++l) {
    int iter = 0;
    for (;;) {
      int mq = s - 1;
      for (int i = l; i < s - 1; ++i)
        if (tb_abs(le[i]) <= eps * (tb_abs(dd[i]) + tb_abs(dd[i + 1]))) { mq = i; break; }
      if (mq == l) break;
      if (++iter > 60) { ok = false; break; }
      int cnt = 0;
      if (lane == 0) {
        T g = (dd[l + 1] - dd[l]) / (T(2) * le[l]);
        T r = tb_sqrt(g * g + T(1));
        g = dd[mq] - dd[l] + le[l] / (g + (g >= T(0) ? r : -r));
        T sn = T(1), c = T(1), pp = T(0);
        bool underflow = false;
        for (int i = mq - 1; i >= l; --i) {
          const T f = sn * le[i], bb = c * le[i];
          const T rr2 = f * f + g * g;
          if (rr2 == T(0)) { dd[i + 1] -= pp; le[mq] = T(0); underflow = true; break; }
          const T ri = chain_rsqrt(rr2);
          r = rr2 * ri;
          le[i + 1] = r;
          sn = f * ri;
          c = g * ri;
          g = dd[i + 1] - pp;
          r = (dd[i] - g) * sn + T(2) * c * bb;
          pp = sn * r;
          dd[i + 1] = g + pp;
          g = c * r - bb;
          rcs[2 * cnt] = c;
          rcs[2 * cnt + 1] = sn;
          ++cnt;
        }
        if (!underflow) { dd[l] -= pp; le[l] = g; le[mq] = T(0); }
      }
      cnt = __shfl_sync(0xffffffffu, cnt, 0);
      __syncwarp();
      if (lane < s) {  // rotation t acts on rows i = mq-1-t and i+1 of U
        for (int t = 0; t < cnt; ++t) {
          const int i = mq - 1 - t;
          const T c = rcs[2 * t], sn = rcs[2 * t + 1];
          const T x = U[i * s + lane], y = U[(i + 1) * s + lane];
          U[(i + 1) * s + lane] = sn * x + c * y;
          U[i * s + lane] = c * x - sn * y;
        }
      }
      __syncwarp();
    }
  }
  for (int x = lane; x < s * s; x += 32) G[(long long)(lo + x / s) * n + lo + x % s] = U[x];
  __syncwarp();
  return ok;
}

// Node b of depth dep of the halving tree: [lo, hi); *plen = its parent's size.
__device__ inline void dc_node(int n, int dep, int b, int* lo_out, int* hi_out, int* plen) {
  int lo = 0, hi = n, pl = n + 1;
  for (int l = 0; l < dep; ++l) {
    const int mid = (lo + hi) >> 1;
    pl = hi - lo;
    if ((b >> (dep - 1 - l)) & 1) lo = mid; else hi = mid;
  }
  *lo_out = lo; *hi_out = hi; *plen = pl;
}

// Eigenvalues (d) and eigenvector rows (Zc <- G Zc) of the tridiagonal
// (d, e) by the merge tree; G0 and G1 are n x n buffers, ws dc_ws_elems(n).
// Returns false if a leaf failed to converge.
template <typename T>
__device__ bool dc_solve(T* d, T* e, T* Z, T* G0, T* G1, int n, T* ws, T* red, long long ws_cap) {
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, wid = tid >> 5, nw = nt >> 5;
  __shared__ int s_fail;
  int depth = 0;  // nodes at this depth have at most kDcLeaf rows
  while (((n + (1 << depth) - 1) >> depth) > kDcLeaf) ++depth;
  if (tid == 0) s_fail = 0;
  // tear every internal node (rho = |e[t-1]| off both neighbours)
  for (int dep = 0; dep < depth; ++dep) {
    for (int b = tid; b < (1 << dep); b += nt) {
      int lo, hi, pl;
      dc_node(n, dep, b, &lo, &hi, &pl);
      if (hi - lo <= kDcLeaf) continue;
      const int t = (lo + hi) >> 1;
      const T rho = tb_abs(e[t - 1]);
      d[t - 1] -= rho;  // nodes of one depth are disjoint
      d[t] -= rho;
    }
    __syncthreads();
  }
  // as many leaf warps as the free shared memory holds blocks for
  const int lw = (int)min((long long)nw, ws_cap / kDcLeafWs);
  T* U = ws + wid * kDcLeafWs;
  for (int dep = depth; dep >= 0; --dep) {
    T* Gi = ((depth - dep - 1) & 1) ? G1 : G0;
    T* Go = ((depth - dep) & 1) ? G1 : G0;
    // leaves of this depth, one warp each
    for (int b = wid; wid < lw && b < (1 << dep); b += lw) {
      int lo, hi, pl;
      dc_node(n, dep, b, &lo, &hi, &pl);
      if (hi - lo < 1 || hi - lo > kDcLeaf || pl <= kDcLeaf) continue;
      if (!dc_leaf<T>(d, e, lo, hi - lo, U, U + kDcLeaf * kDcLeaf, U + kDcLeaf * kDcLeaf + kDcLeaf, Go, n) && lane == 0)
        s_fail = 1;
    }
    __syncthreads();
    if (dep > 0) {
      for (int b = 0; b < (1 << dep); ++b) {
        int lo, hi, pl;
        dc_node(n, dep, b, &lo, &hi, &pl);
        if (hi - lo <= kDcLeaf) continue;
        dc_merge<T>(d, e, n, lo, (lo + hi) >> 1, hi, Gi, Gi, lo, hi - lo, Go, ws, red);
      }
    } else {
      // root: Y = diag(G_left, G_right) Zc into the free buffer, then the
      // merge combines rows of Y straight into Zc
      const int t = n >> 1;
      T* Wt = ws;
      T* Bt = Wt + 64 * kDcK;
      for (int h = 0; h < 2; ++h) {
        const int lc = h ? t : 0, sz = h ? n - t : t;
        dc_gemm<T>(sz, sz, n, [&](int j, int i) { return Gi[(long long)(lc + j) * n + lc + i]; },
                   Z + (long long)lc * n, nullptr, Go, lc, 0, n, Wt, Bt);
      }
      __syncthreads();
      dc_merge<T>(d, e, n, 0, t, n, Gi, Go, 0, n, Z, ws, red);
    }
  }
  return s_fail == 0;
}

// Phase 1 of syev_body: A (n x n, symmetric, row-major) is reduced to
// tridiagonal form in place; reflector k is stored in row k of A from column
// k+1 on (leading 1), its scale in tau[k], the off-diagonal in e.  Out of line
// so that its registers are allocated apart from the later phases.
template <typename T>
__device__ __noinline__ void tridiagonalise(T* A, int n, T* e, T* tau, T* v, T* vn, T* p, T* w, T* d, T* ring,
                                            T* red, T* sh, T* gs) {
  const int tid = threadIdx.x, nt = blockDim.x;
  // tridiagonalisation in panels of PanelCfg<T>::width reflectors.  Within a
  // panel the trailing block keeps its value A0 from the panel start; step k
  // forms p = tau A0 v and corrects it with the open pairs (v_i, w_i):
  // A = A0 - sum_i (v_i w_i^T + w_i v_i^T).  Only the row that yields the next
  // reflector is brought up to date; the block itself is rewritten once, when
  // the panel closes, fused with the next step's product.
  if (n < 3) return;
  {
    const int lane = tid & 31, wid = tid >> 5, nw = nt >> 5;
    constexpr int kPanel = PanelCfg<T>::width;
    T* PV = ring;               // kPanel x n: v_i of the open panel (absolute index)
    T* PW = ring + kPanel * n;  // kPanel x n: w_i
    __shared__ T dots[2 * kPanel];
    const int nref = n - 2;     // reflectors 0 .. n-3
    reflector(A, n, 0, v, tau, e, red, sh);
    // p0 = tau0 * A[1..][1..] v0
    colwalk<T>(A, n, 1, n - 1, v, p, tau[0], w, d, vn);
    __syncthreads();
    int np = 0;  // pairs in the open panel
    for (int k = 0; k < nref; ++k) {
      const int mm = n - k - 1, b0 = k + 1;
      const T tk = tau[k];
      if (np > 0) {  // dots[i] = w_i . v, dots[np + i] = v_i . v over the block, one warp per dot
        for (int q = wid; q < 2 * np; q += nw) {
          const T* src = (q < np ? PW + (long long)q * n : PV + (long long)(q - np) * n) + b0;
          T acc = T(0);
          for (int j = lane; j < mm; j += 32) acc += src[j] * v[j];
          acc = warp_sum(acc);
          if (lane == 0) dots[q] = acc;
        }
        __syncthreads();
      }
      // p = tau (A0 v - sum_i v_i (w_i.v) + w_i (v_i.v)); w = p - (tau/2)(p.v) v
      T part = T(0);
      for (int j = tid; j < mm; j += nt) {
        T pj = p[j];
        for (int i = 0; i < np; ++i)
          pj -= tk * (PV[(long long)i * n + b0 + j] * dots[i] + PW[(long long)i * n + b0 + j] * dots[np + i]);
        p[j] = pj;
        part += pj * v[j];
      }
      const T pv = block_sum_syev(part, red);
      const T kk = T(0.5) * tk * pv;
      for (int j = tid; j < mm; j += nt) {
        PV[(long long)np * n + b0 + j] = v[j];
        PW[(long long)np * n + b0 + j] = p[j] - kk * v[j];
      }
      ++np;
      __syncthreads();
      // row r = k+1 (columns r..n-1) brought up to date; the last step also row n-1's diagonal
      const int r = k + 1;
      if (r == nref) {
        for (int c = r + tid; c < n; c += nt) {
          T x = A[(long long)r * n + c];
          for (int i = 0; i < np; ++i)
            x -= PV[(long long)i * n + r] * PW[(long long)i * n + c] + PW[(long long)i * n + r] * PV[(long long)i * n + c];
          A[(long long)r * n + c] = x;
        }
        if (tid == 0) {
          T x = A[(long long)(n - 1) * n + n - 1];
          for (int i = 0; i < np; ++i) x -= T(2) * PV[(long long)i * n + n - 1] * PW[(long long)i * n + n - 1];
          A[(long long)(n - 1) * n + n - 1] = x;
        }
        __syncthreads();
      }
      if (r < nref) {
        // the updated row goes straight into reflector r (as `reflector` does from A): the
        // diagonal back to A, the rest through vn, then the reflector (or, for a zero tail,
        // the row itself) back into row r
        const int mr = n - r - 1;
        T part2 = T(0);
        for (int c = r + tid; c < n; c += nt) {
          T x = A[(long long)r * n + c];
          for (int i = 0; i < np; ++i)
            x -= PV[(long long)i * n + r] * PW[(long long)i * n + c] + PW[(long long)i * n + r] * PV[(long long)i * n + c];
          if (c == r) {
            A[(long long)r * n + r] = x;
          } else {
            vn[c - r - 1] = x;
            if (c > r + 1) part2 += x * x;
          }
        }
        const T sigma = block_sum_syev(part2, red);  // synchronises
        if (tid == 0) {
          const T alpha = vn[0];
          if (sigma == T(0)) {
            tau[r] = T(0); e[r] = alpha; sh[0] = T(0); sh[1] = T(0);
          } else {
            const T rr = tb_sqrt(alpha * alpha + sigma);
            const T beta = alpha <= T(0) ? rr : -rr;
            tau[r] = (beta - alpha) / beta;
            e[r] = beta;
            sh[0] = tau[r];
            sh[1] = T(1) / (alpha - beta);
          }
        }
        __syncthreads();
        {
          const T scal = sh[1];
          const bool refl = sh[0] != T(0);
          T* rowr = A + (long long)r * n + r + 1;
          for (int i = tid; i < mr; i += nt) {
            const T u = vn[i];
            const T x = i == 0 ? T(1) : (refl ? u * scal : T(0));
            vn[i] = x;
            rowr[i] = refl ? x : u;
          }
          __syncthreads();
        }
        if (np == kPanel) {  // close the panel: A -= V W^T + W V^T on the block, fused with p_r = tau_r A vn
          if constexpr (sizeof(T) == 8) {
            if (gs)  // the lower triangle is stale from the first upper-only walk on
              panel_walk_tc_sym<2>(A, n, r + 1, n - r - 1, PV, PW, vn, p, tau[r], gs);
            else
              panel_walk_tc(A, n, r + 1, n - r - 1, PV, PW, vn, p, tau[r], w, d, v);  // v is in PV already
          } else
            panel_walk<T>(A, n, r + 1, n - r - 1, PV, PW, vn, p, tau[r], w);
          np = 0;
        } else {  // p_r = tau_r A0 vn
          if constexpr (sizeof(T) == 8) {
            if (gs)
              symwalk(A, n, r + 1, n - r - 1, vn, p, tau[r], gs);
            else
              colwalk<T>(A, n, r + 1, n - r - 1, vn, p, tau[r], w, d, v);  // v is in PV already
          } else {
            colwalk<T>(A, n, r + 1, n - r - 1, vn, p, tau[r], w, d, v);
          }
        }
        __syncthreads();
      }
      T* t = v; v = vn; vn = t;
    }
  }
}

// Phase 2 of syev_body: Z = Q^T from the reflectors left in A and tau by
// tridiagonalise.  ring: kQBlock x n of shared memory; stage: 4n free shared
// elements; Sq: an n x n global scratch (or null).  Out of line like phase 1.
template <typename T>
__device__ __noinline__ void form_q(const T* A, T* Z, int n, const T* tau, T* ring, T* stage, T* Sq) {
  const int tid = threadIdx.x, nt = blockDim.x;
  // Zc = Q^T (row c of Zc = column c of Q), Q = H_0 H_1 ... H_{n-3},
  // accumulated backwards in blocks of kQBlock reflectors in compact WY form:
  // H_k0 ... H_k1 = I - V T V^T (V = [v_k0 .. v_k1], T upper triangular), so
  // Zc <- Zc H_k1 ... H_k0 = Zc - (Zc V) T^T V^T on rows and columns >= k0+1.
  // Each row of that block is read twice and written once per block instead of
  // once per reflector.  V is staged in shared memory (the rotation ring is not
  // in use yet); one warp per row: partial dots of the row with the kQBlock
  // reflectors, a warp reduction, T^T applied by kQBlock lanes, then the update.
  for (int i = tid >> 5; i < n; i += nt >> 5)
    for (int j = tid & 31; j < n; j += 32) Z[(long long)i * n + j] = i == j ? T(1) : T(0);
  __syncthreads();
  {
    const int lane = tid & 31, wid = tid >> 5, nw = nt >> 5;
    __shared__ T Ts[kQBlock][kQBlock];          // T of the block
    __shared__ T yv[kQBlock][kQBlock];          // V^T V (upper part)
    __shared__ T wps[kEigThreads / 32][kQBlock];  // per warp: (row . V) T^T
    T* Vs = ring;                               // kQBlock x m, m <= n - 1
    // FP64 with a scratch matrix: each block's products on the tensor pipe
    // (formq_block_tc; Wm in Sq, slabs staged in stage, 4n >= 512)
    const bool tcq = Sq && sizeof(T) == 8 && n >= 128 && nt == 256;  // stage: 4n >= 512
    const int nref = n - 2;
    for (int k1 = nref - 1; k1 >= 0; k1 -= kQBlock) {
      const int k0 = k1 - kQBlock + 1 > 0 ? k1 - kQBlock + 1 : 0, bb = k1 - k0 + 1;
      const int c0 = k0 + 1, m = n - c0;
      // Vs[j][cc] = v_{k0+j}[c0 + cc]: row k0+j of A from column k0+j+1 (which holds 1), zero before
      for (int e = tid; e < kQBlock * m; e += nt) {
        const int j = e / m, cc = e - j * m, c = c0 + cc;
        Vs[e] = (j < bb && c >= k0 + j + 1) ? A[(long long)(k0 + j) * n + c] : T(0);
      }
      __syncthreads();
      for (int pq = wid; pq < kQBlock * kQBlock; pq += nw) {
        const int j = pq / kQBlock, i = pq - j * kQBlock;
        if (j >= i || i >= bb) continue;  // warp-uniform
        T acc = T(0);
        for (int cc = lane; cc < m; cc += 32) acc += Vs[j * m + cc] * Vs[i * m + cc];
        acc = warp_sum(acc);
        if (lane == 0) yv[j][i] = acc;
      }
      __syncthreads();
      if (tid < kQBlock) {  // T column by column, lane r: T[i][i] = tau, T[0:i][i] = -tau T[0:i][0:i] (V^T v_i)[0:i]
        const int r = tid;
        for (int i = 0; i < kQBlock; ++i) {
          const T ti = i < bb ? tau[k0 + i] : T(0);
          T x = T(0);
          if (i < bb) {
            if (r == i) {
              x = ti;
            } else if (r < i) {
              T sacc = T(0);
              for (int q = r; q < i; ++q) sacc += Ts[r][q] * yv[q][i];
              x = -ti * sacc;
            }
          }
          Ts[r][i] = x;
          __syncwarp(0xffffu);
        }
      }
      __syncthreads();
      if (tcq) {
        switch (min(kFqSubMax, n / 128)) {  // stage (4n elements) holds 512 per sub-slab
          case 1: formq_block_tc<T, 1>(Z, n, c0, m, Vs, Ts, Sq, stage); break;
          case 2: formq_block_tc<T, 2>(Z, n, c0, m, Vs, Ts, Sq, stage); break;
          case 3: formq_block_tc<T, 3>(Z, n, c0, m, Vs, Ts, Sq, stage); break;
          default: formq_block_tc<T, 4>(Z, n, c0, m, Vs, Ts, Sq, stage); break;
        }
        __syncthreads();
        continue;
      }
      for (int r = c0 + wid; r < n; r += nw) {
        T* zr = Z + (long long)r * n + c0;
        T acc[kQBlock];
#pragma unroll
        for (int j = 0; j < kQBlock; ++j) acc[j] = T(0);
        for (int cc = lane; cc < m; cc += 32) {
          const T z = zr[cc];
#pragma unroll
          for (int j = 0; j < kQBlock; ++j) acc[j] += z * Vs[j * m + cc];
        }
#pragma unroll
        for (int j = 0; j < kQBlock; ++j) acc[j] = warp_sum(acc[j]);
        if (lane < kQBlock) {  // (row . V) T^T, entry lane
          T x = T(0);
#pragma unroll
          for (int q = 0; q < kQBlock; ++q) x += acc[q] * Ts[lane][q];
          wps[wid][lane] = x;
        }
        __syncwarp();
        T wp[kQBlock];
#pragma unroll
        for (int j = 0; j < kQBlock; ++j) wp[j] = wps[wid][j];
        for (int cc = lane; cc < m; cc += 32) {
          T z = zr[cc];
#pragma unroll
          for (int j = 0; j < kQBlock; ++j) z -= wp[j] * Vs[j * m + cc];
          zr[cc] = z;
        }
        __syncwarp();
      }
      __syncthreads();
    }
  }

}

template <typename T>
__device__ __forceinline__ void syev_body(const DevBatch& B, T* __restrict__ Ab, T* __restrict__ Zb,
                                          T* __restrict__ Sb, double* __restrict__ wout, int* __restrict__ perm,
                                          int* __restrict__ status, const int* __restrict__ active) {
  const int m = B.order ? B.order[blockIdx.x] : blockIdx.x;  // largest structures first
  if (active && !active[m]) return;
  if (status[m] != kStOk) return;
  const int n = B.ooff[m + 1] - B.ooff[m];
  if (on_library(B, n)) return;
  if (sizeof(T) == 8 && n <= B.jacobi_max) return;  // the one-warp Jacobi variant (k_syev_jacobi)
  const long long mo = B.moff[m];
  const long long vo = B.ooff[m];
  T* A = Ab + mo;
  T* Z = Zb + mo;
  extern __shared__ __align__(16) unsigned char syev_smem[];
  T* sm = reinterpret_cast<T*>(syev_smem);
  T* d = sm;          // n
  T* e = d + n;       // n
  T* tau = e + n;     // n
  T* v = tau + n;     // n
  T* vn = v + n;      // n
  T* p = vn + n;      // n
  T* w = p + n;       // n
  T* ring = w + n;    // kRing slots x (n cosines + n sines)
  __shared__ T red[kEigThreads / 32];
  __shared__ T sh[4];
  __shared__ int q_full, q_end, q_fail, sh_head[kRing][2];
  __shared__ int q_done[kEigThreads / 32];  // sweeps finished, per consumer warp
  const int tid = threadIdx.x, nt = blockDim.x;

  if (sizeof(T) == 8 && Sb && B.trid_max > 0 && n >= B.trid_min && n >= kTridMin && n <= B.trid_max) {
    // tridiagonalised in shared memory by k_trid_smem: reflectors in A's rows,
    // d | e | tau in the first 3n entries of the scratch slice
    const T* dte = Sb + mo;
    for (int i = tid; i < n; i += nt) {
      d[i] = dte[i];
      e[i] = i < n - 1 ? dte[n + i] : T(0);
      tau[i] = i < n - 2 ? dte[2 * n + i] : T(0);
    }
    __syncthreads();
  } else {
    // symmetrise
    for (int i = tid >> 5; i < n; i += nt >> 5)
      for (int j = i + 1 + (tid & 31); j < n; j += 32) {
        const T s = T(0.5) * (A[(long long)i * n + j] + A[(long long)j * n + i]);
        A[(long long)i * n + j] = s;
        A[(long long)j * n + i] = s;
      }
    for (int i = tid; i < n; i += nt) { e[i] = T(0); tau[i] = T(0); }
    __syncthreads();

    // d: scratch until the end; the global scratch (8n entries) takes the partial products of symwalk
    const bool symw = sizeof(T) == 8 && Sb && nt == 256 && n >= kSymMin + 1;
    tridiagonalise<T>(A, n, e, tau, v, vn, p, w, d, ring, red, sh, symw ? Sb + mo : nullptr);
    for (int i = tid; i < n; i += nt) d[i] = A[(long long)i * n + i];
    if (tid == 0 && n >= 2) e[n - 2] = A[(long long)(n - 2) * n + n - 1];
    __syncthreads();
  }

  form_q<T>(A, Z, n, tau, ring, tau + n, Sb ? Sb + mo : nullptr);

  // ---- 3a. divide and conquer when a scratch buffer is given (A is free now); the
  // workspace runs from tau to the end of the dynamic shared memory
  unsigned dyn_bytes;
  asm("mov.u32 %0, %%dynamic_smem_size;" : "=r"(dyn_bytes));
  const long long ws_cap = (long long)(dyn_bytes / sizeof(T)) - 2LL * n;
  if (Sb && n >= kDcMin && dc_ws_elems<T>(n) <= ws_cap) {
    if (tid == 0) { q_fail = 0; e[n - 1] = T(0); }
    __syncthreads();
    const bool conv = dc_solve<T>(d, e, Z, A, Sb + mo, n, tau, red, ws_cap);
    for (int i = tid; i < n; i += nt)
      if (!conv || !(tb_abs(d[i]) < T(1e30))) q_fail = 1;  // a leaf did not converge, or non-finite input
  } else {
  // ---- 3b. implicit QL, producer (warp 0) / consumers (warps 1..)
  if (tid == 0) { q_full = 0; q_end = 0; q_fail = 0; e[n - 1] = T(0); }
  if (tid < kEigThreads / 32) q_done[tid] = 0;
  __syncthreads();
  const int ncons = (nt >> 5) - 1;
  if (tid < 32) {
    // producer warp: the deflation scan is warp-parallel (ballot over 32
    // consecutive indices), the rotation chain runs on lane 0
    const int lane = tid;
    const T eps = Eps<T>::v;
    int q = 0;
    bool fail = false;
    for (int l = 0; l < n && !fail; ++l) {
      int iter = 0;
      for (;;) {
        int mq = n - 1;
        for (int base = l; base < n - 1; base += 32) {
          const int i = base + lane;
          bool small = false;
          if (i < n - 1) {
            const T dd = tb_abs(d[i]) + tb_abs(d[i + 1]);
            small = tb_abs(e[i]) <= eps * dd;
          }
          const unsigned bal = __ballot_sync(0xffffffffu, small);
          if (bal) { mq = base + __ffs(bal) - 1; break; }
        }
        if (mq == l) break;
        if (++iter > 60) { fail = true; break; }
        // the ring slot of sweep q held sweep q-kRing: wait until EVERY consumer
        // warp has finished it (warps progress unevenly)
        const int slot = q % kRing;
        if (q >= kRing) {
          if (lane == 0) {
            long long spins = 0;
            for (int cw = 1; cw <= ncons && !fail; ++cw)
              while (*(volatile int*)&q_done[cw] < q - kRing + 1) {
                if (++spins > kSpinLimit) { fail = true; break; }
                __nanosleep(64);
              }
          }
          fail = __shfl_sync(0xffffffffu, fail, 0);
          if (fail) break;
          __threadfence_block();
        }
        if (lane == 0) {
          T* rc = ring + (size_t)slot * 2 * n;
          T* rs = rc + n;
          T g = (d[l + 1] - d[l]) / (T(2) * e[l]);
          T r = tb_sqrt(g * g + T(1));
          g = d[mq] - d[l] + e[l] / (g + (g >= T(0) ? r : -r));
          T s = T(1), c = T(1), pp = T(0);
          int cnt = 0;
          bool underflow = false;
          // d[i+1], d[i], e[i] of the current rotation are carried in registers
          // and the next rotation's d[i-1], e[i-1] are loaded one step ahead, so
          // no shared-memory latency sits on the dependency chain (the sweep
          // writes only d[i+1] and e[i+1], never an entry still to be read).
          T dn = d[mq], di = d[mq - 1], ei = e[mq - 1];
          for (int i = mq - 1; i >= l; --i) {
            const T di_next = i > l ? d[i - 1] : T(0);
            const T ei_next = i > l ? e[i - 1] : T(0);
            const T f = s * ei;
            const T bb = c * ei;
            const T rr2 = f * f + g * g;
            if (rr2 == T(0)) { d[i + 1] = dn - pp; e[mq] = T(0); underflow = true; break; }
            const T ri = chain_rsqrt(rr2);
            r = rr2 * ri;
            e[i + 1] = r;
            s = f * ri;
            c = g * ri;
            g = dn - pp;
            r = (di - g) * s + T(2) * c * bb;
            pp = s * r;
            d[i + 1] = g + pp;
            g = c * r - bb;
            rc[cnt] = c;
            rs[cnt] = s;
            ++cnt;
            dn = di;
            di = di_next;
            ei = ei_next;
          }
          if (!underflow) { d[l] -= pp; e[l] = g; e[mq] = T(0); }
          sh_head[slot][0] = mq;
          sh_head[slot][1] = cnt;
          __threadfence_block();
          *(volatile int*)&q_full = q + 1;
        }
        __syncwarp();  // d and e of this sweep are visible to the whole warp
        ++q;
      }
    }
    if (lane == 0) {
      if (fail) *(volatile int*)&q_fail = 1;
      __threadfence_block();
      *(volatile int*)&q_end = 1;
    }
  } else {
    // consumers: every column r of Zc owned by this thread (r = tid - 32 + k*(nt-32)).
    // Sweeps are taken in groups of kWaveK and applied as a wavefront: sweep k
    // of the group lags sweep k-1 by two rows, so each column streams through
    // a window of 2*kWaveK rows held in registers and every element is loaded
    // and stored once per group instead of once per sweep.
    const int lane = tid & 31;
    int q0 = 0;
    for (;;) {
      long long spins = 0;
      int full;
      bool quit = false;
      while ((full = *(volatile int*)&q_full) < q0 + kWaveK) {
        if (*(volatile int*)&q_end) {
          __threadfence_block();
          full = *(volatile int*)&q_full;
          if (full <= q0) quit = true;
          break;
        }
        if (++spins > kSpinLimit) { *(volatile int*)&q_fail = 1; quit = true; break; }
        __nanosleep(32);
      }
      if (quit) break;
      __threadfence_block();
      const int kg = min(kWaveK, full - q0);
      int mk[kWaveK], lk[kWaveK];
      const T* ck[kWaveK];
      int mx = 0, lmin = n;
#pragma unroll
      for (int k = 0; k < kWaveK; ++k) {
        const int slot = (q0 + k) % kRing;
        ck[k] = ring + (size_t)slot * 2 * n;
        if (k < kg) {
          mk[k] = sh_head[slot][0];
          lk[k] = mk[k] - sh_head[slot][1];
          mx = max(mx, mk[k]);
          lmin = min(lmin, lk[k]);
        } else {
          mk[k] = -1;  // inactive: no index satisfies lk <= i <= mk - 1
          lk[k] = 0;
        }
      }
      const int J = mx - lmin + 2 * (kg - 1);
      const int nblk = (J + kWin - 1) / kWin;
      for (int r = tid - 32; r < n; r += nt - 32) {
        T* zr = Z + r;
        T wv[kWin];
        wv[0] = T(0);
#pragma unroll
        for (int a = 1; a < kWin; ++a) {
          const int row = mx - 1 + a;
          wv[a] = row <= n - 1 ? zr[(long long)row * n] : T(0);
        }
        for (int blk = 0; blk < nblk; ++blk) {
#pragma unroll
          for (int p = 0; p < kWin; ++p) {
            const int j = blk * kWin + p;
            const int sl = (kWin - p) % kWin;
            const int row_out = mx + kWin - 1 - j;
            if (j >= 1 && row_out >= 0 && row_out <= n - 1) zr[(long long)row_out * n] = wv[sl];
            const int row_in = mx - 1 - j;
            wv[sl] = row_in >= 0 ? zr[(long long)row_in * n] : T(0);
#pragma unroll
            for (int k = 0; k < kWaveK; ++k) {
              const int i = mx - 1 - j + 2 * k;
              if (i >= lk[k] && i <= mk[k] - 1) {
                const int t = mk[k] - 1 - i;
                const T c = ck[k][t], sn = ck[k][n + t];
                const int ia = (2 * k - p + 2 * kWin) % kWin, ib = (2 * k + 1 - p + 2 * kWin) % kWin;
                const T x = wv[ia], y = wv[ib];
                wv[ib] = sn * x + c * y;
                wv[ia] = c * x - sn * y;
              }
            }
          }
        }
        // flush the final window (last step has phase kWin - 1)
        const int jl = nblk * kWin - 1;
#pragma unroll
        for (int a = 0; a < kWin; ++a) {
          const int row = mx - 1 - jl + a;
          if (row >= 0 && row <= n - 1) zr[(long long)row * n] = wv[(a + 1) % kWin];
        }
      }
      __syncwarp();
      q0 += kg;
      if (lane == 0) {
        __threadfence_block();
        *(volatile int*)&q_done[tid >> 5] = q0;
      }
    }
  }
  }
  __syncthreads();
  if (q_fail) {
    if (tid == 0) status[m] = kStEigenFailed;  // k_fermi retires the structure
    return;
  }
  // ---- 4. ascending order by rank (ties by index)
  for (int i = tid; i < n; i += nt) {
    const T di = d[i];
    int rank = 0;
    for (int j = 0; j < n; ++j) {
      const T dj = d[j];
      rank += (dj < di || (dj == di && j < i)) ? 1 : 0;
    }
    if (!TB_GUARD(9, rank, 0, n)) continue;
    perm[vo + rank] = i;
    wout[vo + rank] = di;
  }
}

}  // namespace

TB_OOB_EXPORT(oob_linalg)

// ------------------------------------------------ small structures: one-warp Jacobi
// Cyclic Jacobi (Jacobi 1846; the parallel tournament ordering of Brent and
// Luk 1985) for structures of at most 32 AOs, one warp per structure, the
// matrix and the rotation accumulator in shared memory (33-double pitch).
// A round applies n/2 disjoint rotations: lane t forms the rotation of pair t
// (symmetric Schur: tau = (a_qq - a_pp)/(2 a_pq), t = sign(tau)/(|tau| +
// sqrt(1 + tau^2)), c = 1/sqrt(1 + t^2), s = t c, which zeroes a_pq in
// J^T A J), then lane k updates row k of every pair's two columns (A J, V J)
// and column k of every pair's two rows (J^T A).  Sweeps stop when the
// off-diagonal norm is below 1e-14 of the Frobenius norm (at most 50 sweeps,
// else TB_EIGEN_FAILED).  A one-CTA eigensolver spends most of its 256
// threads' time waiting at barriers on such small matrices; a warp per
// structure runs eight times as many structures per SM.
__global__ void __launch_bounds__(kJacobiWarps * 32) k_syev_jacobi(DevBatch B, double* __restrict__ Ab,
                                                                  double* __restrict__ Zb,
                                                                  double* __restrict__ wout,
                                                                  int* __restrict__ perm, int* __restrict__ status,
                                                                  const int* __restrict__ active,
                                                                  const int* __restrict__ list, int nlist) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int li = blockIdx.x * kJacobiWarps + warp;
  if (li >= nlist) return;
  const int m = list[li];
  if ((active && !active[m]) || status[m] != kStOk) return;
  const int n = B.ooff[m + 1] - B.ooff[m];
  if (n > kJacobiMaxN) return;
  constexpr int P = kJacobiPitch;
  extern __shared__ double jac_smem[];
  double* a = jac_smem + (size_t)warp * 2 * kJacobiMaxN * P;  // n x n, pitch P
  double* v = a + kJacobiMaxN * P;
  __shared__ double rot_c[kJacobiWarps][kJacobiMaxN / 2], rot_s[kJacobiWarps][kJacobiMaxN / 2];
  __shared__ int rot_p[kJacobiWarps][kJacobiMaxN / 2], rot_q[kJacobiWarps][kJacobiMaxN / 2];
  const long long mo = B.moff[m], vo = B.ooff[m];
  const double* A = Ab + mo;
  if (lane < n)
    for (int j = 0; j < n; ++j) {
      a[lane * P + j] = 0.5 * (A[(long long)lane * n + j] + A[(long long)j * n + lane]);
      v[lane * P + j] = lane == j ? 1.0 : 0.0;
    }
  __syncwarp();
  const int nn = n + (n & 1);  // players; index n (odd n) sits out
  double fro = 0.0;
  if (lane < n)
    for (int j = 0; j < n; ++j) fro += a[lane * P + j] * a[lane * P + j];
  fro = warp_sum(fro);
  bool conv = n <= 1;
  for (int sweep = 0; sweep < 50 && !conv; ++sweep) {
    double off = 0.0;
    if (lane < n)
      for (int j = 0; j < n; ++j)
        if (j != lane) off += a[lane * P + j] * a[lane * P + j];
    off = warp_sum(off);
    if (off <= 1e-28 * fro) { conv = true; break; }
    for (int r = 0; r < nn - 1; ++r) {
      if (lane < nn / 2) {
        int p = lane == 0 ? r : (r + lane) % (nn - 1);
        int q = lane == 0 ? nn - 1 : (r - lane + nn - 1) % (nn - 1);
        if (p > q) { const int x = p; p = q; q = x; }
        double c = 1.0, s = 0.0;
        if (q < n) {
          const double apq = a[p * P + q];
          if (apq != 0.0) {
            const double tau = (a[q * P + q] - a[p * P + p]) / (2.0 * apq);
            const double t = (tau >= 0.0 ? 1.0 : -1.0) / (fabs(tau) + sqrt(1.0 + tau * tau));
            c = 1.0 / sqrt(1.0 + t * t);
            s = t * c;
          }
        }
        rot_p[warp][lane] = p;
        rot_q[warp][lane] = q < n ? q : p;  // the sitting-out pair becomes the identity
        rot_c[warp][lane] = c;
        rot_s[warp][lane] = q < n ? s : 0.0;
      }
      __syncwarp();
      // columns: A <- A J and V <- V J, lane k on row k
      if (lane < n)
        for (int t = 0; t < nn / 2; ++t) {
          const int p = rot_p[warp][t], q = rot_q[warp][t];
          if (p == q) continue;
          const double c = rot_c[warp][t], s = rot_s[warp][t];
          const double akp = a[lane * P + p], akq = a[lane * P + q];
          a[lane * P + p] = c * akp - s * akq;
          a[lane * P + q] = s * akp + c * akq;
          const double vkp = v[lane * P + p], vkq = v[lane * P + q];
          v[lane * P + p] = c * vkp - s * vkq;
          v[lane * P + q] = s * vkp + c * vkq;
        }
      __syncwarp();
      // rows: A <- J^T A, lane k on column k
      if (lane < n)
        for (int t = 0; t < nn / 2; ++t) {
          const int p = rot_p[warp][t], q = rot_q[warp][t];
          if (p == q) continue;
          const double c = rot_c[warp][t], s = rot_s[warp][t];
          const double apk = a[p * P + lane], aqk = a[q * P + lane];
          a[p * P + lane] = c * apk - s * aqk;
          a[q * P + lane] = s * apk + c * aqk;
        }
      __syncwarp();
    }
  }
  if (!conv) {
    if (lane == 0) status[m] = kStEigenFailed;
    return;
  }
  // eigenvector i (column i of v) as row i of Z; ascending order by rank (ties by index)
  double* Z = Zb + mo;
  if (lane < n && TB_GUARD(10, (long long)lane * n + n - 1, 0, (long long)n * n)) {
    for (int k = 0; k < n; ++k) Z[(long long)lane * n + k] = v[k * P + lane];
    const double di = a[lane * P + lane];
    int rank = 0;
    for (int j = 0; j < n; ++j) {
      const double dj = a[j * P + j];
      rank += (dj < di || (dj == di && j < lane)) ? 1 : 0;
    }
    perm[vo + rank] = lane;
    wout[vo + rank] = di;
  }
}

__global__ void __launch_bounds__(kEigThreads, 3) k_syev(DevBatch B, double* __restrict__ Ab, double* __restrict__ Zb,
                                                      double* __restrict__ Sb, double* __restrict__ wout,
                                                      int* __restrict__ perm, int* __restrict__ status,
                                                      const int* __restrict__ active) {
  syev_body<double>(B, Ab, Zb, Sb, wout, perm, status, active);
}

__global__ void __launch_bounds__(kEigThreads, 4) k_syev_f32(DevBatch B, float* __restrict__ Ab,
                                                          float* __restrict__ Zb, double* __restrict__ wout,
                                                          int* __restrict__ perm, int* __restrict__ status,
                                                          const int* __restrict__ active) {
  syev_body<float>(B, Ab, Zb, nullptr, wout, perm, status, active);
}

}  // namespace tb
