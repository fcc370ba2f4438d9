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
// Left-looking column Cholesky of the structure's overlap S (row-major),
// result stored column-major in W (W[k][i] = L[i][k], i >= k).
__global__ void k_cholesky(DevBatch B, const double* __restrict__ S, double* __restrict__ W,
                           int* __restrict__ status, const int* __restrict__ active) {
  const int m = blockIdx.x;
  if (active && !active[m]) return;
  const int n = B.ooff[m + 1] - B.ooff[m];
  const long long mo = B.moff[m];
  const double* s = S + mo;
  double* w = W + mo;
  __shared__ double red[32];
  __shared__ double ljj;
  __shared__ int bad;
  if (threadIdx.x == 0) bad = 0;
  __syncthreads();
  for (int j = 0; j < n; ++j) {
    double part = 0.0;
    for (int k = threadIdx.x; k < j; k += blockDim.x) {
      const double x = w[(long long)k * n + j];
      part += x * x;
    }
    const double tot = block_sum(part, red);
    if (threadIdx.x == 0) {
      const double d = s[(long long)j * n + j] - tot;
      if (!(d > 0.0)) { bad = 1; ljj = 1.0; } else ljj = sqrt(d);
      w[(long long)j * n + j] = ljj;
    }
    __syncthreads();
    if (bad) break;
    const double inv = 1.0 / ljj;
    for (int i = j + 1 + threadIdx.x; i < n; i += blockDim.x) {
      double t = s[(long long)j * n + i];
      for (int k = 0; k < j; ++k) t -= w[(long long)k * n + i] * w[(long long)k * n + j];
      w[(long long)j * n + i] = t * inv;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0 && bad) status[m] = kStNotSpd;
}

// X = L^-T (upper triangular, row-major): column c solves L^T x = e_c by
// backward substitution; all threads walk r = n-1 .. 0 in lock step so that
// W[r][k] is a broadcast and X[k][c] a coalesced read.
__global__ void k_trinv(DevBatch B, const double* __restrict__ W, double* __restrict__ X,
                        const int* __restrict__ status) {
  const int m = blockIdx.x;
  if (status[m] != kStOk) return;
  const int n = B.ooff[m + 1] - B.ooff[m];
  const long long mo = B.moff[m];
  const double* w = W + mo;
  double* x = X + mo;
  for (int c0 = 0; c0 < n; c0 += blockDim.x) {
    const int c = c0 + threadIdx.x;
    for (int r = n - 1; r >= 0; --r) {
      if (c < n) {
        if (r > c) {
          x[(long long)r * n + c] = 0.0;
        } else {
          double t = (r == c) ? 1.0 : 0.0;
          for (int k = r + 1; k <= c; ++k) t -= w[(long long)r * n + k] * x[(long long)k * n + c];
          x[(long long)r * n + c] = t / w[(long long)r * n + r];
        }
      }
    }
  }
}

// ------------------------------------------------------------ batched GEMM
// C_m = alpha * op(A_m) * diag(ks_m) * op(B_m) + beta * C_m for every tile in
// the list (structure, tile row, tile col).  Square n_m x n_m operands with
// leading dimension n_m at offset moff[m]; K = kdim[m] if kdim != NULL.
// op(B) may gather rows of B^T through perm (eigenvector reordering).
constexpr int GT = 64, GK = 16;

__global__ void __launch_bounds__(256) k_gemm(DevBatch B, const int4* __restrict__ tiles, int ntiles,
                                              const double* __restrict__ Ab, int ta, const double* __restrict__ Bb,
                                              int tb_, const int* __restrict__ perm, const double* __restrict__ ks,
                                              const int* __restrict__ kdim, double* __restrict__ Cb, double alpha,
                                              double beta, const int* __restrict__ active) {
  __shared__ double As[2][GK][GT + 1];
  __shared__ double Bs[2][GK][GT + 1];
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int4 tl = tiles[t];
    const int m = tl.x;
    if (active && !active[m]) continue;
    const int n = B.ooff[m + 1] - B.ooff[m];
    const int K = kdim ? kdim[m] : n;
    const long long mo = B.moff[m];
    const long long vo = B.ooff[m];
    const double* A = Ab + mo;
    const double* Bm = Bb + mo;
    const int* pm = perm ? perm + vo : nullptr;
    const double* kv = ks ? ks + vo : nullptr;
    const int i0 = tl.y * GT, j0 = tl.z * GT;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    double acc[4][4];
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] = 0.0;

    auto load = [&](int buf, int k0) {
      // A tile: op(A)[i0+ii][k0+kk] -> As[kk][ii]; B tile: op(B)[k0+kk][j0+jj] -> Bs[kk][jj]
      for (int e = threadIdx.x; e < GT * GK; e += blockDim.x) {
        int ii, kk;
        if (ta) { ii = e % GT; kk = e / GT; } else { kk = e % GK; ii = e / GK; }
        const int gi = i0 + ii, gk = k0 + kk;
        double v = 0.0;
        if (gi < n && gk < K) v = ta ? A[(long long)gk * n + gi] : A[(long long)gi * n + gk];
        if (kv && gk < K) v *= kv[gk];
        As[buf][kk][ii] = v;
        int jj, kb;
        if (tb_) { kb = e % GK; jj = e / GK; } else { jj = e % GT; kb = e / GT; }
        const int gj = j0 + jj, gk2 = k0 + kb;
        double u = 0.0;
        if (gj < n && gk2 < K) {
          if (tb_) {
            const int row = pm ? pm[gj] : gj;
            u = Bm[(long long)row * n + gk2];
          } else {
            u = Bm[(long long)gk2 * n + gj];
          }
        }
        Bs[buf][kb][jj] = u;
      }
    };
    const int nk = (K + GK - 1) / GK;
    __syncthreads();
    if (nk > 0) load(0, 0);
    __syncthreads();
    for (int kt = 0; kt < nk; ++kt) {
      const int cur = kt & 1;
      if (kt + 1 < nk) load(cur ^ 1, (kt + 1) * GK);
#pragma unroll
      for (int kk = 0; kk < GK; ++kk) {
        double a[4], b[4];
#pragma unroll
        for (int x = 0; x < 4; ++x) { a[x] = As[cur][kk][ty + 16 * x]; b[x] = Bs[cur][kk][tx + 16 * x]; }
#pragma unroll
        for (int x = 0; x < 4; ++x)
#pragma unroll
          for (int y = 0; y < 4; ++y) acc[x][y] = fma(a[x], b[y], acc[x][y]);
      }
      __syncthreads();
    }
#pragma unroll
    for (int x = 0; x < 4; ++x) {
      const int gi = i0 + ty + 16 * x;
      if (gi >= n) continue;
#pragma unroll
      for (int y = 0; y < 4; ++y) {
        const int gj = j0 + tx + 16 * y;
        if (gj >= n) continue;
        double* c = Cb + mo + (long long)gi * n + gj;
        *c = beta == 0.0 ? alpha * acc[x][y] : alpha * acc[x][y] + beta * (*c);
      }
    }
  }
}

// ------------------------------------------------------------ eigensolver
// Symmetric eigenproblem of A (n x n, row-major, overwritten) for every
// active structure: w ascending, eigenvector j = row perm[j] of Zc.
__global__ void __launch_bounds__(kEigThreads) k_syev(DevBatch B, double* __restrict__ Ab, double* __restrict__ Zb,
                                                      double* __restrict__ wout, int* __restrict__ perm,
                                                      int* __restrict__ status, const int* __restrict__ active) {
  const int m = blockIdx.x;
  if (active && !active[m]) return;
  if (status[m] != kStOk) return;
  const int n = B.ooff[m + 1] - B.ooff[m];
  const long long mo = B.moff[m];
  const long long vo = B.ooff[m];
  double* A = Ab + mo;
  double* Z = Zb + mo;
  extern __shared__ double sm[];
  double* d = sm;             // n
  double* e = d + n;          // n
  double* tau = e + n;        // n
  double* vs = tau + n;       // n
  double* ps = vs + n;        // n (reused for rotation cosines)
  double* ws = ps + n;        // n (reused for rotation sines)
  __shared__ double red[kEigThreads / 32];
  __shared__ double sh_scal, sh_tau;
  __shared__ int sh_m, sh_cnt, sh_fail;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int lane = tid & 31, wid = tid >> 5, nw = nt >> 5;

  // symmetrise
  for (long long x = tid; x < (long long)n * n; x += nt) {
    const int i = (int)(x / n), j = (int)(x % n);
    if (i < j) {
      const double s = 0.5 * (A[(long long)i * n + j] + A[(long long)j * n + i]);
      A[(long long)i * n + j] = s;
      A[(long long)j * n + i] = s;
    }
  }
  for (int i = tid; i < n; i += nt) { e[i] = 0.0; tau[i] = 0.0; }
  __syncthreads();

  // ---- Householder tridiagonalisation; reflector k stored in row k of A
  for (int k = 0; k + 2 < n; ++k) {
    const int mm = n - k - 1;
    double* rowk = A + (long long)k * n + k + 1;
    double part = 0.0;
    for (int i = 1 + tid; i < mm; i += nt) part += rowk[i] * rowk[i];
    const double sigma = block_sum(part, red);
    if (tid == 0) {
      const double alpha = rowk[0];
      if (sigma == 0.0) {
        tau[k] = 0.0; e[k] = alpha; sh_tau = 0.0; sh_scal = 0.0;
      } else {
        const double r = sqrt(alpha * alpha + sigma);
        const double beta = alpha <= 0.0 ? r : -r;
        tau[k] = (beta - alpha) / beta;
        e[k] = beta;
        sh_tau = tau[k];
        sh_scal = 1.0 / (alpha - beta);
      }
    }
    __syncthreads();
    const double tk = sh_tau;
    if (tk == 0.0) continue;  // uniform across the block
    const double scal = sh_scal;
    for (int i = tid; i < mm; i += nt) {
      const double v = i == 0 ? 1.0 : rowk[i] * scal;
      vs[i] = v;
      rowk[i] = v;
    }
    __syncthreads();
    // p = tau * A22 v (one warp per row)
    double* A22 = A + (long long)(k + 1) * n + k + 1;
    for (int i = wid; i < mm; i += nw) {
      const double* ar = A22 + (long long)i * n;
      double s = 0.0;
      for (int j = lane; j < mm; j += 32) s += ar[j] * vs[j];
      s = warp_sum(s);
      if (lane == 0) ps[i] = tk * s;
    }
    __syncthreads();
    part = 0.0;
    for (int i = tid; i < mm; i += nt) part += ps[i] * vs[i];
    const double pv = block_sum(part, red);
    const double kk = 0.5 * tk * pv;
    for (int i = tid; i < mm; i += nt) ws[i] = ps[i] - kk * vs[i];
    __syncthreads();
    for (long long x = tid; x < (long long)mm * mm; x += nt) {
      const int i = (int)(x / mm), j = (int)(x % mm);
      A22[(long long)i * n + j] -= vs[i] * ws[j] + ws[i] * vs[j];
    }
    __syncthreads();
  }
  for (int i = tid; i < n; i += nt) d[i] = A[(long long)i * n + i];
  if (tid == 0 && n >= 2) e[n - 2] = A[(long long)(n - 2) * n + n - 1];
  __syncthreads();

  // ---- Zc = Q^T (row c of Zc = column c of Q), backward accumulation
  for (long long x = tid; x < (long long)n * n; x += nt) Z[x] = ((x / n) == (x % n)) ? 1.0 : 0.0;
  __syncthreads();
  for (int k = n - 3; k >= 0; --k) {
    const double tk = tau[k];
    if (tk == 0.0) continue;
    const int mm = n - k - 1;
    const double* rowk = A + (long long)k * n + k + 1;
    for (int i = tid; i < mm; i += nt) vs[i] = rowk[i];
    __syncthreads();
    double* Z22 = Z + (long long)(k + 1) * n + k + 1;
    for (int c = wid; c < mm; c += nw) {
      double* zr = Z22 + (long long)c * n;
      double s = 0.0;
      for (int r = lane; r < mm; r += 32) s += zr[r] * vs[r];
      s = warp_sum(s) * tk;
      for (int r = lane; r < mm; r += 32) zr[r] -= s * vs[r];
    }
    __syncthreads();
  }

  // ---- implicit QL; rotations of one sweep in (ps, ws), applied to rows of Zc
  if (tid == 0) { sh_fail = 0; e[n - 1] = 0.0; }
  __syncthreads();
  const double eps = 2.220446049250313e-16;
  for (int l = 0; l < n; ++l) {
    int iter = 0;
    for (;;) {
      if (tid == 0) {
        int mq = l;
        for (; mq < n - 1; ++mq) {
          const double dd = fabs(d[mq]) + fabs(d[mq + 1]);
          if (fabs(e[mq]) <= eps * dd) break;
        }
        sh_m = mq;
        sh_cnt = 0;
        if (mq != l) {
          if (++iter > 60) {
            sh_fail = 1;
          } else {
            double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
            double r = sqrt(g * g + 1.0);
            g = d[mq] - d[l] + e[l] / (g + (g >= 0.0 ? r : -r));
            double s = 1.0, c = 1.0, p = 0.0;
            int i = mq - 1;
            bool underflow = false;
            for (; i >= l; --i) {
              const double f = s * e[i];
              const double b = c * e[i];
              r = sqrt(f * f + g * g);
              e[i + 1] = r;
              if (r == 0.0) { d[i + 1] -= p; e[mq] = 0.0; underflow = true; break; }
              const double ri = 1.0 / r;
              s = f * ri;
              c = g * ri;
              g = d[i + 1] - p;
              r = (d[i] - g) * s + 2.0 * c * b;
              p = s * r;
              d[i + 1] = g + p;
              g = c * r - b;
              ps[sh_cnt] = c;
              ws[sh_cnt] = s;
              ++sh_cnt;
            }
            if (!underflow) { d[l] -= p; e[l] = g; e[mq] = 0.0; }
          }
        }
      }
      __syncthreads();
      const int mq = sh_m, cnt = sh_cnt, failed = sh_fail;
      __syncthreads();  // everyone has read the sweep bounds before thread 0 rewrites them
      if (mq == l || failed) break;
      // apply rotations i = mq-1, mq-2, ... (cnt of them) to rows i, i+1 of Zc
      for (int r = tid; r < n; r += nt) {
        double f = Z[(long long)mq * n + r];
        for (int t = 0; t < cnt; ++t) {
          const int i = mq - 1 - t;
          const double c = ps[t], s = ws[t];
          const double z = Z[(long long)i * n + r];
          Z[(long long)(i + 1) * n + r] = s * z + c * f;
          f = c * z - s * f;
        }
        Z[(long long)(mq - cnt) * n + r] = f;
      }
      __syncthreads();
    }
    if (sh_fail) break;  // written before the last barrier, uniform
  }
  if (sh_fail) {
    if (tid == 0) status[m] = kStEigenFailed;  // k_fermi retires the structure
    return;
  }
  // ---- ascending order by rank (ties by index)
  for (int i = tid; i < n; i += nt) {
    const double di = d[i];
    int rank = 0;
    for (int j = 0; j < n; ++j) {
      const double dj = d[j];
      rank += (dj < di || (dj == di && j < i)) ? 1 : 0;
    }
    perm[vo + rank] = i;
    wout[vo + rank] = di;
  }
}

}  // namespace tb
