// Mixed-precision form of the SCF iteration.
//
// Each structure runs in one of two phases (MolState::phase):
//  * mixed (0): the contractions F' = X^T F X, C = X V and P = C f C^T are
//    TF32x3 split-precision tensor-core GEMMs accumulated in FP32 on
//    FP64-stored operands (k_gemm_tc, tb_tc.cu);
//  * FP64 (1): entered once the mixed phase meets the (loosened) convergence
//    test; the same contractions as FP64 GEMMs.  A structure retires only
//    after at least two FP64 iterations and the full-accuracy convergence test.
// In both phases the eigensolve is the FP32 k_syev_f32 (whose vectors are
// orthogonal to about n * 1e-7) followed by FP64 refinement of the eigenpairs,
// GEMMs included: one step in the mixed phase, two in the FP64 phase.  A step
// is Ogita-Aishima iterative refinement (T. Ogita, K. Aishima, Japan J.
// Indust. Appl. Math. 35 (2018) 1007-1035, algorithm RefSyEv) with an exact
// Rayleigh-Ritz solve inside clusters of near-degenerate eigenvalues (their
// treatment of clustered eigenvalues, same journal 36 (2019) 435-459); without
// it the second step turns the unresolved rotations inside a cluster into
// large first-order updates and loses orthogonality.  Fermi level, Fock build,
// Mulliken analysis, energies and Broyden mixing are FP64 throughout.
// The kernels here follow the batch conventions of tb_linalg.cu: tile lists of
// (structure, tile row, tile col), per-structure masks, row-major N x N blocks
// at moff[m].
#include "tb_common.cuh"
#include "tb_kernels.h"

namespace tb {

namespace {
constexpr int MT = 64;
}  // namespace

// lo[m] = active and in the mixed phase; hi[m] = active and in the FP64 phase.
__global__ void k_phase_masks(int nmol, const int* __restrict__ active, const int* __restrict__ phase,
                              int* __restrict__ lo, int* __restrict__ hi) {
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < nmol; m += gridDim.x * blockDim.x) {
    const int a = active[m];
    lo[m] = a && phase[m] == 0;
    hi[m] = a && phase[m] != 0;
  }
}

// Af = (float) F' for the masked structures, tile by tile.
__global__ void k_to_f32(DevBatch B, const int4* __restrict__ tiles, int ntiles, const double* __restrict__ F,
                         float* __restrict__ Af, const int* __restrict__ mask) {
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int4 tl = tiles[t];
    const int m = tl.x;
    if (!mask[m]) continue;
    const int n = B.ooff[m + 1] - B.ooff[m];
    const long long mo = B.moff[m];
    for (int e = threadIdx.x; e < MT * MT; e += blockDim.x) {
      const int i = tl.y * MT + e / MT, j = tl.z * MT + e % MT;
      if (i < n && j < n) Af[mo + (long long)i * n + j] = (float)F[mo + (long long)i * n + j];
    }
  }
}

// V[i][j] = Zf[perm[j]][i] in FP64: eigenvector j (ascending) as column j.
__global__ void k_gather_vectors(DevBatch B, const int4* __restrict__ tiles, int ntiles, const float* __restrict__ Zf,
                                 const int* __restrict__ perm, double* __restrict__ V, const int* __restrict__ mask) {
  __shared__ float tile[32][33];
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
    const int4 tl = tiles[t];
    const int m = tl.x;
    if (!mask[m]) continue;
    const int n = B.ooff[m + 1] - B.ooff[m];
    const long long mo = B.moff[m];
    const int* pm = perm + B.ooff[m];
    // the 64 x 64 tile as four 32 x 32 transposes
    for (int q = 0; q < 4; ++q) {
      const int i0 = tl.y * MT + 32 * (q >> 1), j0 = tl.z * MT + 32 * (q & 1);
      __syncthreads();
      for (int e = threadIdx.x; e < 32 * 32; e += blockDim.x) {
        const int jj = e / 32, ii = e % 32;  // row perm[j0+jj] of Zf read along i (coalesced)
        const int j = j0 + jj, i = i0 + ii;
        tile[jj][ii] = (j < n && i < n) ? Zf[mo + (long long)pm[j] * n + i] : 0.0f;
      }
      __syncthreads();
      for (int e = threadIdx.x; e < 32 * 32; e += blockDim.x) {
        const int ii = e / 32, jj = e % 32;
        const int i = i0 + ii, j = j0 + jj;
        if (i < n && j < n) V[mo + (long long)i * n + j] = (double)tile[jj][ii];
      }
    }
  }
}

// One refinement step, coefficient part, one CTA per masked structure.
// In: G = V^T V, Sm = V^T A V (FP64) and V.
//  1. lambda_i = Sm_ii / G_ii, delta = 2 (||Sm - diag(lambda)||_F +
//     max|lambda| ||I - G||_F) (Frobenius norms bound the published 2-norms
//     from above, so delta is conservative);
//  2. clusters = maximal index runs with |lambda_{i+1} - lambda_i| <= delta
//     (runs longer than kClusterMax are cut into pieces);
//  3. per cluster J: G_JJ = L L^T, M = L^-1 Sm_JJ L^-T = U diag U^T (cyclic
//     Jacobi in parallel order), T_J = L^-T U with columns in ascending order;
//     V_:J <- V_:J T_J, G <- T^T G T, Sm <- T^T Sm T (rows and columns J);
//  4. lambda recomputed, E (overwrites G) with R = I - G:
//       E_ij = (Sm_ij + lambda_j R_ij) / (lambda_j - lambda_i)  if |lambda_j - lambda_i| > delta
//            = R_ij / 2                                          otherwise (and on the diagonal).
// The caller then forms V + V E.  Refined eigenvalues go to w.  Steps 2-3 run
// only for structures with rr_mask set: a single step (or a second step after
// one with Rayleigh-Ritz) needs no cluster solve, since clustered pairs then
// only carry rotations inside the cluster, which leave the density unchanged.
// Dynamic shared memory: oa_smem_bytes(nmax).
__global__ void __launch_bounds__(256) k_oa_step(DevBatch B, double* __restrict__ G, double* __restrict__ Sm,
                                                 double* __restrict__ Vb, double* __restrict__ w,
                                                 const int* __restrict__ mask, const int* __restrict__ rr_mask) {
  const int m = blockIdx.x;
  if (!mask[m]) return;
  const int n = B.ooff[m + 1] - B.ooff[m];
  const long long mo = B.moff[m];
  double* g = G + mo;
  double* s = Sm + mo;
  double* V = Vb + mo;
  double* lam = w + B.ooff[m];
  constexpr int KM = kClusterMax;
  extern __shared__ __align__(16) double oa_sm[];
  double* Lm = oa_sm;            // KM x KM  Cholesky factor of G_JJ
  double* M = Lm + KM * KM;      // KM x KM  projected block, then T
  double* U = M + KM * KM;       // KM x KM  accumulated Jacobi rotations
  double* ev = U + KM * KM;      // KM       eigenvalues of the block
  double* cs = ev + KM;          // KM       cosines | sines of one round
  int* cstart = reinterpret_cast<int*>(cs + KM);  // n + 1 cluster starts
  int* csize = cstart + n + 1;                    // n + 1 cluster sizes
  __shared__ double red[32];
  __shared__ double sh_amax, sh_off;
  __shared__ int ncl;
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, wid = tid >> 5, nw = nt >> 5;

  // ---- 1. lambda and delta
  double amax = 0.0;
  for (int i = tid; i < n; i += nt) {
    const double l = s[(long long)i * n + i] / g[(long long)i * n + i];
    lam[i] = l;
    amax = fmax(amax, fabs(l));
  }
  for (int o = 16; o > 0; o >>= 1) amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
  if (lane == 0) red[wid] = amax;
  __syncthreads();  // also publishes lam
  if (tid == 0) {
    double a = 0.0;
    for (int k = 0; k < nw; ++k) a = fmax(a, red[k]);
    sh_amax = a;
  }
  __syncthreads();
  double so = 0.0, rr = 0.0;
  for (long long e = tid; e < (long long)n * n; e += nt) {
    const int i = (int)(e / n), j = (int)(e - (long long)i * n);
    const double r = (i == j ? 1.0 : 0.0) - g[e];
    const double d = i == j ? s[e] - lam[i] : s[e];
    so += d * d;
    rr += r * r;
  }
  so = block_sum(so, red);
  rr = block_sum(rr, red);
  const double delta = 2.0 * (sqrt(so) + sh_amax * sqrt(rr));

  // ---- 2. clusters (only where rr_mask asks for the Rayleigh-Ritz solve)
  if (tid == 0 && !(rr_mask && rr_mask[m])) ncl = 0;
  if (tid == 0 && rr_mask && rr_mask[m]) {
    int c = 0, i = 0;
    while (i < n) {
      int j = i;
      while (j + 1 < n && j + 1 - i < KM && fabs(lam[j + 1] - lam[j]) <= delta) ++j;
      if (j > i) { cstart[c] = i; csize[c] = j - i + 1; ++c; }
      i = j + 1;
    }
    ncl = c;
  }
  __syncthreads();

  // ---- 3. Rayleigh-Ritz inside each cluster
  for (int c = 0; c < ncl; ++c) {
    const int j0 = cstart[c], k = csize[c];
    for (int e = tid; e < k * k; e += nt) {
      const int i = e / k, j = e % k;
      Lm[i * KM + j] = g[(long long)(j0 + i) * n + j0 + j];
      M[i * KM + j] = s[(long long)(j0 + i) * n + j0 + j];
    }
    __syncthreads();
    // Cholesky of G_JJ (lower triangle, in place), column by column
    for (int j = 0; j < k; ++j) {
      if (tid == 0) {
        double d = Lm[j * KM + j];
        for (int p = 0; p < j; ++p) d -= Lm[j * KM + p] * Lm[j * KM + p];
        Lm[j * KM + j] = sqrt(fmax(d, 1e-300));
      }
      __syncthreads();
      for (int i = j + 1 + tid; i < k; i += nt) {
        double t = Lm[i * KM + j];
        for (int p = 0; p < j; ++p) t -= Lm[i * KM + p] * Lm[j * KM + p];
        Lm[i * KM + j] = t / Lm[j * KM + j];
      }
      __syncthreads();
    }
    // M <- L^-1 M L^-T: forward substitution on the columns, transpose, again
    for (int pass = 0; pass < 2; ++pass) {
      for (int col = tid; col < k; col += nt) {
        for (int i = 0; i < k; ++i) {
          double t = M[i * KM + col];
          for (int p = 0; p < i; ++p) t -= Lm[i * KM + p] * M[p * KM + col];
          M[i * KM + col] = t / Lm[i * KM + i];
        }
      }
      __syncthreads();
      for (int e = tid; e < k * k; e += nt) {
        const int i = e / k, j = e % k;
        if (i < j) {
          const double t = M[i * KM + j];
          M[i * KM + j] = M[j * KM + i];
          M[j * KM + i] = t;
        }
      }
      __syncthreads();
    }
    for (int e = tid; e < k * k; e += nt) {
      const int i = e / k, j = e % k;
      U[i * KM + j] = i == j ? 1.0 : 0.0;
      if (i < j) {  // symmetrise the rounding
        const double t = 0.5 * (M[i * KM + j] + M[j * KM + i]);
        M[i * KM + j] = t;
        M[j * KM + i] = t;
      }
    }
    __syncthreads();
    // cyclic Jacobi, round-robin pairing of kk players (kk even; index >= k sits out)
    const int kk = k + (k & 1);
    for (int sweep = 0; sweep < 40; ++sweep) {
      double off = 0.0, dia = 0.0;
      for (int e = tid; e < k * k; e += nt) {
        const int i = e / k, j = e % k;
        const double x = M[i * KM + j];
        if (i == j) dia += x * x; else off += x * x;
      }
      off = block_sum(off, red);
      dia = block_sum(dia, red);
      if (tid == 0) sh_off = off;
      __syncthreads();
      if (!(sh_off > 1e-30 * dia)) break;
      for (int r = 0; r < kk - 1; ++r) {
        // pair t of round r: (r, kk-1) for t = 0, else ((r+t) mod (kk-1), (r-t) mod (kk-1))
        for (int t = tid; t < kk / 2; t += nt) {
          int p = t == 0 ? r : (r + t) % (kk - 1);
          int q = t == 0 ? kk - 1 : (r - t + kk - 1) % (kk - 1);
          if (p > q) { const int x = p; p = q; q = x; }
          double cc = 1.0, ss = 0.0;
          if (q < k) {
            const double apq = M[p * KM + q];
            if (apq != 0.0) {
              const double th = (M[q * KM + q] - M[p * KM + p]) / (2.0 * apq);
              const double tt = (th >= 0.0 ? 1.0 : -1.0) / (fabs(th) + sqrt(th * th + 1.0));
              cc = 1.0 / sqrt(tt * tt + 1.0);
              ss = tt * cc;
            }
          }
          cs[t] = cc;
          cs[KM / 2 + t] = ss;
        }
        __syncthreads();
        // rows: M <- J^T M
        for (int e = tid; e < (kk / 2) * k; e += nt) {
          const int t = e / k, j = e % k;
          int p = t == 0 ? r : (r + t) % (kk - 1);
          int q = t == 0 ? kk - 1 : (r - t + kk - 1) % (kk - 1);
          if (p > q) { const int x = p; p = q; q = x; }
          if (q >= k) continue;
          const double cc = cs[t], ss = cs[KM / 2 + t];
          const double xp = M[p * KM + j], xq = M[q * KM + j];
          M[p * KM + j] = cc * xp - ss * xq;
          M[q * KM + j] = ss * xp + cc * xq;
        }
        __syncthreads();
        // columns: M <- M J, U <- U J
        for (int e = tid; e < (kk / 2) * k; e += nt) {
          const int t = e / k, i = e % k;
          int p = t == 0 ? r : (r + t) % (kk - 1);
          int q = t == 0 ? kk - 1 : (r - t + kk - 1) % (kk - 1);
          if (p > q) { const int x = p; p = q; q = x; }
          if (q >= k) continue;
          const double cc = cs[t], ss = cs[KM / 2 + t];
          const double xp = M[i * KM + p], xq = M[i * KM + q];
          M[i * KM + p] = cc * xp - ss * xq;
          M[i * KM + q] = ss * xp + cc * xq;
          const double up = U[i * KM + p], uq = U[i * KM + q];
          U[i * KM + p] = cc * up - ss * uq;
          U[i * KM + q] = ss * up + cc * uq;
        }
        __syncthreads();
      }
    }
    // ascending order inside the cluster (rank sort), sorted U into M
    for (int i = tid; i < k; i += nt) ev[i] = M[i * KM + i];
    __syncthreads();
    for (int i = tid; i < k; i += nt) {
      int rank = 0;
      for (int j = 0; j < k; ++j) rank += (ev[j] < ev[i] || (ev[j] == ev[i] && j < i)) ? 1 : 0;
      for (int r = 0; r < k; ++r) M[r * KM + rank] = U[r * KM + i];
    }
    __syncthreads();
    // T = L^-T U_sorted by back substitution, column by column, in place
    for (int col = tid; col < k; col += nt) {
      for (int i = k - 1; i >= 0; --i) {
        double t = M[i * KM + col];
        for (int p = i + 1; p < k; ++p) t -= Lm[p * KM + i] * M[p * KM + col];
        M[i * KM + col] = t / Lm[i * KM + i];
      }
    }
    __syncthreads();
    // V, G, Sm: columns J <- (.)_:J T (one warp per row); G, Sm rows J <- T^T (.)_J: (one warp per column)
    for (int pass = 0; pass < 5; ++pass) {
      double* X = pass == 0 ? V : (pass < 3 ? g : s);
      const bool rows = pass == 2 || pass == 4;
      for (int r = wid; r < n; r += nw) {
        double o0 = 0.0, o1 = 0.0;
        const int c0 = lane, c1 = lane + 32;
        for (int p = 0; p < k; ++p) {
          const double x = rows ? X[(long long)(j0 + p) * n + r] : X[(long long)r * n + j0 + p];
          if (c0 < k) o0 += x * M[p * KM + c0];
          if (c1 < k) o1 += x * M[p * KM + c1];
        }
        __syncwarp();
        if (rows) {
          if (c0 < k) X[(long long)(j0 + c0) * n + r] = o0;
          if (c1 < k) X[(long long)(j0 + c1) * n + r] = o1;
        } else {
          if (c0 < k) X[(long long)r * n + j0 + c0] = o0;
          if (c1 < k) X[(long long)r * n + j0 + c1] = o1;
        }
      }
      __syncthreads();
    }
    for (int i = tid; i < k; i += nt)
      lam[j0 + i] = s[(long long)(j0 + i) * n + j0 + i] / g[(long long)(j0 + i) * n + j0 + i];
    __syncthreads();
  }

  // ---- 4. E into G
  for (long long e = tid; e < (long long)n * n; e += nt) {
    const int i = (int)(e / n), j = (int)(e - (long long)i * n);
    const double r = (i == j ? 1.0 : 0.0) - g[e];
    const double gap = lam[j] - lam[i];
    double x;
    if (i != j && fabs(gap) > delta) x = (s[e] + lam[j] * r) / gap;
    else x = 0.5 * r;
    g[e] = x;
  }
}

}  // namespace tb
