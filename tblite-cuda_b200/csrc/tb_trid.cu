// Householder tridiagonalisation held entirely in shared memory, one thread
// block cluster per structure (phase 1 of the eigensolver, sygvd_solver's
// dsytrd step, src/lapack/sygvd.cu:223-313; the eigenvectors follow in k_syev).
//
// The matrix lives in the clusters' shared memory for the whole reduction, so
// the n - 2 Householder steps never touch L2 or DRAM: the one-CTA kernel
// (k_syev's tridiagonalise) streams the trailing block from L2/DRAM at every
// step and is bound by those round trips.  Layout:
//  * the upper triangle of tiles (16 x 16 doubles, row-major, the diagonal
//    tiles stored whole and symmetric); tile row I belongs to CTA owner[I]
//    (greedy balance of the tile counts), and a CTA stores its tiles ordered
//    by tile row DEScending, so the tiles still live at step k (tile rows
//    >= (k+1)/16) are a prefix of its tile list;
//  * per tile: the row partial sums (16) and column partial sums (16) of p;
//  * vectors of the padded order np = 16 ceil(n/16): the reflector of the
//    step (x, two alternating buffers), the previous step's (v, w)
//    interleaved, p / the new row, and the exchange buffers of the cluster:
//    cvec (this CTA's share of p, two step parities) and pub (the next
//    reflector's row, published by its owner, two parities).
// Step k (reflector k from row k, trailing block k+1..n-1):
//  A. every CTA of the cluster forms, redundantly and with identical
//     arithmetic, p_{k-1} = tau sum_c cvec_c (fixed rank order), w_{k-1} =
//     p - (tau/2)(p.v)v and row k of the updated matrix from the row its owner
//     published, then reflector k (alpha, sigma, beta, tau as LAPACK's dlarfg);
//  B. one pass over the CTA's live tiles applies the previous rank-2 update
//     A -= v w^T + w v^T and accumulates A x (x = reflector k) as row sums
//     (lanes on columns, reduced once per tile by 15 shuffles) and column
//     sums (off-diagonal tiles only); the owner of row k+1 publishes it;
//  C. the CTA adds its tiles' partials per column in a fixed order into
//     cvec[k & 1]; one cluster barrier.
// Outputs match k_syev's tridiagonalise: reflector k (v_k, v_k[k+1] = 1) in
// row k of A from column k+1 on; d, e and tau in the structure's scratch
// slice (d at 0, e at n, tau at 2n), which k_syev reads instead of
// tridiagonalising.  A is taken as symmetric: (A + A^T)/2 is loaded.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "tb_common.cuh"
#include "tb_kernels.h"

namespace cg = cooperative_groups;

namespace tb {

namespace {

constexpr int TT = kTridTile;                       // tile side
constexpr int kThreads = kTridThreads;              // 16 warps, 32 half-warps
constexpr int kWarps = kThreads / 32;

// Tile rows to cluster ranks: tile row I (T - I tiles) goes to the rank with
// the fewest tiles so far (lowest rank on ties).  Returns the largest count.
__host__ __device__ inline int trid_owners(int T, int C, int* owner) {
  int cnt[kTridMaxCluster] = {0};
  for (int I = 0; I < T; ++I) {
    int c = 0;
    for (int r = 1; r < C; ++r)
      if (cnt[r] < cnt[c]) c = r;
    if (owner) owner[I] = c;
    cnt[c] += T - I;
  }
  int mx = 0;
  for (int r = 0; r < C; ++r) mx = cnt[r] > mx ? cnt[r] : mx;
  return mx;
}

// Shared-memory layout of one CTA (offsets in doubles; ints after the doubles).
struct TridSmem {
  int T, np, mt;
  int o_rowp, o_colp, o_x, o_upd, o_pr, o_cvec, o_pub, o_red, o_fin, o_int, total_doubles;
  __host__ __device__ TridSmem(int n, int C) {
    T = (n + TT - 1) / TT;
    np = TT * T;
    mt = trid_owners(T, C, nullptr);
    int o = mt * TT * TT;
    o_rowp = o; o += mt * TT;
    o_colp = o; o += mt * TT;
    o_x = o; o += 2 * np;
    o_upd = o; o += 2 * np;
    o_pr = o; o += np;
    o_cvec = o; o += 2 * np;
    o_pub = o; o += 2 * np;
    o_red = o; o += 2 * kWarps;
    o_fin = o; o += 2;
    o_int = o;
    const int ints = 3 * T + 1 + mt;
    total_doubles = o + (ints + 1) / 2;
  }
  __host__ __device__ size_t bytes() const { return (size_t)total_doubles * sizeof(double); }
};

// sum over the block in a fixed order; red: kWarps doubles, alternated by the
// caller between consecutive calls (so no barrier is needed before the write)
__device__ __forceinline__ double bsum(double v, double* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  v = warp_sum(v);
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double t = 0.0;
#pragma unroll
  for (int w = 0; w < kWarps; ++w) t += red[w];
  return t;
}

// a - (vi wj + wi vj) with the two products rounded separately and added
// commutatively, so the (i, j) and (j, i) entries of a diagonal tile stay equal
__device__ __forceinline__ double rank2(double a, double vi, double wi, double vj, double wj) {
  return __dsub_rn(a, __dadd_rn(__dmul_rn(vi, wj), __dmul_rn(wi, vj)));
}

template <int C>
struct Cluster {
  __device__ static int rank() {
    if constexpr (C == 1) return 0;
    else return (int)cg::this_cluster().block_rank();
  }
  __device__ static void sync() {
    if constexpr (C == 1) __syncthreads();
    else cg::this_cluster().sync();
  }
  template <typename P>
  __device__ static P* at(P* p, int r) {
    if constexpr (C == 1) return p;
    else return cg::this_cluster().map_shared_rank(p, (unsigned)r);
  }
};

template <int C>
__global__ void __launch_bounds__(kThreads, 1) k_trid_smem(DevBatch B, double* __restrict__ Ab,
                                                           double* __restrict__ Sb, const int* __restrict__ status,
                                                           const int* __restrict__ active,
                                                           const int* __restrict__ list) {
  const int m = list[blockIdx.x / C];
  if ((active && !active[m]) || status[m] != kStOk) return;  // the whole cluster leaves together
  const int n = B.ooff[m + 1] - B.ooff[m];
  const int rank = Cluster<C>::rank();
  const TridSmem L(n, C);
  const int T = L.T, np = L.np;
  extern __shared__ __align__(16) double trid_sm[];
  double* tiles = trid_sm;
  double* rowp = trid_sm + L.o_rowp;
  double* colp = trid_sm + L.o_colp;
  double* X = trid_sm + L.o_x;                        // x of step k in X + (k & 1) np
  double2* upd = reinterpret_cast<double2*>(trid_sm + L.o_upd);  // (v, w) of the previous step
  double* pr = trid_sm + L.o_pr;                      // p, then the new row
  double* cvec = trid_sm + L.o_cvec;                  // [2][np]
  double* pub = trid_sm + L.o_pub;                    // [2][np]
  double* red = trid_sm + L.o_red;                    // [2][kWarps]
  double* fin = trid_sm + L.o_fin;                    // A(n-1, n-1) before the last update
  int* owner = reinterpret_cast<int*>(trid_sm + L.o_int);
  int* rowstart = owner + T;
  int* live = rowstart + T;                           // [T + 1]
  int* tij = live + T + 1;                            // tile (I, J) of slot s: I << 16 | J
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const long long mo = B.moff[m];
  double* A = Ab + mo;
  double* dout = Sb + mo;
  double* eout = dout + n;
  double* tout = eout + n;

  if (tid == 0) {
    trid_owners(T, C, owner);
    int s = 0;
    for (int I = T - 1; I >= 0; --I) {
      rowstart[I] = -1;
      if (owner[I] != rank) continue;
      rowstart[I] = s;
      for (int J = I; J < T; ++J) tij[s + J - I] = (I << 16) | J;
      s += T - I;
    }
    int acc = 0;
    live[T] = 0;
    for (int K0 = T - 1; K0 >= 0; --K0) {
      if (owner[K0] == rank) acc += T - K0;
      live[K0] = acc;
    }
  }
  __syncthreads();
  const int nown = live[0];
  // ---- load (A + A^T)/2 into the own tiles, zero beyond n; clear the vectors
  for (int e = tid; e < nown * TT * TT; e += kThreads) {
    const int s = e >> 8, r = (e >> 4) & 15, l = e & 15;
    const int I = tij[s] >> 16, J = tij[s] & 0xffff;
    const int i = TT * I + r, j = TT * J + l;
    double v = 0.0;
    if (i < n && j < n) v = 0.5 * (A[(long long)i * n + j] + A[(long long)j * n + i]);
    tiles[e] = v;
  }
  for (int j = tid; j < np; j += kThreads) {
    X[j] = 0.0; X[np + j] = 0.0;
    upd[j] = make_double2(0.0, 0.0);
    cvec[j] = 0.0; cvec[np + j] = 0.0;
    pub[j] = 0.0; pub[np + j] = 0.0;
  }
  __syncthreads();
  if (owner[0] == rank) {  // row 0 published for reflector 0
    for (int j = tid; j < np; j += kThreads) pub[j] = tiles[(rowstart[0] + (j >> 4)) * TT * TT + (j & 15)];
  }
  Cluster<C>::sync();

  double tau_prev = 0.0;
  for (int k = 0; k < n - 2; ++k) {
    const int K0 = (k + 1) >> 4;
    double* xprev = X + ((k - 1) & 1) * np;
    double* xcur = X + (k & 1) * np;
    double* redA = red + (k & 1) * kWarps;
    double* redB = red + ((k + 1) & 1) * kWarps;
    // ---- A. p_{k-1}, w_{k-1}, row k of the updated matrix, reflector k.  The
    // remote loads of a thread (its entries of every rank's cvec, its entries of
    // the published row and entry k of the cvecs) are issued together.
    double sq = 0.0;
    if (k == 0) {
      const double* prow = Cluster<C>::at(pub, owner[0]);
      for (int j = tid; j < np; j += kThreads) {
        const double rj = prow[j];
        pr[j] = rj;
        if (j >= 2 && j < n) sq += rj * rj;
      }
    } else {
      const int par = (k - 1) & 1;
      const double* prow = Cluster<C>::at(pub, owner[k >> 4]) + (k & 1) * np;
      constexpr int kPer = (kTridMaxN + kThreads - 1) / kThreads;  // entries per thread
      double sj[kPer], rowj[kPer];
      double sk = 0.0;
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const double* cv = Cluster<C>::at(cvec, c) + par * np;
        sk += cv[k];
#pragma unroll
        for (int q = 0; q < kPer; ++q) {
          const int j = tid + q * kThreads;
          const double x = j < np ? cv[j] : 0.0;
          sj[q] = c == 0 ? x : sj[q] + x;
        }
      }
#pragma unroll
      for (int q = 0; q < kPer; ++q) {
        const int j = tid + q * kThreads;
        rowj[q] = (j >= k && j < np) ? prow[j] : 0.0;
      }
      double part = 0.0;
#pragma unroll
      for (int q = 0; q < kPer; ++q) {
        const int j = tid + q * kThreads;
        if (j >= k && j < np) part += tau_prev * sj[q] * xprev[j];
      }
      const double dot = bsum(part, redA);
      const double kk = 0.5 * tau_prev * dot;
      const double vk = xprev[k];
      const double wk = tau_prev * sk - kk * vk;
#pragma unroll
      for (int q = 0; q < kPer; ++q) {
        const int j = tid + q * kThreads;
        if (j >= np) break;
        const double vj = xprev[j];
        double wj = 0.0;
        if (j >= k) {
          wj = tau_prev * sj[q] - kk * vj;
          const double rj = rowj[q] - (vk * wj + wk * vj);
          pr[j] = rj;
          if (j >= k + 2 && j < n) sq += rj * rj;
        }
        upd[j] = make_double2(vj, wj);
      }
    }
    const double sigma = bsum(sq, redB);
    const double alpha = pr[k + 1];
    double beta, tk, scal;
    const bool refl = sigma != 0.0;
    if (refl) {
      const double rr = sqrt(alpha * alpha + sigma);
      beta = alpha <= 0.0 ? rr : -rr;
      tk = (beta - alpha) / beta;
      scal = 1.0 / (alpha - beta);
    } else {
      beta = alpha; tk = 0.0; scal = 0.0;
    }
    for (int j = tid; j < np; j += kThreads) {
      double x = 0.0;
      if (j == k + 1) x = 1.0;
      else if (j > k + 1 && j < n && refl) x = pr[j] * scal;
      xcur[j] = x;
      if (rank == 0 && j > k && j < n) A[(long long)k * n + j] = x;
    }
    if (rank == 0 && tid == 0) {
      dout[k] = pr[k];
      eout[k] = beta;
      tout[k] = tk;
    }
    tau_prev = tk;
    __syncthreads();
    // ---- B. rank-2 update of the live tiles with (v, w) of step k-1, partial
    // sums of A x.  A half-warp takes a tile (lane l on column 16 J + l): the
    // 16 tile values and the row vectors are loaded before anything is stored,
    // then the 16 row partials are transpose-reduced over the 16 lanes.
    {
      const int nlive = live[K0];
      const int half = lane >> 4, l = lane & 15;
      const int kp1 = k + 1;
      double* pubn = pub + (kp1 & 1) * np;
      for (int base = 2 * wid; base < nlive; base += 2 * kWarps) {
        const int t = base + half;
        const bool valid = t < nlive;
        const int s = valid ? t : base;
        const int I = tij[s] >> 16, J = tij[s] & 0xffff;
        double* tp = tiles + s * TT * TT;
        const int j = TT * J + l;
        const double2 uj = upd[j];
        const double xj = xcur[j];
        double a[TT];
#pragma unroll
        for (int r = 0; r < TT; ++r) a[r] = tp[TT * r + l];
        const int rpub = kp1 - TT * I;  // row of this tile to publish (owner of row k+1)
        // the owner of A(n-1, n-1) keeps it before the last update
        const bool last = k == n - 3 && I == (n - 1) >> 4 && I == J && l == ((n - 1) & 15);
        double racc[TT];
        double cacc = 0.0;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          double2 ui[TT / 2];
          double xi[TT / 2];
#pragma unroll
          for (int q = 0; q < TT / 2; ++q) {
            ui[q] = upd[TT * I + 8 * h + q];
            xi[q] = xcur[TT * I + 8 * h + q];
          }
#pragma unroll
          for (int q = 0; q < TT / 2; ++q) {
            const int r = 8 * h + q;
            const double x = rank2(a[r], ui[q].x, ui[q].y, uj.x, uj.y);
            racc[r] = x * xj;
            cacc = fma(x, xi[q], cacc);
            if (valid) {
              tp[TT * r + l] = x;
              if (r == rpub) pubn[j] = x;
              if (last && r == ((n - 1) & 15)) fin[0] = x;
            }
          }
        }
        // transpose-reduce the 16 row partials over the 16 lanes: lane l ends with row l
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const bool up = l & 8;
          const double snd = up ? racc[q] : racc[q + 8];
          const double kp = up ? racc[q + 8] : racc[q];
          racc[q] = kp + __shfl_xor_sync(0xffffffffu, snd, 8);
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const bool up = l & 4;
          const double snd = up ? racc[q] : racc[q + 4];
          const double kp = up ? racc[q + 4] : racc[q];
          racc[q] = kp + __shfl_xor_sync(0xffffffffu, snd, 4);
        }
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const bool up = l & 2;
          const double snd = up ? racc[q] : racc[q + 2];
          const double kp = up ? racc[q + 2] : racc[q];
          racc[q] = kp + __shfl_xor_sync(0xffffffffu, snd, 2);
        }
        {
          const bool up = l & 1;
          const double snd = up ? racc[0] : racc[1];
          const double kp = up ? racc[1] : racc[0];
          racc[0] = kp + __shfl_xor_sync(0xffffffffu, snd, 1);
        }
        if (valid) {
          rowp[s * TT + l] = racc[0];
          colp[s * TT + l] = I == J ? 0.0 : cacc;
        }
      }
    }
    __syncthreads();
    // ---- C. this CTA's share of p for column blocks >= K0, fixed order: a
    // warp per column block J, lane l on column 16 J + l; the first half-warp
    // adds the column partials of the own tiles (I, J), I < J (increasing I),
    // the second the row partials of tile row J if owned (increasing J2)
    {
      double* cv = cvec + (k & 1) * np;
      const int half = lane >> 4, l = lane & 15;
      for (int J = K0 + wid; J < T; J += kWarps) {
        double sacc = 0.0;
        if (half == 0) {
          for (int I = K0; I < J; ++I)
            if (owner[I] == rank) sacc += colp[(rowstart[I] + J - I) * TT + l];
        } else if (owner[J] == rank) {
          const int r0 = rowstart[J];
          for (int J2 = J; J2 < T; ++J2) sacc += rowp[(r0 + J2 - J) * TT + l];
        }
        sacc += __shfl_xor_sync(0xffffffffu, sacc, 16);
        if (half == 0) cv[TT * J + l] = sacc;
      }
    }
    Cluster<C>::sync();
  }
  // ---- the last 2 x 2 block: update with (v, w) of step n-3
  if (rank == 0 && tid == 0 && n >= 3) {
    const int k = n - 2, par = (k - 1) & 1;
    const double* xprev = X + par * np;
    double s2 = 0.0, s3 = 0.0;
    for (int c = 0; c < C; ++c) {
      const double* cv = Cluster<C>::at(cvec, c) + par * np;
      s2 += cv[n - 2];
      s3 += cv[n - 1];
    }
    const double p2 = tau_prev * s2, p3 = tau_prev * s3;
    const double v2 = xprev[n - 2], v3 = xprev[n - 1];
    const double kk = 0.5 * tau_prev * (p2 * v2 + p3 * v3);
    const double w2 = p2 - kk * v2, w3 = p3 - kk * v3;
    const double* prow = Cluster<C>::at(pub, owner[(n - 2) >> 4]) + ((n - 2) & 1) * np;
    const double a33 = Cluster<C>::at(fin, owner[(n - 1) >> 4])[0];
    dout[n - 2] = rank2(prow[n - 2], v2, w2, v2, w2);
    eout[n - 2] = rank2(prow[n - 1], v2, w2, v3, w3);
    dout[n - 1] = rank2(a33, v3, w3, v3, w3);
  }
  Cluster<C>::sync();  // no CTA leaves while another reads its shared memory
}

template <int C>
cudaError_t launch_c(const DevBatch& B, double* A, double* Sb, const int* status, const int* active, const int* list,
                     int cnt, size_t smem, cudaStream_t st) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)(cnt * C));
  cfg.blockDim = dim3(kThreads);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeClusterDimension;
  at[0].val.clusterDim.x = C;
  at[0].val.clusterDim.y = 1;
  at[0].val.clusterDim.z = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_trid_smem<C>, B, A, Sb, status, active, list);
}

}  // namespace

int trid_cluster_for(int n) {
  for (int i = 0; i < kTridClasses; ++i)
    if (n <= trid_class_max(i)) return kTridClusterSizes[i];
  return 0;
}

size_t trid_smem_bytes(int n, int C) { return TridSmem(n, C).bytes(); }

cudaError_t trid_raise_limits() {
  int dev = 0, optin = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  const void* ks[] = {(const void*)k_trid_smem<1>, (const void*)k_trid_smem<2>, (const void*)k_trid_smem<3>,
                      (const void*)k_trid_smem<4>, (const void*)k_trid_smem<6>, (const void*)k_trid_smem<8>};
  for (const void* k : ks) {
    cudaFuncAttributes a;
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, k);
    if (e == cudaSuccess)
      e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)a.sharedSizeBytes);
  }
  return e;
}

cudaError_t launch_trid(const DevBatch& B, double* A, double* Sb, const int* status, const int* active,
                        const int* list, int cnt, int C, int nmax, cudaStream_t st) {
  if (cnt <= 0) return cudaSuccess;
  const size_t smem = trid_smem_bytes(nmax, C);
  switch (C) {
    case 1: return launch_c<1>(B, A, Sb, status, active, list, cnt, smem, st);
    case 2: return launch_c<2>(B, A, Sb, status, active, list, cnt, smem, st);
    case 3: return launch_c<3>(B, A, Sb, status, active, list, cnt, smem, st);
    case 4: return launch_c<4>(B, A, Sb, status, active, list, cnt, smem, st);
    case 6: return launch_c<6>(B, A, Sb, status, active, list, cnt, smem, st);
    case 8: return launch_c<8>(B, A, Sb, status, active, list, cnt, smem, st);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace tb
