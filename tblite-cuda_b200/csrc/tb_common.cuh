// Shared device-side types of the tblite-b200 engine.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace tb {

constexpr int kMaxL = 2;        // s, p, d
constexpr int kMaxPrim = 12;    // maxg (reference src/limits.h:18)
constexpr int kMaxShPerAtom = 3;
constexpr int kD4MaxRef = 4;    // D4 reference systems per element (parameter file)

// One shell type of one species (cgto_type, src/basis/type.h:18-23, plus the
// per-shell Hamiltonian parameters of tb_hamiltonian, src/h0.h:27-40).
struct ShellParam {
  int ang, nprim, species, local;
  double alpha[kMaxPrim];
  double coeff[kMaxPrim];
  double selfenergy, kcn, shpoly, refocc, hubbard, hubbard_deriv, slater;
};

struct SpeciesParam {
  int z, nsh, sh0;  // sh0: index of the first ShellParam of this species
  double rad, rcov, en, rep_alpha, rep_zeff, mp_rad, mp_vcn, dkernel, qkernel;
  // D4 dispersion: r4/r2 factor, reference systems and their coordination numbers
  double d4_r4r2;
  int d4_nref;
  double d4_cn[kD4MaxRef];
};

// Calculator parameters as seen by kernels (passed by value).
struct DevParams {
  const SpeciesParam* sp;
  const ShellParam* sh;
  const double* hscale;  // [nshtype][nshtype], hscale(jsh,ish,jzp,izp) by shell type
  int nsp, nshtype;
  double gexp, kdmp3, kdmp5, mp_shift, mp_kexp, mp_rmax;
  double rep_kexp, rep_kexp_light, rep_rexp, cn_cutoff, rep_cutoff;
  double intcut, cutoff;  // integral screening (25) and neighbour-list cutoff
  // D4 dispersion (d4 = 0: the parameter file has no D4 block): reference C6 of
  // species pair (a, b), references (i, j) at ((a nsp + b) kD4MaxRef + i) kD4MaxRef + j,
  // and the model's constants (tb_disp.cu)
  int d4;
  const double* d4_c6ref;
  double d4_s6, d4_s8, d4_a1, d4_a2, d4_s9, d4_alp, d4_wf, d4_k0, d4_k1, d4_k4, d4_k5, d4_k6;
  double d4_cn_cut, d4_atm_cut, d4_pair_cut;
};

// Per-batch layout: structures packed back to back.  Offsets are [nmol+1].
struct DevBatch {
  int nmol, nat_tot, nsh_tot, nao_tot;
  const int* aoff;       // atom offset
  const int* soff;       // shell offset
  const int* ooff;       // AO offset
  const long long* moff; // N*N matrix offset
  const long long* poff; // neighbour pair capacity offset (nat*(nat-1)/2)
  const int* mixoff;     // Broyden vector offset (nsh + 9 nat)
  const double* xyz;     // [nat_tot][3]
  const int* id;         // [nat_tot] species
  const int* at_mol;     // [nat_tot] owning structure
  const int* sh_type;    // [nsh_tot] global shell type (ShellParam index)
  const int* sh_at;      // [nsh_tot] local atom index
  const int* sh_iao;     // [nsh_tot] local AO offset
  const int* at_ish;     // [nat_tot] local shell offset of the atom
  const int* ao_at;      // [nao_tot] local atom index
  const int* ao_sh;      // [nao_tot] local shell index
  const int* order;      // [nmol] structures by decreasing N (one-CTA-per-structure kernels), may be null
  const long long* s2off;  // shell-pair table offset (nsh^2 per structure), may be null
  const long long* a2off;  // atom-pair table offset (nat^2 per structure), may be null
  int lib_above;         // 0: every structure on the in-house kernels; else structures with N > lib_above
                         // (all of them when -1) are factorised and diagonalised by the library path
  int jacobi_max;        // structures of N <= jacobi_max use the one-warp Jacobi eigensolver (0: none)
  int trid_min, trid_max;  // FP64 structures of trid_min <= N <= trid_max arrive at k_syev
                           // tridiagonalised by k_trid_smem (d | e | tau in their scratch slice;
                           // trid_max 0: none)
};

// True when structure size n is handled by the library (cuSOLVER) path.
__host__ __device__ inline bool on_library(const DevBatch& B, int n) { return B.lib_above != 0 && n > B.lib_above; }

__host__ __device__ inline int msao(int l) { return 2 * l + 1; }
__host__ __device__ inline int mlao(int l) { return (l + 1) * (l + 2) / 2; }
__host__ __device__ inline int lmap(int l) { return l == 0 ? 0 : (l == 1 ? 1 : 4); }

// ---- checked build (-DTB_BOUNDS_CHECK: `make check`, lib/libtblite_b200_check.so)
// Index guards at the global-memory accesses of the per-structure kernels: an
// access outside its structure's own slice (matrix, AO, shell, atom-pair or
// mixer slice) is skipped and recorded -- the number of violations and the
// first one's guard site, index and bounds -- in the translation unit's
// device record, which the host reads back.  No trap, no assert.  In the
// normal build a guard is the constant true.
struct OobRecord {
  unsigned long long count;
  int site, pad;
  long long index, lo, hi;
};
#ifdef TB_BOUNDS_CHECK
static __device__ OobRecord g_oob;
__device__ inline bool tb_guard(int site, long long i, long long lo, long long hi) {
  if (i >= lo && i < hi) return true;
  if (atomicAdd(&g_oob.count, 1ULL) == 0ULL) {
    g_oob.site = site;
    g_oob.index = i;
    g_oob.lo = lo;
    g_oob.hi = hi;
  }
  return false;
}
#define TB_GUARD(site, i, lo, hi) tb::tb_guard((site), (long long)(i), (long long)(lo), (long long)(hi))
#define TB_OOB_EXPORT(fn)                                                               \
  cudaError_t fn(OobRecord* r, bool reset) {                                           \
    cudaError_t e = cudaMemcpyFromSymbol(r, g_oob, sizeof(OobRecord));                 \
    if (e == cudaSuccess && reset) {                                                   \
      OobRecord z{};                                                                   \
      e = cudaMemcpyToSymbol(g_oob, &z, sizeof(OobRecord));                            \
    }                                                                                  \
    return e;                                                                          \
  }
#else
#define TB_GUARD(site, i, lo, hi) true
#define TB_OOB_EXPORT(fn)                         \
  cudaError_t fn(OobRecord* r, bool) {           \
    *r = OobRecord{};                            \
    return cudaSuccess;                          \
  }
#endif

// Status bits per structure (device), mapped to tb_status on the host.
enum DevStatus : int {
  kStOk = 0, kStBadInput = 1, kStNotSpd = 2, kStScfNotConverged = 3,
  kStFermiNotConverged = 4, kStEigenFailed = 5
};

template <typename T>
__device__ inline T warp_sum(T v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum in a fixed order (deterministic); all threads get the result.
// `red` must hold blockDim.x/32 values.
template <typename T>
__device__ inline T block_sum(T v, T* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) red[wid] = v;
  __syncthreads();
  T t = T(0);
  for (int w = 0; w < nw; ++w) t += red[w];
  return t;
}

}  // namespace tb
