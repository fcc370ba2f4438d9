// Kernel declarations and per-structure SCF state of the tblite-b200 engine.
#pragma once

#include <string>
#include <vector>

#include "tb_common.cuh"

namespace tb {

constexpr int kEigThreads = 256;
constexpr int kRing = 8;  // QL sweeps buffered between the k_syev producer and consumers
// k_syev's divide and conquer: structures of kDcMin+ rows (more than two leaves of
// 24), merge products in 64 x 64 tiles with reduction slabs of kDcK (Wt 64 x kDcK,
// Bt kDcK x kDcBs, rows padded by 4 against bank conflicts)
constexpr int kDcMin = 64;
constexpr int kDcK = 8;
constexpr int kDcBs = 64 + 4;
constexpr int kDcTileElems = 64 * kDcK + kDcK * kDcBs;
// workspace of one merge of m entries, in units of T (the ints after the T arrays)
template <typename T>
__host__ __device__ constexpr int dc_ws_elems(int m) {
  return 8 * m + kDcTileElems + (7 * m * (int)sizeof(int) + (int)sizeof(T) - 1) / (int)sizeof(T);
}
// shared memory of k_syev: d, e, tau, v, vn, p, w (7n) + the rotation ring (2 n kRing);
// in FP64 at least d, e and the divide-and-conquer workspace (from tau on) for
// kDcMin+ rows, so that the solver chosen for a structure depends on its size only
inline size_t syev_smem_bytes(int n, size_t elem = sizeof(double)) {
  size_t v = (7 + 2 * (size_t)kRing) * (size_t)n;
  if (elem == sizeof(double) && n >= kDcMin) {
    const size_t dc = 2 * (size_t)n + (size_t)dc_ws_elems<double>(n);
    if (dc > v) v = dc;
  }
  return v * elem;
}
constexpr int kSyevMaxN = 1216;
// k_trid_smem (tb_trid.cu): the tridiagonalisation of FP64 structures of
// kTridMin..kTridClassMax[last] AOs held in the shared memory of a thread block
// cluster of kTridClusterSizes[c] CTAs (class c: up to kTridClassMax[c] AOs,
// the largest order whose tiles fit 227 KiB per CTA); k_syev then starts from
// its output (DevBatch::trid_max)
constexpr int kTridTile = 16;
constexpr int kTridThreads = 512;
constexpr int kTridMaxCluster = 8;
constexpr int kTridClasses = 6;
constexpr int kTridMin = 64;
constexpr int kTridClusterSizes[kTridClasses] = {1, 2, 3, 4, 6, 8};
constexpr int kTridClassMax[kTridClasses] = {208, 288, 352, 400, 480, 560};
constexpr int kTridMaxN = 560;  // kTridClassMax[kTridClasses - 1]
inline int trid_class_max(int c) { return kTridClassMax[c]; }
// class of a structure of n AOs (-1: not handled)
inline int trid_class_of(int n) {
  if (n < kTridMin) return -1;
  for (int c = 0; c < kTridClasses; ++c)
    if (n <= kTridClassMax[c]) return c;
  return -1;
}
int trid_cluster_for(int n);
size_t trid_smem_bytes(int n, int C);
cudaError_t trid_raise_limits();
// structures list[0..cnt) (all of one class, cluster size C, at most nmax AOs):
// reflectors into A, d | e | tau into the first 3n doubles of Sb's slice
cudaError_t launch_trid(const DevBatch& B, double* A, double* Sb, const int* status, const int* active,
                        const int* list, int cnt, int C, int nmax, cudaStream_t st);
constexpr int kGemmThreads = 128;  // block size of k_gemm

// cuSOLVER dense path for structures above the in-house size bound
// (tb_large.cu); one instance per batch, used from one host thread at a time.
struct LargeSolver {
  void* handle = nullptr;  // cusolverDnHandle_t
  void* params = nullptr;  // cusolverDnParams_t
  std::vector<char> host;  // host workspace
  ~LargeSolver();
  std::string init();
  // device workspace in bytes for potrf, trtri and syevd of order n
  std::string workspace(int n, size_t* dev_bytes);
  // X = L^-T of S (row-major, both n x n); info[0..1], status: device ints
  std::string factor(cudaStream_t st, const double* S, double* X, int n, void* dwork, size_t dbytes, int* info,
                     int* status);
  // eigenpairs of A: eigenvector j in row j of Z, w ascending, perm = identity
  std::string syev(cudaStream_t st, const double* A, double* Z, double* w, int* perm, int n, void* dwork,
                   size_t dbytes, int* info, int* status);
  // the same in FP32 (mixed-precision form); wtmp: n floats of scratch, w written as double
  std::string syev32(cudaStream_t st, const float* A, float* Z, float* wtmp, double* w, int* perm, int n,
                     void* dwork, size_t dbytes, int* info, int* status);
};

// Per-structure scalars of the SCF (device arrays of length nmol; nel is 2*nmol).
struct MolState {
  double* e_rep;
  double* nel;
  int* iscf;
  int* mix_iter;
  double* eelec;
  int* active;
  int* status;
  double* e_ts;
  double* e_band;
  double* e_es2;
  double* e_aes2;
  double* e_es3;
  double* scf_error;
  int* fermi_warn;
  double* dipole;   // 3*nmol
  double* e_fermi;  // optional (may be null): Fermi level of spin channel 0
  int* n_active;    // single counter
  int* phase;       // mixed-precision form only (else null): 0 mixed phase, 1 FP64 phase
  int* n64;         // mixed-precision form only: FP64 iterations done
};

// Matrix outputs of the integral kernels (D, Q planar [3|6][N][N] per structure).
struct MatOut {
  double* S;
  double* H0;
  double* D;
  double* Q;
};

// setup
__global__ void k_atoms(DevParams P, DevBatch B, double* cn, double* mrad, double* erep, double* se);
__global__ void k_adj_count(DevBatch B, double cutoff, int* cnt);
__global__ void k_adj_scan(DevBatch B, const int* cnt, long long* inl, int* npair);
__global__ void k_adj_fill(DevBatch B, double cutoff, const long long* inl, int* pair_i, int* pair_j);
// Work space of the integral setup: the shell-pair items sorted by (li, lj)
// class (list, `items` entries), the item of each (pair slot, shell pair)
// (idx, pair_cap * maxsp), the computed blocks (rec, `rec_len` doubles:
// per item s[SI SJ], hij, d[3 SI SJ], q[6 SI SJ]), the pair slot of each
// atom pair i > j (tab, at a2off, nat^2 per structure) and the class counts
// and cursors (cls, 32 ints).
struct SpLists {
  int2* list;
  int* idx;
  double* rec;
  int* tab;
  int* cls;
  long long items, rec_len, tab_len;
};
__host__ __device__ constexpr int sp_record(int li, int lj) { return 10 * (2 * li + 1) * (2 * lj + 1) + 1; }
cudaError_t launch_integrals(const DevParams& P, const DevBatch& B, const int* npair, const int* pair_i,
                             const int* pair_j, const double* se, const MatOut& out, int maxsp, long long pair_cap,
                             int lmask, const SpLists& W, cudaStream_t st, int64_t* launches);

// linear algebra
__global__ void k_cholesky(DevBatch B, const double* S, double* W, int* status, const int* active);
__global__ void k_trinv(DevBatch B, const double* W, double* X, const int* status);
// k_gemm shapes (bit mask): zeros of a triangular factor and symmetric results
constexpr int kGemmKUpToJ = 1, kGemmKUpToI = 2, kGemmKFromI = 4, kGemmSym = 8;
__global__ void k_gemm(DevBatch B, const int4* tiles, int ntiles, const double* Ab, int ta, const double* Bb, int tb_,
                       const int* perm, const double* ks, const int* kdim, double* Cb, double alpha, double beta,
                       const int* active, int shape = 0);
// the same GEMM on 32 x 32 tiles (tile list in units of 32; the same bits as k_gemm)
__global__ void k_gemm32(DevBatch B, const int4* tiles, int ntiles, const double* Ab, int ta, const double* Bb,
                         int tb_, const int* perm, const double* ks, const int* kdim, double* Cb, double alpha,
                         double beta, const int* active, int shape = 0);
// Sb: optional n x n scratch per structure (same offsets as Ab); with it,
// structures of at least kDcMin (64) AOs take divide and conquer instead of QL
__global__ void k_syev(DevBatch B, double* Ab, double* Zb, double* Sb, double* wout, int* perm, int* status,
                       const int* active);
// the same eigensolver in FP32 (A and Z float, eigenvalues written as double)
__global__ void k_syev_f32(DevBatch B, float* Ab, float* Zb, double* wout, int* perm, int* status, const int* active);
// small-structure variant: one warp per structure of N <= kJacobiMaxN (cyclic Jacobi
// in shared memory), structures list[0..nlist), kJacobiWarps structures per CTA;
// same outputs as k_syev (w ascending, eigenvector j = row perm[j] of Z)
constexpr int kJacobiMaxN = 32;
constexpr int kJacobiWarps = 4;
constexpr int kJacobiPitch = kJacobiMaxN + 1;
inline size_t jacobi_smem_bytes() { return (size_t)kJacobiWarps * 2 * kJacobiMaxN * kJacobiPitch * sizeof(double); }
__global__ void k_syev_jacobi(DevBatch B, double* Ab, double* Zb, double* wout, int* perm, int* status,
                              const int* active, const int* list, int nlist);

// mixed-precision form (tb_mixed.cu)
__global__ void k_phase_masks(int nmol, const int* active, const int* phase, int* lo, int* hi);
// the same contractions as TF32x3 (split precision) tcgen05 GEMMs over 128 x 128 tiles (tb_tc.cu);
// kTcThreads threads, dynamic shared memory gemm_tc_smem_bytes(), status marks a structure whose waits ran out
constexpr int kTcTile = 128;
constexpr int kTcThreads = 256;
__global__ void k_gemm_tc(DevBatch B, const int4* tiles, int ntiles, const double* Ab, int ta, const double* Bb,
                          int tb_, const int* perm, const double* ks, const int* kdim, double* Cb, double alpha,
                          double beta, const int* active, int* status);
size_t gemm_tc_smem_bytes();
__global__ void k_to_f32(DevBatch B, const int4* tiles, int ntiles, const double* F, float* Af, const int* mask);
__global__ void k_gather_vectors(DevBatch B, const int4* tiles, int ntiles, const float* Zf, const int* perm,
                                 double* V, const int* mask);
// refinement step (Rayleigh-Ritz in clusters + Ogita-Aishima coefficients)
constexpr int kClusterMax = 64;
inline size_t oa_smem_bytes(int nmax) {
  return (3 * (size_t)kClusterMax * kClusterMax + 2 * kClusterMax) * sizeof(double) +
         2 * ((size_t)nmax + 1) * sizeof(int);
}
__global__ void k_oa_step(DevBatch B, double* G, double* Sm, double* V, double* w, const int* mask,
                          const int* rr_mask);

// records of the checked build's index guards, one per translation unit
// (all zero in the normal build); reset clears them after the read
cudaError_t oob_setup(OobRecord* r, bool reset);
cudaError_t oob_scf(OobRecord* r, bool reset);
cudaError_t oob_linalg(OobRecord* r, bool reset);

// D4 dispersion (tb_disp.cu; only when DevParams::d4): per atom cn, W and dW
// (kD4MaxRef each), energy share e_at, dE/dCN and gradient g [3 nat]; per
// structure e_disp.  Five launches on st.
cudaError_t launch_dispersion(const DevParams& P, const DevBatch& B, int nmol, double* cn, double* W, double* dW,
                              double* e_at, double* dEdcn, double* g, double* e_disp, cudaStream_t st);
__global__ void k_d4_add_grad(DevBatch B, const int* flag, const double* gd, double* grad);

// nuclear gradient (read-out after the SCF, structures with flag[m] set)
cudaError_t launch_grad_pairs(const DevParams& P, const DevBatch& B, const int* npair, const int* pair_i,
                              const int* pair_j, const double* se, const double* Pm, const double* Wm,
                              const double* vsh, const double* vat, const double* vdp, const double* vqp,
                              const int* flag, int maxsp, long long items, int lmask, double* item, double* ese_tab,
                              cudaStream_t st);
__global__ void k_grad_prep(DevBatch B, const int* flag, const double* focc, const double* w, const double* qsh,
                            const double* dpat, const double* qpat, double* fe, double* qv);
__global__ void k_grad_pair_reduce(DevBatch B, const int* npair, const int* pair_i, const int* pair_j,
                                   const int* flag, int maxsp, long long pair_cap, const double* item, double* G);
__global__ void k_grad_cn(DevParams P, DevBatch B, const int* flag, const double* Pm, const double* ese_tab,
                          const double* cn, const double* mrad, const double* qat, const double* dpat,
                          const double* qpat, double* dEdcn);
__global__ void k_grad_atoms(DevParams P, DevBatch B, const int* flag, const double* G, const double* dEdcn,
                             const double* mrad, const double* qsh, const double* qat, const double* dpat,
                             const double* qpat, double* grad);
__global__ void k_grad_sigma(DevBatch B, const int* flag, const double* grad, double* sigma);

// SCF
__global__ void k_scf_init(DevParams P, DevBatch B, const double* charge, const int* uhf, const double* erep,
                           double* n0sh, double* q_in, MolState S);
// end of one iteration of the SCF loop graph: counts it and sets the loop condition
__global__ void k_loop_control(cudaGraphConditionalHandle h, const int* n_active, int* it, int max_iter);
// SCF state of structure map[k] of batch Bo moved to structure k of batch Bn
// (serving: compaction of a micro-batch to its unfinished structures)
struct ScfState {
  double *q_in, *dq, *dqlast, *qlast, *df, *u, *amat, *omega;
  MolState S;
};
__global__ void k_compact_state(DevBatch Bo, DevBatch Bn, const int* map, ScfState so, ScfState sn, int memory);
// caller's starting moments (wavefunction guess) into q_in for flagged structures
__global__ void k_apply_guess(DevBatch B, const double* guess, const int* flag, double* q_in);
// pair tables of the fixed geometry (gtab: gamma per shell pair, atab: 1/r, f3, f5 per atom pair)
__global__ void k_pair_tables(DevParams P, DevBatch B, const double* mrad, double* gtab, double* atab);
// gtab/atab may be null: the pair terms are then recomputed
// shells / atoms per CTA of k_potential (one warp each: CTAs of 32 x kPotTargets threads)
constexpr int kPotTargets = 8;
__global__ void k_potential(DevParams P, DevBatch B, const double* q_in, const double* mrad, double* vsh, double* vat,
                            double* vdp, double* vqp, const int* active, const double* gtab, const double* atab);
// dynamic shared memory of k_fock (the nine staged transposed tiles)
size_t fock_smem_bytes();
__global__ void k_fock(DevBatch B, const int4* tiles, int ntiles, const double* S, const double* H0, const double* D,
                       const double* Q, const double* vsh, const double* vat, const double* vdp, const double* vqp,
                       double* F, const int* active);
__global__ void k_fermi(DevBatch B, const double* w, double kt, double* focc, int* kdim, MolState S);
// nspin = 2 read-out: per-channel occupations f[0] alpha, f[1] beta, f[2] alpha - beta (f: 3 x nao_tot)
__global__ void k_spin_occupations(DevBatch B, const double* w, double kt, const double* nel, const int* flag,
                                   double* f);
// moments of the magnetization density from its Mulliken column sums (colred)
__global__ void k_spin_moments(DevParams P, DevBatch B, const double* colred, const int* flag, double* qsh,
                               double* qat, double* dpat, double* qpat);
__global__ void k_mulliken_cols(DevBatch B, const int2* chunks, int nchunks, const double* P, const double* S,
                                const double* H0, const double* D, const double* Q, double* colred,
                                const int* active);
__global__ void k_finalize(DevParams P, DevBatch B, const double* colred, const double* n0sh, const double* mrad,
                           const double* q_in, double* dq, double* qsh_out, double* qat_out, double* dpat_out,
                           double* qpat_out, double econv, double pconv, int max_iter, MolState S,
                           double econv_lo, double pconv_lo, const double* gtab, const double* atab);
__global__ void k_mix_next(DevBatch B, double* q_in, const double* dq, double* dqlast, double* qlast, double* df,
                           double* u, double* amat, double* omega, int memory, double damp, MolState S);

}  // namespace tb
