/*
 * tblite-b200: B200-native (sm_100a) GFN2-xTB singlepoint engine -- C ABI.
 *
 * The reference (tornikeo/tblite-cuda) has no host API at all: its only entry
 * is the device function
 *   __device__ void xtb_singlepoint(const structure_type &mol,
 *       const xtb_calculator &calc, wavefunction_type &wfn, float accuracy,
 *       float energy, float (&gradient)[MAX_NAT][3], float (&sigma)[3][3],
 *       int verbosity)                                   (src/xtb.cu:188-197)
 * launched one thread per molecule from a test kernel (src/xtb.cu:436-481).
 * This header is the drop-in boundary for that path: plain C types, caller
 * owned host buffers, a status per call and per structure, no exit/trap.
 * Each declaration names the reference interface it replaces.
 *
 * Conventions: coordinates in Bohr, energies in Hartree.  Species indices are
 * 0-based positions in the parameter file's element list (the reference's
 * mol%id).  Shell order within an atom follows the parameter file; AOs are
 * spherical (s; p as y,z,x; d as tblite orders them).  Matrices are row-major.
 * D[k][mu][nu] and Q[c][mu][nu] are planar with the moment operator on the
 * atom of the column index nu (tblite's "centered on last index",
 * src/integral/type.h:13-16); quadrupoles are traceless (xx,xy,yy,xz,yz,zz).
 *
 * Thread safety: a calculator may be shared by threads for read-only calls;
 * tb_singlepoint_batch serialises on the calculator's workspace.  All device
 * work is ordered on the caller's stream (NULL = default stream).
 */
#ifndef TBLITE_B200_H
#define TBLITE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum tb_status {
  TB_OK = 0,
  TB_BAD_INPUT = 1,            /* invalid sizes, species or pointers            */
  TB_NOT_SPD = 2,              /* overlap matrix not positive definite          */
  TB_SCF_NOT_CONVERGED = 3,    /* max_iter reached                              */
  TB_FERMI_NOT_CONVERGED = 4,  /* Fermi level solve hit its iteration cap       */
  TB_EIGEN_FAILED = 5,         /* tridiagonal solve failed: QL (or a divide-and-
                                  conquer leaf) hit its sweep cap, or the matrix
                                  was not finite                                */
  TB_CAPACITY_EXCEEDED = 6,    /* request larger than a stated maximum          */
  TB_CUDA_ERROR = 7,           /* CUDA runtime error (see tb_last_error)        */
  TB_PARAM_ERROR = 8           /* parameter file could not be read              */
} tb_status;

/* structure_type (src/structure.h:5-15): nat atoms, 0-based species id[nat],
 * Cartesian xyz[nat][3] in Bohr, total charge and unpaired electrons. */
typedef struct tb_structure {
  int32_t nat;
  int32_t uhf;
  double charge;
  const int32_t* id;
  const double* xyz;
} tb_structure;

/* Calculator options: accuracy/verbosity arguments of xtb_singlepoint
 * (src/xtb.cu:192,197) and xtb_calculator%max_iter, %mixer_damping
 * (src/xtb.h:115-116).  econv = 1e-6*accuracy, pconv = 2e-5*accuracy. */
typedef struct tb_options {
  double accuracy;        /* default 1.0                                       */
  double kt;              /* electronic temperature in Eh, default 300 K       */
  int32_t max_iter;       /* SCF iterations = Broyden memory, default 32       */
  double mixer_damping;   /* default 0.4                                       */
  int32_t verbosity;      /* 0 silent                                          */
  int32_t use_graphs;     /* 1: replay each SCF iteration as a CUDA graph      */
  int32_t solver;         /* 0 auto: in-house batched eigensolver up to 1216 AOs,
                             cuSOLVER Xsyevd above; 1 in-house only (larger
                             structures: TB_CAPACITY_EXCEEDED); 2 cuSOLVER only */
  int32_t profile;        /* 1: time every kernel class with CUDA events        */
  int32_t precision;      /* 0 plain FP64; 1 mixed: FP32 eigensolve refined in
                             FP64 and FP32-product contractions until the SCF
                             nearly converges, then at least two FP64
                             iterations before the final convergence test     */
} tb_options;

/* Per-structure results: the energy/wavefunction outputs of xtb_singlepoint.
 * Array pointers are caller-owned and may be NULL (not written). */
typedef struct tb_result {
  double energy;          /* total energy = e_elec + e_rep + e_disp            */
  double e_rep;           /* classical repulsion                               */
  double e_elec;          /* electronic: band + (-TS) + ES2 + AES2 + ES3        */
  double e_band, e_ts, e_es2, e_aes2, e_es3;
  double dipole[3];       /* sum_A q_A R_A + mu_A (a.u.)                       */
  double scf_error;       /* last RMS charge/multipole change                  */
  int32_t iterations;
  int32_t status;         /* tb_status of this structure                       */
  int32_t nsh, nao;
  double* qat;            /* [nat]    atomic partial charges                   */
  double* qsh;            /* [nsh]    shell partial charges                    */
  double* dpat;           /* [nat][3] atomic dipoles                           */
  double* qpat;           /* [nat][6] atomic quadrupoles                       */
  /* the gradient and sigma arguments of xtb_singlepoint (src/xtb.cu:195-196):
   * gradient [nat][3] dE/dR in Eh/Bohr, computed when not NULL; sigma the
   * virial sum_A gradient_A R_A^T (row-major 3x3), written with gradient */
  double* gradient;
  double sigma[9];
  double e_disp;          /* D4 dispersion (0 without a D4 parameter block)     */
} tb_result;

/* wavefunction_type (src/wavefunction/type.h:81-99) of one structure, as the
 * in/out argument `wfn` of xtb_singlepoint (src/xtb.cu:188-197).  The arrays
 * are caller-owned host buffers sized from tb_basis_size; a NULL array is
 * neither read nor written.
 *   in:  guess = 1 starts the SCF from qsh, dpat and qpat as given (for
 *        example the result of an earlier singlepoint of the same or a nearby
 *        geometry, the reference's wfn carried from call to call); guess = 0
 *        uses the default start (the charge spread over the shells by their
 *        reference occupations, no multipoles).  With nspin = 2 channel 0 of
 *        the moments is read.
 *        nspin = 1 (or 0): one density for both spin channels, uhf only
 *        splitting the electrons (get_alpha_beta_occupation,
 *        src/wavefunction/type.cu:3-14).  nspin = 2: tblite's open-shell
 *        representation, every array with a leading channel index (the
 *        reference's [MAX_NSPIN] dimension): emo and coeff per channel (the
 *        same in both: GFN2 has no spin-dependent potential), focc and
 *        density per channel (alpha, beta: each channel's own Fermi
 *        filling), and qat, qsh, dpat, qpat as (total, up - down)
 *        (updown_to_magnet, src/wavefunction/spin.h:4-16).  The SCF and the
 *        energy are the same for both.
 *   out: everything else, from the last SCF iteration of the structure. */
typedef struct tb_wavefunction {
  int32_t guess;          /* in                                                */
  int32_t nspin;          /* in/out: 1 or 2 (see above)                        */
  int32_t nat, nsh, nao;
  int32_t homo[2];        /* highest orbital of the aufbau filling per channel
                             (1-based count, floor(nel[s]))                    */
  double kt;              /* electronic temperature (Eh)                       */
  double nocc;            /* electrons                                         */
  double nuhf;            /* unpaired electrons                                */
  double nel[2];          /* alpha, beta electrons                             */
  double* n0at;           /* [nat]   reference occupation per atom             */
  double* n0sh;           /* [nsh]   reference occupation per shell            */
  double* emo;            /* [nao]   orbital energies, ascending               */
  double* focc;           /* [nao]   occupations, alpha + beta                 */
  double* density;        /* [nao][nao] P = C diag(focc) C^T                   */
  double* coeff;          /* [nao][nao] coeff[mu * nao + i]: AO mu of orbital i */
  double* qat;            /* [nat]   atomic charges                            */
  double* qsh;            /* [nsh]   shell charges        (in with guess = 1)  */
  double* dpat;           /* [nat][3] atomic dipoles      (in with guess = 1)  */
  double* qpat;           /* [nat][6] atomic quadrupoles  (in with guess = 1)  */
} tb_wavefunction;

typedef struct tb_calculator tb_calculator;

/* xtb_calculator construction (src/xtb.h:105-126; the reference never builds
 * one: new_hamiltonian is declared at src/h0.h:80-86 but not defined).  Reads a
 * tblite-b200 parameter file (.tbp). */
tb_status tb_calculator_create(const char* param_file, tb_calculator** out);
/* Destroy batches and servers made from the calculator before it: they share
 * its workspace and pinned host buffers. */
void tb_calculator_destroy(tb_calculator* calc);
int32_t tb_calculator_nspecies(const tb_calculator* calc);
void tb_default_options(tb_options* opt);
/* Text of the last error on this thread. */
const char* tb_last_error(void);

/* Autotuner (no counterpart in the reference, whose only eigensolver is a
 * one-thread Jacobi, src/lapack/sygvd.cu:74-133).  The per-size eigensolver
 * variant is measured once per calculator, on first need: structures of at
 * most 32 AOs use a one-warp Jacobi solver up to the largest size at which
 * it is measured faster than the one-CTA solver (Householder + implicit QL
 * below 64 AOs, + divide and conquer from 64); above 1216 AOs, and above a
 * size chosen per batch from measured cost models, cuSOLVER Xsyevd (see
 * tb_options.solver).  The choice depends on the size only, so a structure
 * gives the same bits alone and in any batch.
 * tb_calculator_set_small_solver: jacobi_max -1 (default) measured choice,
 * 0 never, 1..32 fixed bound.  tb_calculator_tuning writes the measurements
 * and choices as JSON text into buf (NUL-terminated, at most len bytes) and
 * returns the full length. */
tb_status tb_calculator_set_small_solver(tb_calculator* calc, int32_t jacobi_max);

/* Householder tridiagonalisation of the FP64 eigensolver (the dsytrd step of
 * sygvd_solver::solve, src/lapack/sygvd.cu:223-313) held in the shared memory
 * of a thread block cluster: structures of 64..560 AOs, one cluster of 1, 2,
 * 3, 4, 6 or 8 CTAs by size (the choice depends on the size only).  It cuts
 * the latency of a structure's reduction (a 384-AO one: 4 SMs instead of a
 * third of one), but spends more SM time per structure, so it pays where
 * latency bounds the call -- single structures, small batches, the request
 * loop at low load -- and not for large batches.  min_n: structures of at
 * least min_n AOs (and 64..560) take it; 0 (default): the one-CTA kernel
 * reduces every size.  Applies to batches built afterwards.  tb_sygvd_batch
 * always uses it from 64 AOs. */
tb_status tb_calculator_set_smem_tridiag(tb_calculator* calc, int32_t min_n);

/* FP64 GEMM tile shape (the batched matrix products of every SCF iteration:
 * X^T F X, C = X V, P = C diag(f) C^T; the reference's get_density_matrix,
 * src/wavefunction/type.cu:37, is a loop nest per structure with no tiling
 * choice).  Each structure's products run on 64 x 64 or on 32 x 32 tiles.
 * The calculator measures both per size (16..384 AOs in steps of 16) on the
 * first batch that holds a structure of at most 384 AOs; larger structures
 * always take 64 x 64.  A batch takes the faster shape per structure, but is
 * split over both kernels only when the modelled saving is at least 5% of the
 * better single shape (a second launch per product has its own ramp and
 * tail); tb_calculator_tuning reports the table.  Both shapes accumulate
 * every element in the same order, so the choice never changes a result's
 * bits.  max_n32: -1 (default) measured choice, 0 always 64 x 64, N > 0
 * 32 x 32 up to N AOs.  Applies to batches built afterwards. */
tb_status tb_calculator_set_gemm_tiles(tb_calculator* calc, int32_t max_n32);

/* Checked build (the library built with -DTB_BOUNDS_CHECK, `make check`:
 * lib/libtblite_b200_check.so; no counterpart in the reference, whose only
 * checks are device asserts): index guards at the global-memory accesses of
 * the per-structure kernels skip and record any access outside its
 * structure's own slice.  tb_bounds_check_build returns 1 in that build, 0
 * otherwise; tb_bounds_violations returns the number of guarded accesses
 * skipped since the last reset and the first one's guard site, index and
 * bounds (all 0 in the normal build), and clears the records when reset is
 * set.  Needs a CUDA device. */
int32_t tb_bounds_check_build(void);
tb_status tb_bounds_violations(int64_t* count, int32_t* site, int64_t* index, int64_t* lo, int64_t* hi,
                               int32_t reset);
int32_t tb_calculator_tuning(const tb_calculator* calc, char* buf, int32_t len);

/* Structure input (the structure file I/O of the reference's host-side
 * plan beside periodic images, src/xtb.cu:342-346): an XYZ file (count line,
 * comment line, "symbol x y z" per atom in Angstrom; a symbol may also be an
 * atomic number) into nat, atomic numbers z[nat] and xyz[nat][3] in Bohr;
 * with more than cap atoms only *nat is set (TB_CAPACITY_EXCEEDED), so a
 * first call with cap = 0 sizes the buffers.  comment (optional) receives the
 * second line.  Host only: needs no CUDA device.
 * tb_calculator_species maps an atomic number to the species index of the
 * parameter file (tb_structure.id), -1 if it has none. */
tb_status tb_read_xyz(const char* path, int32_t cap, int32_t* nat, int32_t* z, double* xyz, char* comment,
                      int32_t comment_len);
int32_t tb_calculator_species(const tb_calculator* calc, int32_t z);

/* basis_type sizes (src/basis/type.h:56-73). */
tb_status tb_basis_size(const tb_calculator* calc, const tb_structure* mol, int32_t* nsh, int32_t* nao);

/* xtb_singlepoint (src/xtb.cu:188-434) for nmol structures at once, host
 * buffers in and out.  wfn_inout is NULL or nmol records (the reference's
 * wavefunction_type& wfn, in and out).  Returns TB_OK when every structure
 * succeeded, else the first failing structure's status; per-structure status
 * is in out[i].status. */
tb_status tb_singlepoint_batch(tb_calculator* calc, const tb_structure* mols, int32_t nmol,
                               const tb_options* opt, tb_wavefunction* wfn_inout, tb_result* out,
                               void* stream);

/* Device-resident batches (for serving and for timing without host copies):
 * create uploads geometry and sizes workspaces, run executes the full
 * singlepoint on the device, results copies them back. */
typedef struct tb_batch tb_batch;
tb_status tb_batch_create(tb_calculator* calc, const tb_structure* mols, int32_t nmol,
                          const tb_options* opt, tb_batch** out);
tb_status tb_batch_run(tb_batch* batch, void* stream);
tb_status tb_batch_results(tb_batch* batch, tb_result* out, void* stream);
/* Starting guesses for the next tb_batch_run from nmol wavefunction records
 * (records with guess = 0 keep the default start), and the wavefunctions of
 * the last run (the same records as tb_singlepoint_batch's wfn_inout). */
tb_status tb_batch_set_guess(tb_batch* batch, const tb_wavefunction* wfn);
/* Analytic nuclear gradient of the last run: grad [nat_tot][3] (the batch's
 * atoms in order), sigma [nmol][9]; either may be NULL. */
tb_status tb_batch_gradient(tb_batch* batch, double* grad, double* sigma, void* stream);
tb_status tb_batch_wavefunction(tb_batch* batch, tb_wavefunction* wfn, void* stream);
/* kernels launched by the last tb_batch_run (device work items, not host calls) */
int64_t tb_batch_launches(const tb_batch* batch);
/* Instrumentation (no counterpart in the reference, which only times its one
 * launch with cudaEvent, src/xtb.cu:488-506).
 * With tb_options.profile = 1: per kernel class of the last run, its name
 * (name[i*32], NUL-terminated), launches, total device time in ms (CUDA events
 * on the run's stream) and algorithmic work (flops or bytes, see units: 0 none,
 * 1 FP64 flops, 2 bytes moved).  Returns the number of classes (<= max). */
int32_t tb_batch_profile(const tb_batch* batch, int32_t max, char* names, int64_t* launches, double* ms,
                         double* work, int32_t* units);
void tb_batch_destroy(tb_batch* batch);

/* ---- serving: continuous batching of singlepoint requests ------------------
 * No counterpart in the reference (its driver runs one fixed batch,
 * src/xtb.cu:483-509).  Requests are queued by tb_server_submit.  Each
 * tb_server_step admits queued requests (first in, first out) as one new
 * resident micro-batch while the device workspace of all resident
 * micro-batches stays within hbm_budget_bytes (at most max_batch per
 * micro-batch) and advances every resident micro-batch without waiting for
 * any: each runs its SCF iterations on its own stream, so their work overlaps
 * on the device; one whose iteration has finished is collected (structures
 * that converged are retired) and given its next iteration.  Once at most half
 * of a micro-batch is unfinished, the rest moves to a smaller one (see
 * tb_server_compactions); a micro-batch's workspace returns to the pool when
 * its last structure finishes.  Call it in a loop.  tb_server_poll hands out finished results in completion
 * order.  Each result equals the one tb_singlepoint_batch gives for the same
 * structure alone (the kernels treat every structure independently).
 * Calls on one server must come from one host thread at a time. */
typedef struct tb_server tb_server;
tb_status tb_server_create(tb_calculator* calc, const tb_options* opt, int64_t hbm_budget_bytes,
                           int32_t max_batch, tb_server** out);
/* Copies the structure into the queue; *ticket identifies its result.
 * TB_CAPACITY_EXCEEDED if the structure alone needs more than the budget. */
tb_status tb_server_submit(tb_server* server, const tb_structure* mol, int64_t* ticket);
/* One scheduling step (see above); optional outputs: requests resident on the
 * device, requests still queued, workspace bytes resident. */
tb_status tb_server_step(tb_server* server, int32_t* n_resident, int32_t* n_queued, int64_t* bytes_resident);
/* Up to max finished results: tickets[i], results[i] (scalar fields; the array
 * pointers of results[i], when not NULL, receive that structure's qat / qsh /
 * dpat / qpat).  Returns the number written. */
int32_t tb_server_poll(tb_server* server, int32_t max, int64_t* tickets, tb_result* results);
/* Number of compactions so far: once at most half of a micro-batch (of 4 or
 * more structures) is still iterating, its unfinished structures continue in
 * a new, smaller micro-batch with their SCF state, and the old workspace
 * returns to the server's pool, where admission can use it at once. */
int64_t tb_server_compactions(const tb_server* server);
void tb_server_destroy(tb_server* server);

/* ---- stage entry points (host buffers; one structure each) ---------------- */

/* get_cutoff (src/basis/type.cu:66-79). */
double tb_get_cutoff(const tb_calculator* calc, double accuracy);

/* new_adjacency_list / generate (src/adjlist.cu:3-101): half list, jat < iat,
 * r2 >= eps and r2 <= cutoff^2.  inl[nat], nnl[nat], nlat[cap] (0-based atom
 * indices), npair out.  Bit-exact with the FP64 restatement. */
tb_status tb_adjacency_list(const tb_calculator* calc, const tb_structure* mol, double cutoff,
                            int32_t* inl, int32_t* nnl, int32_t* nlat, int32_t cap, int32_t* npair);

/* ncoord_get_cn (src/coulomb.cu:334-347), get_mrad (:374-408) and
 * get_selfenergy (src/h0.cu:125-199). cn[nat], mrad[nat], se[nsh]; any NULL. */
tb_status tb_atomic_properties(const tb_calculator* calc, const tb_structure* mol, double* cn,
                               double* mrad, double* selfenergy);

/* get_engrad energy part (src/xtb.cu:47-182): erep[nat]. */
tb_status tb_repulsion(const tb_calculator* calc, const tb_structure* mol, double* erep);

/* dispersion_get_engrad (src/xtb.cu:274-277, a TODO in the reference; tblite
 * calls dftd4 there): D4 dispersion of the geometry at the neutral reference
 * charges from the parameter file's D4 block -- edisp[nat] per-atom energies,
 * gradient[nat][3] and sigma[3][3] (either may be NULL); all zero when the
 * parameter file has no D4 block.  tb_singlepoint_batch adds the same term to
 * the energy (tb_result.e_disp) and to the gradient. */
tb_status tb_dispersion(const tb_calculator* calc, const tb_structure* mol, double* edisp, double* gradient,
                        double* sigma);

/* get_hamiltonian (src/h0.cu:292-502) incl. on-site blocks: S, H0 [nao][nao],
 * D [3][nao][nao], Q [6][nao][nao]. */
tb_status tb_get_hamiltonian(const tb_calculator* calc, const tb_structure* mol, double* S,
                             double* H0, double* D, double* Q);

/* tb_coulomb::get_potential (src/coulomb.cu:793-809): ES2 + AES2 + ES3
 * potential shifts for given shell charges and atomic multipoles. */
tb_status tb_coulomb_potential(const tb_calculator* calc, const tb_structure* mol, const double* qsh,
                               const double* dpat, const double* qpat, double* vsh, double* vat,
                               double* vdp, double* vqp);

/* add_pot_to_h1 (src/scf/potential.cu:224-272): F = H0 - potentials. */
tb_status tb_add_pot_to_h1(const tb_calculator* calc, const tb_structure* mol, const double* S,
                           const double* H0, const double* D, const double* Q, const double* vsh,
                           const double* vat, const double* vdp, const double* vqp, double* F);

/* sygvd_solver::solve (src/lapack/sygvd.cu:223-313): batched generalized
 * symmetric-definite eigenproblems H C = S C e, ascending e, S-orthonormal C.
 * Matrices packed back to back ([n_i][n_i] each), host buffers. */
tb_status tb_sygvd_batch(int32_t nmat, const int32_t* n, const double* H, const double* S,
                         double* w, double* C);

/* Allocation-free variant of tb_sygvd_batch for one problem, for callers that
 * cannot let a library allocate device memory (frameworks that own all GPU
 * memory through their own pool, latency-critical loops where cudaMalloc
 * would synchronise the device, processes with a fixed memory budget).  No
 * counterpart in the reference.  H, S (n x n, row-major), w (n) and C (n x n)
 * are DEVICE pointers owned by the caller; every intermediate lives in a
 * static ~2 MiB device array of the library (held by each GPU that loads the
 * library until exit).  n <= 256, else TB_CAPACITY_EXCEEDED.  All calls on a
 * device share that array: calls whose GPU work overlaps race, so serialise
 * them.  The first call on a device does a one-time set-up (it looks up the
 * array's address and raises the eigensolver's shared memory limit, neither of
 * which allocates); make it before any stream capture.  Synchronous on
 * `stream`. */
tb_status tb_sygvd_noalloc(int32_t n, const double* H, const double* S, double* w, double* C, void* stream);

/* get_fermi_filling (src/wavefunction/fermi.cu:100-124) for one spin channel. */
tb_status tb_fermi_filling(int32_t n, double nel, double kt, const double* emo, double* occ,
                           double* efermi, double* ts);

#ifdef __cplusplus
}
#endif
#endif
