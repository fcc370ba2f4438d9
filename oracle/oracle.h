/*
 * FP64 CPU oracle for the GFN2-xTB singlepoint path -- TEST INFRASTRUCTURE ONLY.
 *
 * This library is a host restatement of the semantics that tornikeo/tblite-cuda
 * quotes from tblite (Fortran) next to each of its device functions, with the
 * reference's translation defects fixed.  It is the checker for the CUDA
 * product library and the timed CPU baseline; nothing in the product links it.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use it.
 *
 * Parity status: pinned on the reference's own known-answer data
 * (src/test.old:97-150 multipole_3d s-s, src/test.old:152-176 transform0 s-d,
 * src/blas/level2.cu:14-26 gemv case 1, src/lapack/sygvd.cu:180-186 2x2 sygvd)
 * and on scipy.linalg.eigh; singlepoint energies/charges have no golden values
 * anywhere in the reference (its SCF never runs), so they are unpinned.
 *
 * Array conventions (row-major C):
 *   xyz[nat][3] Bohr; id[nat] 0-based species index of the parameter file.
 *   S, H0 [nao][nao] symmetric.
 *   D[3][nao][nao], Q[6][nao][nao] planar: D[k][mu][nu] = <mu|(r-R_at(nu))_k|nu>,
 *   i.e. the moment operator sits on the atom of the column index (tblite's
 *   "centered on last index", reference src/integral/type.h:13-16).
 *   Quadrupole components are (xx, xy, yy, xz, yz, zz), traceless.
 *   dpat[nat][3], qpat[nat][6]; qsh[nsh]; qat[nat] are partial charges.
 */
#ifndef TB_ORACLE_H
#define TB_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_params orc_params;

typedef struct orc_options {
  double accuracy;       /* tblite accuracy; econv = 1e-6*acc, pconv = 2e-5*acc */
  double kt;             /* electronic temperature in Eh */
  int max_iter;          /* SCF iterations and Broyden memory */
  double damping;        /* Broyden damping */
  int verbosity;
} orc_options;

typedef struct orc_result {
  double energy;         /* total = e_elec + e_rep + e_disp */
  double e_rep, e_elec;  /* repulsion; electronic incl. Coulomb and -TS */
  double e_band, e_ts, e_es2, e_aes2, e_es3;
  double dipole[3];
  int iterations;
  int status;            /* 0 ok, see ORC_* below */
  int nsh, nao;
  double e_disp;         /* D4 dispersion (0 without a D4 block in the parameter file) */
} orc_result;

enum { ORC_OK = 0, ORC_BAD_INPUT = 1, ORC_NOT_SPD = 2, ORC_SCF_NOT_CONVERGED = 3,
       ORC_FERMI_NOT_CONVERGED = 4, ORC_EIGEN_FAILED = 5 };

orc_params* orc_params_load(const char* path, char* err, int errlen);
void orc_params_free(orc_params* p);
int orc_nspecies(const orc_params* p);
void orc_default_options(orc_options* opt);
int orc_basis_size(const orc_params* p, int nat, const int* id, int* nsh, int* nao);
/* shell/AO maps (any may be NULL): ish_at[nat], iao_sh[nsh], ao2at[nao], ao2sh[nao], sh2at[nsh], ang_sh[nsh] */
int orc_basis_maps(const orc_params* p, int nat, const int* id, int* ish_at, int* iao_sh,
                   int* ao2at, int* ao2sh, int* sh2at, int* ang_sh);

/* ---- stages (each mirrors one reference function) ---- */
double orc_cutoff(const orc_params* p, double accuracy);
int orc_adjacency_list(int nat, const double* xyz, double cutoff, int* inl, int* nnl,
                       int* nlat, int* nltr, int cap, int* npair);
int orc_coordination_number(const orc_params* p, int nat, const int* id, const double* xyz, double* cn);
int orc_mrad(const orc_params* p, int nat, const int* id, const double* cn, double* mrad);
int orc_selfenergy(const orc_params* p, int nat, const int* id, const double* cn, double* se);
int orc_hamiltonian(const orc_params* p, int nat, const int* id, const double* xyz,
                    double* S, double* H0, double* D, double* Q);
int orc_repulsion(const orc_params* p, int nat, const int* id, const double* xyz, double* erep_at);
/* dispersion_get_engrad (src/xtb.cu:274-277): D4 at the neutral reference
 * charges from the parameter file's D4 block; per-atom energies, gradient
 * grad[nat][3] and virial sigma[3][3] (either may be NULL); all zero without
 * a D4 block (orc_has_dispersion returns 0). */
int orc_dispersion(const orc_params* p, int nat, const int* id, const double* xyz, double* edisp_at, double* grad,
                   double* sigma);
int orc_has_dispersion(const orc_params* p);
int orc_coulomb_matrices(const orc_params* p, int nat, const int* id, const double* xyz,
                         double* gamma, double* amat_sd, double* amat_dd, double* amat_sq);
int orc_coulomb_potential(const orc_params* p, int nat, const int* id, const double* xyz,
                          const double* qsh, const double* dpat, const double* qpat,
                          double* vsh, double* vat, double* vdp, double* vqp);
int orc_coulomb_energy(const orc_params* p, int nat, const int* id, const double* xyz,
                       const double* qsh, const double* dpat, const double* qpat,
                       double* e_es2, double* e_aes2, double* e_es3);
int orc_fock(const orc_params* p, int nat, const int* id, const double* S, const double* H0,
             const double* D, const double* Q, const double* vsh, const double* vat,
             const double* vdp, const double* vqp, double* F);
int orc_sygvd(int n, const double* H, const double* S, double* w, double* C);
int orc_fermi(int n, double nel, double kt, const double* emo, double* occ, double* efermi, double* ts);
int orc_density(int n, const double* C, const double* focc, double* P);
int orc_mulliken(const orc_params* p, int nat, const int* id, const double* S, const double* D,
                 const double* Q, const double* P, double* qsh, double* qat, double* dpat, double* qpat);

/* ---- singlepoint ---- */
int orc_singlepoint(const orc_params* p, int nat, const int* id, const double* xyz, double charge,
                    int uhf, const orc_options* opt, orc_result* res, double* qat, double* qsh,
                    double* dpat, double* qpat, double* emo, double* P);
/* The same singlepoint in tblite's nspin = 2 representation: per channel
 * (alpha, beta) occupations focc2[2][nao] and densities P2[2][nao][nao]; the
 * moments in the charge/magnetization representation (channel 0 = total,
 * channel 1 = up - down): qsh2[2][nsh], qat2[2][nat], dpat2[2][nat][3],
 * qpat2[2][nat][6].  Any output may be NULL. */
int orc_singlepoint_spin(const orc_params* p, int nat, const int* id, const double* xyz, double charge,
                         int uhf, const orc_options* opt, orc_result* res, double* focc2, double* P2,
                         double* qsh2, double* qat2, double* dpat2, double* qpat2);
/* The singlepoint and its analytic nuclear gradient grad[nat][3] (Eh/Bohr) and
 * virial sigma[3][3] = sum_A grad_A R_A^T. */
int orc_singlepoint_gradient(const orc_params* p, int nat, const int* id, const double* xyz, double charge,
                             int uhf, const orc_options* opt, orc_result* res, double* grad, double* sigma);
/* nmol structures packed back to back (atom offsets in aoff[nmol+1]), nthreads std::threads */
int orc_singlepoint_batch(const orc_params* p, int nmol, const int* aoff, const int* id,
                          const double* xyz, const double* charge, const int* uhf,
                          const orc_options* opt, int nthreads, orc_result* res);

/* ---- primitives for the reference's known-answer tests ---- */
void orc_multipole_3d(const double* rpj, const double* rpi, double aj, double ai, const int* lj,
                      const int* li, const double* s1d, double* s3d, double* d3d, double* q3d);
void orc_transform0(int lj, int li, const double* cart, double* sphr);
void orc_gemv(int m, int n, const double* A, const double* x, double* y, double alpha,
              double beta, int trans);
/* one shell pair: blocks s[msao_i][msao_j], d[msao_i][msao_j][3], q[...][6]; vec = ri - rj */
int orc_multipole_cgto(const orc_params* p, int jsp, int jsh, int isp, int ish, double r2,
                       const double* vec, double intcut, double* s, double* d, double* q);

#ifdef __cplusplus
}
#endif
#endif
