// SCF iteration kernels (next_scf, reference src/scf/iterators.cu:317-424 and
// the quoted Fortran src/scf/iterators.h:53-95), batched over structures.
//
// Coulomb interaction matrices are never stored: the ES2 gamma (get_amat_0d,
// src/coulomb.cu:15-47) and the AES2 multipole tensors
// (get_multipole_matrix_0d, :409-467) are re-evaluated from the coordinates
// inside the potential and energy kernels, which replaces 8*(S^2 + 18 A^2)
// bytes of matrix traffic per iteration by a few flops per pair.
#include "tb_common.cuh"
#include "tb_kernels.h"

namespace tb {

__device__ const double kMpScale[6] = {1, 2, 1, 2, 2, 1};

// gamma between shell a (type ta, atom A) and shell b (type tb, atom Bq)
__device__ inline double gamma_ab(const DevParams& P, int ta, int tbt, bool same_atom, double r2) {
  const double gam = 0.5 * (P.sh[ta].hubbard + P.sh[tbt].hubbard);
  if (same_atom) return gam;
  if (P.gexp == 2.0) return 1.0 / sqrt(r2 + 1.0 / (gam * gam));
  const double r1 = sqrt(r2);
  return 1.0 / pow(pow(r1, P.gexp) + pow(gam, -P.gexp), 1.0 / P.gexp);
}

// AES2 damping functions fdmp3, fdmp5 (quoted Fortran, src/coulomb.cu:449-451)
__device__ inline void aes_damp(const DevParams& P, double rA, double rB, double g1, double& f3, double& f5) {
  const double rr = 0.5 * (rA + rB) * g1;
  const double lr = log(rr);
  f3 = 1.0 / (1.0 + 6.0 * exp(P.kdmp3 * lr));
  f5 = 1.0 / (1.0 + 6.0 * exp(P.kdmp5 * lr));
}

__device__ inline void tcomp(const double* v, double* tc) {
  tc[0] = v[0] * v[0]; tc[1] = 2 * v[0] * v[1]; tc[2] = v[1] * v[1];
  tc[3] = 2 * v[0] * v[2]; tc[4] = 2 * v[1] * v[2]; tc[5] = v[2] * v[2];
}

// ------------------------------------------------------------ initial state
// Per structure: repulsion sum, reference occupations (get_occupation,
// src/h0.cu:61-91), alpha/beta split (src/xtb.cu:300-313 and
// src/wavefunction/type.cu:3-14), charge guess, mixer reset.
__global__ void k_scf_init(DevParams P, DevBatch B, const double* __restrict__ charge, const int* __restrict__ uhf,
                           const double* __restrict__ erep, double* __restrict__ n0sh, double* __restrict__ q_in,
                           MolState S) {
  const int m = blockIdx.x;
  __shared__ double red[32];
  const int a0 = B.aoff[m], nat = B.aoff[m + 1] - a0;
  const int s0 = B.soff[m], nsh = B.soff[m + 1] - s0;
  double e = 0.0, r = 0.0;
  for (int a = threadIdx.x; a < nat; a += blockDim.x) e += erep[a0 + a];
  for (int s = threadIdx.x; s < nsh; s += blockDim.x) {
    const double ro = P.sh[B.sh_type[s0 + s]].refocc;
    n0sh[s0 + s] = ro;
    r += ro;
  }
  const double etot = block_sum(e, red);
  const double nref = block_sum(r, red);
  const double q = charge[m];
  // guess: q/nat per atom split over its shells by reference occupation
  const int mo = B.mixoff[m];
  for (int a = threadIdx.x; a < nat; a += blockDim.x) {
    const SpeciesParam& sp = P.sp[B.id[a0 + a]];
    double tot = 0.0;
    for (int s = 0; s < sp.nsh; ++s) tot += P.sh[sp.sh0 + s].refocc;
    const int is = B.at_ish[a0 + a];
    for (int s = 0; s < sp.nsh; ++s) {
      const double f = tot > 0.0 ? P.sh[sp.sh0 + s].refocc / tot : 1.0 / sp.nsh;
      q_in[mo + is + s] = q / nat * f;
    }
    for (int k = 0; k < 9; ++k) q_in[mo + nsh + 9 * a + k] = 0.0;
  }
  if (threadIdx.x == 0) {
    S.e_rep[m] = etot;
    const double nocc = nref - q;
    const long long inel = llround(nocc);
    const int nuhf = ((uhf[m] % 2) == (int)(inel % 2)) ? uhf[m] : (int)(inel % 2);
    const double diff = fmin((double)nuhf, nocc), ntmp = nocc - diff;
    S.nel[2 * m] = ntmp / 2 + diff;
    S.nel[2 * m + 1] = ntmp / 2;
    S.iscf[m] = 0;
    S.mix_iter[m] = 0;
    S.eelec[m] = 0.0;
    S.active[m] = S.status[m] == kStOk ? 1 : 0;
    if (S.phase) { S.phase[m] = 0; S.n64[m] = 0; }  // mixed-precision form starts in the mixed phase
    if (S.active[m]) atomicAdd(S.n_active, 1);
  }
}

// Serving: the unfinished structures of a micro-batch continue in a smaller
// batch (server_compact).  Everything a structure carries from one SCF
// iteration to the next moves with it: the mixer vectors and its Broyden
// history slab, the per-structure scalars (iteration counters, energies,
// phase of the mixed form, status).  Geometry-derived data (integrals, X,
// pair tables) is recomputed by the new batch's setup, bit for bit the same.
__global__ void k_compact_state(DevBatch Bo, DevBatch Bn, const int* __restrict__ map, ScfState so, ScfState sn,
                                int memory) {
  const int k = blockIdx.x, m = map[k];
  const int mo = Bo.mixoff[m], mn = Bn.mixoff[k], n = Bo.mixoff[m + 1] - mo;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    sn.q_in[mn + i] = so.q_in[mo + i];
    sn.dq[mn + i] = so.dq[mo + i];
    sn.dqlast[mn + i] = so.dqlast[mo + i];
    sn.qlast[mn + i] = so.qlast[mo + i];
  }
  const long long ho = (long long)mo * memory, hn = (long long)mn * memory;
  for (long long i = threadIdx.x; i < (long long)n * memory; i += blockDim.x) {
    sn.df[hn + i] = so.df[ho + i];
    sn.u[hn + i] = so.u[ho + i];
  }
  for (int i = threadIdx.x; i < memory * memory; i += blockDim.x)
    sn.amat[(long long)k * memory * memory + i] = so.amat[(long long)m * memory * memory + i];
  for (int i = threadIdx.x; i < memory; i += blockDim.x) sn.omega[(long long)k * memory + i] = so.omega[(long long)m * memory + i];
  if (threadIdx.x == 0) {
    const MolState& a = so.S;
    const MolState& b = sn.S;
    b.e_rep[k] = a.e_rep[m];
    b.nel[2 * k] = a.nel[2 * m];
    b.nel[2 * k + 1] = a.nel[2 * m + 1];
    b.iscf[k] = a.iscf[m];
    b.mix_iter[k] = a.mix_iter[m];
    b.eelec[k] = a.eelec[m];
    b.active[k] = a.active[m];
    b.status[k] = a.status[m];
    b.e_ts[k] = a.e_ts[m];
    b.e_band[k] = a.e_band[m];
    b.e_es2[k] = a.e_es2[m];
    b.e_aes2[k] = a.e_aes2[m];
    b.e_es3[k] = a.e_es3[m];
    b.scf_error[k] = a.scf_error[m];
    b.fermi_warn[k] = a.fermi_warn[m];
    for (int x = 0; x < 3; ++x) b.dipole[3 * k + x] = a.dipole[3 * m + x];
    if (a.phase && b.phase) { b.phase[k] = a.phase[m]; b.n64[k] = a.n64[m]; }
  }
}

// Last node of the body of the SCF loop graph (one graph launch runs the whole
// loop): counts the iteration and keeps the WHILE node looping while a
// structure is still active and the iteration budget is not spent (the
// convergence test itself is made per structure by k_finalize).
__global__ void k_loop_control(cudaGraphConditionalHandle h, const int* __restrict__ n_active, int* __restrict__ it,
                               int max_iter) {
  const int done = *it + 1;
  *it = done;
  cudaGraphSetConditional(h, (*n_active > 0 && done < max_iter) ? 1u : 0u);
}

// Starting point of the SCF taken from the caller's wavefunction (the
// reference's xtb_singlepoint takes wfn in and out, src/xtb.cu:188-197, and
// its first iteration builds the potential from the charges it holds): the
// moments [qsh, dpat, qpat] of flagged structures replace the default guess
// that k_scf_init wrote.
__global__ void k_apply_guess(DevBatch B, const double* __restrict__ guess, const int* __restrict__ flag,
                              double* __restrict__ q_in) {
  const int m = blockIdx.x;
  if (!flag[m]) return;
  const int mo = B.mixoff[m], ndim = B.mixoff[m + 1] - mo;
  for (int i = threadIdx.x; i < ndim; i += blockDim.x) q_in[mo + i] = guess[mo + i];
}

// ------------------------------------------------------------ pair tables
// The geometry is fixed during the SCF, so the shell-pair Coulomb kernel
// gamma_ab (ES2) and the atom-pair 1/r and AES2 damping factors are
// evaluated once per batch: gtab[s2off + a nsh + b] = gamma_ab(a, b);
// atab[3 (a2off + A nat + B) + {0, 1, 2}] = {1/r, f3, f5} (zero for A = B).
// Both tables are symmetric bit for bit (the terms only see squared
// differences and symmetric sums), so the per-iteration kernels read column
// t of them (coalesced) instead of recomputing log/exp/sqrt per pair.  The
// reference likewise fills its Coulomb cache once per geometry
// (effective_coulomb::update, src/coulomb.cu:82-98; damped_multipole::update,
// :153) and reuses it in every iteration.
__global__ void k_pair_tables(DevParams P, DevBatch B, const double* __restrict__ mrad, double* __restrict__ gtab,
                              double* __restrict__ atab) {
  const int m = blockIdx.x;
  const int a0 = B.aoff[m], nat = B.aoff[m + 1] - a0;
  const int s0 = B.soff[m], nsh = B.soff[m + 1] - s0;
  const double* xyz = B.xyz + 3 * a0;
  double* g = gtab + B.s2off[m];
  double* at = atab + 3 * B.a2off[m];
  for (long long e = blockIdx.y * (long long)blockDim.x + threadIdx.x; e < (long long)nsh * nsh;
       e += (long long)gridDim.y * blockDim.x) {
    const int a = (int)(e / nsh), b = (int)(e - (long long)a * nsh);
    const int A = B.sh_at[s0 + a], Bq = B.sh_at[s0 + b];
    const double dx = xyz[3 * A] - xyz[3 * Bq], dy = xyz[3 * A + 1] - xyz[3 * Bq + 1], dz = xyz[3 * A + 2] - xyz[3 * Bq + 2];
    g[e] = gamma_ab(P, B.sh_type[s0 + a], B.sh_type[s0 + b], A == Bq, dx * dx + dy * dy + dz * dz);
  }
  for (long long e = blockIdx.y * (long long)blockDim.x + threadIdx.x; e < (long long)nat * nat;
       e += (long long)gridDim.y * blockDim.x) {
    const int A = (int)(e / nat), Bq = (int)(e - (long long)A * nat);
    double g1 = 0.0, f3 = 0.0, f5 = 0.0;
    if (A != Bq) {
      const double v[3] = {xyz[3 * Bq] - xyz[3 * A], xyz[3 * Bq + 1] - xyz[3 * A + 1], xyz[3 * Bq + 2] - xyz[3 * A + 2]};
      const double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
      g1 = 1.0 / sqrt(r2);
      aes_damp(P, mrad[a0 + A], mrad[a0 + Bq], g1, f3, f5);
    }
    at[3 * e] = g1;
    at[3 * e + 1] = f3;
    at[3 * e + 2] = f5;
  }
}

// ------------------------------------------------------------ potentials
// tb_coulomb::get_potential for the mixed input moments q_in = [qsh, dpat,
// qpat]: ES2 (vsh += gamma qsh), ES3 (vsh += qsh^2 dGamma), AES2 (the five
// gemv of the quoted Fortran src/coulomb.cu:665-676) and the on-site kernels
// (get_kernel_potential, :564-589).  grid = (structure, target chunk of
// kPotTargets); one warp per target shell and atom, lanes over the partners
// (row t of the pair tables, which are symmetric bit for bit, so the lanes
// read contiguously), partial sums reduced across the warp in a fixed order.
// With the pair tables (gtab, atab non-null) the pair terms are read, not
// recomputed; the arithmetic on them is unchanged.
__global__ void k_potential(DevParams P, DevBatch B, const double* __restrict__ q_in,
                            const double* __restrict__ mrad, double* __restrict__ vsh, double* __restrict__ vat,
                            double* __restrict__ vdp, double* __restrict__ vqp, const int* __restrict__ active,
                            const double* __restrict__ gtab, const double* __restrict__ atab) {
  const int m = blockIdx.x;
  if (!active[m]) return;
  const int a0 = B.aoff[m], nat = B.aoff[m + 1] - a0;
  const int s0 = B.soff[m], nsh = B.soff[m + 1] - s0;
  const double* qsh = q_in + B.mixoff[m];
  const double* dp = qsh + nsh;
  const double* qp = dp + 3 * nat;
  const int lane = threadIdx.x & 31;
  const int t = blockIdx.y * kPotTargets + (threadIdx.x >> 5);
  const double* xyz = B.xyz + 3 * a0;
  // shells
  if (t < nsh) {
    const int ta = B.sh_type[s0 + t], A = B.sh_at[s0 + t];
    double v = 0.0;
    if (gtab) {
      const double* gr = gtab + B.s2off[m] + (long long)t * nsh;  // row t = column t
      for (int b = lane; b < nsh; b += 32) v += gr[b] * qsh[b];
    } else {
      for (int b = lane; b < nsh; b += 32) {
        const int Bq = B.sh_at[s0 + b];
        const double dx = xyz[3 * A] - xyz[3 * Bq], dy = xyz[3 * A + 1] - xyz[3 * Bq + 1], dz = xyz[3 * A + 2] - xyz[3 * Bq + 2];
        v += gamma_ab(P, ta, B.sh_type[s0 + b], A == Bq, dx * dx + dy * dy + dz * dz) * qsh[b];
      }
    }
    v = warp_sum(v);
    if (lane == 0) vsh[s0 + t] = v + qsh[t] * qsh[t] * P.sh[ta].hubbard_deriv;
  }
  // atoms
  if (t < nat) {
    const int A = t;
    double va = 0.0, vd[3] = {0, 0, 0}, vq[6] = {0, 0, 0, 0, 0, 0};
    const double rA = mrad[a0 + A];
    const double* ar = atab ? atab + 3 * (B.a2off[m] + (long long)A * nat) : nullptr;  // row A = column A
    for (int Bq = lane; Bq < nat; Bq += 32) {
      if (Bq == A) continue;
      const double v[3] = {xyz[3 * Bq] - xyz[3 * A], xyz[3 * Bq + 1] - xyz[3 * A + 1], xyz[3 * Bq + 2] - xyz[3 * A + 2]};
      double g1, f3, f5;
      if (ar) {
        const double* e = ar + 3LL * Bq;
        g1 = e[0]; f3 = e[1]; f5 = e[2];
      } else {
        const double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        g1 = 1.0 / sqrt(r2);
        aes_damp(P, rA, mrad[a0 + Bq], g1, f3, f5);
      }
      const double g3 = g1 * g1 * g1, g5 = g3 * g1 * g1;
      // qat of atom Bq from its shells
      const int isb = B.at_ish[a0 + Bq], nsb = P.sp[B.id[a0 + Bq]].nsh;
      double qb = 0.0;
      for (int s = 0; s < nsb; ++s) qb += qsh[isb + s];
      const double* db = dp + 3 * Bq;
      const double* qpb = qp + 6 * Bq;
      const double vdb = v[0] * db[0] + v[1] * db[1] + v[2] * db[2];
      double tc[6];
      tcomp(v, tc);
      for (int k = 0; k < 3; ++k) vd[k] += v[k] * g3 * f3 * qb + (g3 * db[k] - 3.0 * v[k] * vdb * g5) * f5;
      for (int c = 0; c < 6; ++c) vq[c] += tc[c] * g5 * f5 * qb;
      double tq = 0.0;
      for (int c = 0; c < 6; ++c) tq += tc[c] * qpb[c];
      va += -vdb * g3 * f3 + tq * g5 * f5;
    }
    va = warp_sum(va);
    for (int k = 0; k < 3; ++k) vd[k] = warp_sum(vd[k]);
    for (int c = 0; c < 6; ++c) vq[c] = warp_sum(vq[c]);
    if (lane == 0) {
      const SpeciesParam& sp = P.sp[B.id[a0 + A]];
      for (int k = 0; k < 3; ++k) vd[k] += 2.0 * sp.dkernel * dp[3 * A + k];
      for (int c = 0; c < 6; ++c) vq[c] += 2.0 * sp.qkernel * qp[6 * A + c] * kMpScale[c];
      vat[a0 + A] = va;
      for (int k = 0; k < 3; ++k) vdp[3 * (a0 + A) + k] = vd[k];
      for (int c = 0; c < 6; ++c) vqp[6 * (a0 + A) + c] = vq[c];
    }
  }
}

// ------------------------------------------------------------ Fock build
// add_pot_to_h1 (src/scf/potential.cu:224-272 with the quoted add_vat_to_vsh,
// add_vsh_to_vao, add_vao_to_h1 and add_vmp_to_h1): 32x32 tiles.  F is
// symmetric (the moment planes enter as M[mu][nu] v(nu) + M[nu][mu] v(mu)), so
// the tile list holds only tiles on and above the diagonal; an off-diagonal
// tile is also written transposed (through shared memory), which halves the
// reads.  The kernel is bound by how many bytes are in flight: every CTA
// issues all of its loads in one round -- the nine transposed moment tiles
// (M[nu][mu]) as cp.async copies into shared memory (74 KiB, no registers
// held), the nine direct tiles and S, H0 into registers -- and waits once.
constexpr int kFockPitch = 33;  // padded rows: the transposed reads are conflict-free
size_t fock_smem_bytes() { return (size_t)9 * 32 * kFockPitch * sizeof(double); }

__device__ __forceinline__ void fock_cp_async8(double* smem, const double* gmem, bool valid) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  const int nb = valid ? 8 : 0;  // bytes read; the rest of the 8 is zero-filled
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(sa), "l"(gmem), "r"(nb) : "memory");
}

__global__ void __launch_bounds__(256, 2) k_fock(DevBatch B, const int4* __restrict__ tiles, int ntiles,
                                                 const double* __restrict__ S, const double* __restrict__ H0,
                                                 const double* __restrict__ D, const double* __restrict__ Q,
                                                 const double* __restrict__ vsh, const double* __restrict__ vat,
                                                 const double* __restrict__ vdp, const double* __restrict__ vqp,
                                                 double* __restrict__ F, const int* __restrict__ active) {
  extern __shared__ double fock_T[];  // [9][32][kFockPitch]: T[q][row][col] = M_q[c0 + row][r0 + col]
  const int t = blockIdx.x;
  if (t >= ntiles) return;
  const int4 tl = tiles[t];
  const int m = tl.x;
  if (!active[m] || tl.y > tl.z) return;
  const int n = B.ooff[m + 1] - B.ooff[m];
  const long long mo = B.moff[m], nn = (long long)n * n;
  const int o0 = B.ooff[m], a0 = B.aoff[m], s0 = B.soff[m];
  const int r0 = tl.y * 32, c0 = tl.z * 32;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 8 rows of 32
  // 1. the transposed tiles of the nine moment planes, asynchronously
#pragma unroll
  for (int q = 0; q < 9; ++q) {
    const double* M = q < 3 ? D + 3 * mo + q * nn : Q + 6 * mo + (q - 3) * nn;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int row = c0 + ty + 8 * r, col = r0 + tx;
      const bool ok = row < n && col < n;
      fock_cp_async8(&fock_T[(q * 32 + ty + 8 * r) * kFockPitch + tx], ok ? M + (long long)row * n + col : M, ok);
    }
  }
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  // 2. the direct elements of S, H0 and the nine planes, into registers
  int mu[4];
  bool ok[4];
  const int nu = c0 + tx;
  const bool nu_ok = nu < n;
  double s_[4], h_[4], dir[9][4];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    mu[r] = r0 + ty + 8 * r;
    ok[r] = mu[r] < n && nu_ok;
    const long long e = mo + (long long)mu[r] * n + nu;
    if (ok[r] && !TB_GUARD(4, e, mo, mo + nn)) ok[r] = false;
    s_[r] = ok[r] ? S[e] : 0.0;
    h_[r] = ok[r] ? H0[e] : 0.0;
#pragma unroll
    for (int q = 0; q < 9; ++q) {
      const double* M = q < 3 ? D + 3 * mo + q * nn : Q + 6 * mo + (q - 3) * nn;
      dir[q][r] = ok[r] ? M[(long long)mu[r] * n + nu] : 0.0;
    }
  }
  // 3. potentials of the column's AO and of the rows' AOs
  const int at_nu = nu_ok ? B.ao_at[o0 + nu] : 0;
  const double vao_nu = nu_ok ? vsh[s0 + B.ao_sh[o0 + nu]] + vat[a0 + at_nu] : 0.0;
  double vm_nu[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) vm_nu[q] = nu_ok ? (q < 3 ? vdp[3 * (a0 + at_nu) + q] : vqp[6 * (a0 + at_nu) + q - 3]) : 0.0;
  double acc[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    acc[r] = 0.0;
    if (!ok[r]) continue;
    const int at_mu = B.ao_at[o0 + mu[r]];
    const double vao_mu = vsh[s0 + B.ao_sh[o0 + mu[r]]] + vat[a0 + at_mu];
    acc[r] = h_[r] - s_[r] * 0.5 * (vao_mu + vao_nu);
  }
  asm volatile("cp.async.wait_all;\n" ::: "memory");
  __syncthreads();
  // 4. -0.5 * (M[q][mu][nu] v[at(nu)][q] + M[q][nu][mu] v[at(mu)][q]), planes in order
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    if (!ok[r]) continue;
    const int at_mu = a0 + B.ao_at[o0 + mu[r]];
#pragma unroll
    for (int q = 0; q < 9; ++q) {
      const double vmu = q < 3 ? vdp[3 * at_mu + q] : vqp[6 * at_mu + q - 3];
      acc[r] -= 0.5 * (dir[q][r] * vm_nu[q] + fock_T[(q * 32 + tx) * kFockPitch + ty + 8 * r] * vmu);
    }
  }
#pragma unroll
  for (int r = 0; r < 4; ++r)
    if (ok[r] && TB_GUARD(5, (long long)mu[r] * n + nu, 0, nn)) F[mo + (long long)mu[r] * n + nu] = acc[r];
  if (r0 != c0) {  // F[c0.., r0..] = this tile transposed
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 4; ++r) fock_T[(ty + 8 * r) * kFockPitch + tx] = acc[r];
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int row = c0 + ty + 8 * r, col = r0 + tx;
      if (row < n && col < n && TB_GUARD(5, (long long)row * n + col, 0, nn))
        F[mo + (long long)row * n + col] = fock_T[tx * kFockPitch + ty + 8 * r];
    }
  }
}

// ------------------------------------------------------------ Fermi
// get_fermi_filling (src/wavefunction/fermi.cu:6-124) on the ascending
// eigenvalues: aufbau guess, Newton on E_F safeguarded by bisection, tolerance
// |N(E_F) - homo| <= 1e-10, entropy -TS over all 0 < f < 1.  Writes the total
// occupation per orbital (both spin channels, nspin = 1) and K = number of
// leading nonzero occupations.
__device__ double fermi_channel(int n, double nel, double kt, const double* w, double* occ, double* red,
                                int& ok, double& efermi) {
  const int tid = threadIdx.x, nt = blockDim.x;
  int homo = (int)floor(nel);
  const double frac = fmod(nel, 1.0);
  for (int i = tid; i < n; i += nt) occ[i] = i < homo ? 1.0 : (i == homo ? frac : 0.0);
  if (frac > 0.5) homo += 1;
  ok = 1;
  efermi = 0.0;
  if (homo <= 0) { __syncthreads(); return 0.0; }
  const double occt = (double)homo;
  double ef = 0.5 * (w[max(homo - 1, 0)] + w[min(homo, n - 1)]);
  double lo = w[0] - 1.0, hi = w[n - 1] + 1.0;
  ok = 0;
  for (int cycle = 0; cycle < 200; ++cycle) {
    double tot = 0.0, dtot = 0.0;
    for (int i = tid; i < n; i += nt) {
      const double x = (w[i] - ef) / kt;
      double f = 0.0, df = 0.0;
      if (x < 50.0) {
        const double ex = exp(x);
        f = 1.0 / (ex + 1.0);
        df = ex / (kt * (ex + 1.0) * (ex + 1.0));
      }
      occ[i] = f;
      tot += f;
      dtot += df;
    }
    tot = block_sum(tot, red);
    dtot = block_sum(dtot, red);
    if (fabs(occt - tot) <= 1e-10) { ok = 1; break; }
    if (tot < occt) lo = ef; else hi = ef;
    double next = ef + (occt - tot) / dtot;
    if (!(dtot > 0.0) || !(next > lo && next < hi)) next = 0.5 * (lo + hi);
    ef = next;
  }
  efermi = ef;
  double s = 0.0;
  for (int i = tid; i < n; i += nt) {
    const double o = occ[i];
    if (o > 0.0 && o < 1.0) s += o * log(o) + (1.0 - o) * log(1.0 - o);
  }
  return block_sum(s, red) * kt;
}

__global__ void k_fermi(DevBatch B, const double* __restrict__ w, double kt, double* __restrict__ focc,
                        int* __restrict__ kdim, MolState S) {
  const int m = blockIdx.x;
  if (!S.active[m]) return;
  if (S.status[m] != kStOk) {  // eigensolver failure: retire the structure
    // (the density GEMMs of the mixed form mask by the phase at the start of
    // the iteration and still visit it: no orbitals are occupied)
    if (threadIdx.x == 0) { S.active[m] = 0; atomicSub(S.n_active, 1); kdim[m] = 0; }
    return;
  }
  const int n = B.ooff[m + 1] - B.ooff[m];
  const int o0 = B.ooff[m];
  extern __shared__ double occ[];  // n
  __shared__ double red[32];
  __shared__ int last;
  double* f = focc + o0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) f[i] = 0.0;
  double ts = 0.0;
  int ok_all = 1;
  const double na = S.nel[2 * m], nb = S.nel[2 * m + 1];
  for (int spin = 0; spin < 2; ++spin) {
    if (spin == 1 && na == nb) {
      for (int i = threadIdx.x; i < n; i += blockDim.x) f[i] *= 2.0;
      ts *= 2.0;
      break;
    }
    int ok;
    double ef;
    __syncthreads();
    ts += fermi_channel(n, spin == 0 ? na : nb, kt, w + o0, occ, red, ok, ef);
    ok_all &= ok;
    if (spin == 0 && S.e_fermi && threadIdx.x == 0) S.e_fermi[m] = ef;
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) f[i] += occ[i];
  }
  __syncthreads();
  if (threadIdx.x == 0) last = 0;
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x)
    if (f[i] > 0.0) atomicMax(&last, i + 1);
  __syncthreads();
  if (threadIdx.x == 0) {
    kdim[m] = last;
    S.e_ts[m] = ts;
    if (!ok_all) S.fermi_warn[m] = 1;
  }
}

// nspin = 2 (tblite's open-shell representation; the reference stops at
// "Unimplemented", src/scf/iterators.cu:247-248).  GFN2 has no spin-dependent
// potential, so both channels share the Fock matrix, its orbital energies and
// coefficients, and the SCF is the one above; the channels differ only in
// their Fermi filling (nel(spin) electrons, the spin loop of get_density,
// src/scf/iterators.cu:223-239).  Recomputed here for the read-out with the
// same fermi_channel as k_fermi, so the channels add up to its occupations.
__global__ void k_spin_occupations(DevBatch B, const double* __restrict__ w, double kt,
                                   const double* __restrict__ nel, const int* __restrict__ flag,
                                   double* __restrict__ f) {
  const int m = blockIdx.x;
  if (!flag[m]) return;
  const int n = B.ooff[m + 1] - B.ooff[m], o0 = B.ooff[m], no = B.nao_tot;
  extern __shared__ double occ[];  // n
  __shared__ double red[32];
  for (int spin = 0; spin < 2; ++spin) {
    int ok;
    double ef;
    __syncthreads();
    fermi_channel(n, nel[2 * m + spin], kt, w + o0, occ, red, ok, ef);
    __syncthreads();
    for (int i = threadIdx.x; i < n; i += blockDim.x) f[spin * no + o0 + i] = occ[i];
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) f[2 * no + o0 + i] = f[o0 + i] - f[no + o0 + i];
}

// Channel 1 of the charge/magnetization representation (updown_to_magnet,
// src/wavefunction/spin.h:4-16: (up, down) -> (up + down, up - down)): with
// q(spin) = n0/2 - population(P_spin), up - down is minus the population of
// P_alpha - P_beta, whose Mulliken column sums colred holds; dipoles and
// quadrupoles likewise (same reduction as k_finalize with no reference
// occupation).
__global__ void k_spin_moments(DevParams P, DevBatch B, const double* __restrict__ colred,
                               const int* __restrict__ flag, double* __restrict__ qsh, double* __restrict__ qat,
                               double* __restrict__ dpat, double* __restrict__ qpat) {
  const int m = blockIdx.x;
  if (!flag[m]) return;
  const int a0 = B.aoff[m], nat = B.aoff[m + 1] - a0, s0 = B.soff[m], nsh = B.soff[m + 1] - s0, o0 = B.ooff[m];
  for (int s = threadIdx.x; s < nsh; s += blockDim.x) {
    const int i0 = B.sh_iao[s0 + s], na = msao(P.sh[B.sh_type[s0 + s]].ang);
    double v = 0.0;
    for (int x = 0; x < na; ++x) v += colred[12 * (long long)(o0 + i0 + x)];
    qsh[s0 + s] = -v;
  }
  __syncthreads();
  for (int a = threadIdx.x; a < nat; a += blockDim.x) {
    const int is = B.at_ish[a0 + a];
    const SpeciesParam& sp = P.sp[B.id[a0 + a]];
    double q = 0.0, d[3] = {0, 0, 0}, qq[6] = {0, 0, 0, 0, 0, 0};
    for (int s = 0; s < sp.nsh; ++s) {
      q += qsh[s0 + is + s];
      const int i0 = B.sh_iao[s0 + is + s], na = msao(P.sh[sp.sh0 + s].ang);
      for (int x = 0; x < na; ++x) {
        const double* c = colred + 12 * (long long)(o0 + i0 + x);
        for (int k = 0; k < 3; ++k) d[k] -= c[2 + k];
        for (int k = 0; k < 6; ++k) qq[k] -= c[5 + k];
      }
    }
    qat[a0 + a] = q;
    for (int k = 0; k < 3; ++k) dpat[3 * (a0 + a) + k] = d[k];
    for (int k = 0; k < 6; ++k) qpat[6 * (a0 + a) + k] = qq[k];
  }
}

// ------------------------------------------------------------ Mulliken
// Column sums of P o {S, D, Q, H0} (get_mulliken_shell_charges,
// src/wavefunction/mulliken.h:8-34; get_mulliken_atomic_multipoles,
// src/wavefunction/mulliken.cu:40-64; get_electronic_energy,
// src/scf/iterators.cu:254-272).  One CTA = 32 columns x 8 row groups;
// results per column in colred[ao][12] (deterministic order).
__global__ void __launch_bounds__(256) k_mulliken_cols(DevBatch B, const int2* __restrict__ chunks, int nchunks,
                                                       const double* __restrict__ P, const double* __restrict__ S,
                                                       const double* __restrict__ H0, const double* __restrict__ D,
                                                       const double* __restrict__ Q, double* __restrict__ colred,
                                                       const int* __restrict__ active) {
  __shared__ double part[8][11][32];
  const int c = blockIdx.x;
  if (c >= nchunks) return;
  const int2 ch = chunks[c];
  const int m = ch.x;
  if (!active[m]) return;
  const int n = B.ooff[m + 1] - B.ooff[m];
  const long long mo = B.moff[m], nn = (long long)n * n;
  const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
  const int nu = ch.y * 32 + tx;
  double acc[11];
  for (int k = 0; k < 11; ++k) acc[k] = 0.0;
  if (nu < n && TB_GUARD(6, (long long)(n - 1) * n + nu, 0, nn)) {  // the column's last element in the slice
    // two rows per step so that 22 independent loads are in flight
    int mu = ty;
    for (; mu + 8 < n; mu += 16) {
      const long long e = (long long)mu * n + nu, e2 = e + 8LL * n;
      const double p = P[mo + e], p2 = P[mo + e2];
      double v[11], v2[11];
      v[0] = S[mo + e]; v2[0] = S[mo + e2];
      v[1] = H0[mo + e]; v2[1] = H0[mo + e2];
#pragma unroll
      for (int k = 0; k < 3; ++k) { v[2 + k] = D[3 * mo + k * nn + e]; v2[2 + k] = D[3 * mo + k * nn + e2]; }
#pragma unroll
      for (int k = 0; k < 6; ++k) { v[5 + k] = Q[6 * mo + k * nn + e]; v2[5 + k] = Q[6 * mo + k * nn + e2]; }
#pragma unroll
      for (int k = 0; k < 11; ++k) acc[k] += p * v[k] + p2 * v2[k];
    }
    for (; mu < n; mu += 8) {
      const long long e = (long long)mu * n + nu;
      const double p = P[mo + e];
      acc[0] += p * S[mo + e];
      acc[1] += p * H0[mo + e];
      for (int k = 0; k < 3; ++k) acc[2 + k] += p * D[3 * mo + k * nn + e];
      for (int k = 0; k < 6; ++k) acc[5 + k] += p * Q[6 * mo + k * nn + e];
    }
  }
  for (int k = 0; k < 11; ++k) part[ty][k][tx] = acc[k];
  __syncthreads();
  if (ty == 0 && nu < n && TB_GUARD(7, B.ooff[m] + nu, B.ooff[m], B.ooff[m + 1])) {
    double* out = colred + 12 * (long long)(B.ooff[m] + nu);
    for (int k = 0; k < 11; ++k) {
      double s = 0.0;
      for (int g = 0; g < 8; ++g) s += part[g][k][tx];
      out[k] = s;
    }
  }
}

// ------------------------------------------------------------ finalize
// Per structure: reduce the column sums to shell charges and atomic
// multipoles, evaluate the Coulomb energies with the output moments
// (tb_coulomb::get_energy: ES2 quoted :111-136, AES2 quoted :697-727, ES3
// quoted :866-899), diff the mixer (diff_mixer), the energy/density
// convergence test of xtb_singlepoint and the iteration bookkeeping.
__global__ void k_finalize(DevParams P, DevBatch B, const double* __restrict__ colred, const double* __restrict__ n0sh,
                           const double* __restrict__ mrad, const double* __restrict__ q_in, double* __restrict__ dq,
                           double* __restrict__ qsh_out, double* __restrict__ qat_out, double* __restrict__ dpat_out,
                           double* __restrict__ qpat_out, double econv, double pconv, int max_iter, MolState S,
                           double econv_lo, double pconv_lo, const double* __restrict__ gtab,
                           const double* __restrict__ atab) {
  const int m = blockIdx.x;
  if (!S.active[m]) return;
  __shared__ double red[32];
  const int a0 = B.aoff[m], nat = B.aoff[m + 1] - a0;
  const int s0 = B.soff[m], nsh = B.soff[m + 1] - s0;
  const int o0 = B.ooff[m], n = B.ooff[m + 1] - o0;
  const int tid = threadIdx.x, nt = blockDim.x;
  // shells: qsh = n0sh - sum over the shell's AO columns
  for (int s = tid; s < nsh; s += nt) {
    const int i0 = B.sh_iao[s0 + s], na = msao(P.sh[B.sh_type[s0 + s]].ang);
    double v = 0.0;
    for (int x = 0; x < na; ++x) v += colred[12 * (long long)(o0 + i0 + x)];
    qsh_out[s0 + s] = n0sh[s0 + s] - v;
  }
  double eb = 0.0;
  for (int x = tid; x < n; x += nt) eb += colred[12 * (long long)(o0 + x) + 1];
  const double e_band = block_sum(eb, red);
  __syncthreads();
  // atoms: dipole/quadrupole over the atom's AO columns, qat over its shells
  for (int a = tid; a < nat; a += nt) {
    const int is = B.at_ish[a0 + a];
    const SpeciesParam& sp = P.sp[B.id[a0 + a]];
    double q = 0.0, d[3] = {0, 0, 0}, qq[6] = {0, 0, 0, 0, 0, 0};
    for (int s = 0; s < sp.nsh; ++s) {
      q += qsh_out[s0 + is + s];
      const int i0 = B.sh_iao[s0 + is + s], na = msao(P.sh[sp.sh0 + s].ang);
      for (int x = 0; x < na; ++x) {
        const double* c = colred + 12 * (long long)(o0 + i0 + x);
        for (int k = 0; k < 3; ++k) d[k] -= c[2 + k];
        for (int k = 0; k < 6; ++k) qq[k] -= c[5 + k];
      }
    }
    qat_out[a0 + a] = q;
    for (int k = 0; k < 3; ++k) dpat_out[3 * (a0 + a) + k] = d[k];
    for (int k = 0; k < 6; ++k) qpat_out[6 * (a0 + a) + k] = qq[k];
  }
  __syncthreads();
  const double* xyz = B.xyz + 3 * a0;
  const double* qs = qsh_out + s0;
  // ES2 + ES3 and AES2: one warp per shell (atom), lanes over the partners
  // (row a of the symmetric pair tables), reduced across the warp in a fixed
  // order; lane 0 adds the target's energy terms
  const int lane = tid & 31, warp = tid >> 5, nwarp = nt >> 5;
  double e2 = 0.0, e3 = 0.0;
  for (int a = warp; a < nsh; a += nwarp) {
    const int ta = B.sh_type[s0 + a], A = B.sh_at[s0 + a];
    double v = 0.0;
    if (gtab) {
      const double* gr = gtab + B.s2off[m] + (long long)a * nsh;  // row a = column a
      for (int b = lane; b < nsh; b += 32) v += gr[b] * qs[b];
    } else {
      for (int b = lane; b < nsh; b += 32) {
        const int Bq = B.sh_at[s0 + b];
        const double dx = xyz[3 * A] - xyz[3 * Bq], dy = xyz[3 * A + 1] - xyz[3 * Bq + 1], dz = xyz[3 * A + 2] - xyz[3 * Bq + 2];
        v += gamma_ab(P, ta, B.sh_type[s0 + b], A == Bq, dx * dx + dy * dy + dz * dz) * qs[b];
      }
    }
    v = warp_sum(v);
    if (lane == 0) {
      e2 += 0.5 * v * qs[a];
      e3 += qs[a] * qs[a] * qs[a] * P.sh[ta].hubbard_deriv / 3.0;
    }
  }
  // AES2: vd = sd q + 0.5 dd dp, vq = sq q; E = dp.vd + qp.vq + kernels
  double ea = 0.0;
  for (int A = warp; A < nat; A += nwarp) {
    const double* dA = dpat_out + 3 * (a0 + A);
    const double* qA = qpat_out + 6 * (a0 + A);
    double vd[3] = {0, 0, 0}, vq[6] = {0, 0, 0, 0, 0, 0};
    const double rA = mrad[a0 + A];
    const double* ar = atab ? atab + 3 * (B.a2off[m] + (long long)A * nat) : nullptr;  // row A = column A
    for (int Bq = lane; Bq < nat; Bq += 32) {
      if (Bq == A) continue;
      const double v[3] = {xyz[3 * Bq] - xyz[3 * A], xyz[3 * Bq + 1] - xyz[3 * A + 1], xyz[3 * Bq + 2] - xyz[3 * A + 2]};
      double g1, f3, f5;
      if (ar) {
        const double* e = ar + 3LL * Bq;
        g1 = e[0]; f3 = e[1]; f5 = e[2];
      } else {
        const double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        g1 = 1.0 / sqrt(r2);
        aes_damp(P, rA, mrad[a0 + Bq], g1, f3, f5);
      }
      const double g3 = g1 * g1 * g1, g5 = g3 * g1 * g1;
      const double qb = qat_out[a0 + Bq];
      const double* db = dpat_out + 3 * (a0 + Bq);
      const double vdb = v[0] * db[0] + v[1] * db[1] + v[2] * db[2];
      double tc[6];
      tcomp(v, tc);
      for (int k = 0; k < 3; ++k) vd[k] += v[k] * g3 * f3 * qb + 0.5 * (g3 * db[k] - 3.0 * v[k] * vdb * g5) * f5;
      for (int c = 0; c < 6; ++c) vq[c] += tc[c] * g5 * f5 * qb;
    }
    for (int k = 0; k < 3; ++k) vd[k] = warp_sum(vd[k]);
    for (int c = 0; c < 6; ++c) vq[c] = warp_sum(vq[c]);
    if (lane == 0) {
      const SpeciesParam& sp = P.sp[B.id[a0 + A]];
      double dd = 0.0, qq = 0.0;
      for (int k = 0; k < 3; ++k) { ea += dA[k] * vd[k]; dd += dA[k] * dA[k]; }
      for (int c = 0; c < 6; ++c) { ea += qA[c] * vq[c]; qq += qA[c] * qA[c] * kMpScale[c]; }
      ea += sp.dkernel * dd + sp.qkernel * qq;
    }
  }
  const double e_es2 = block_sum(e2, red);
  const double e_es3 = block_sum(e3, red);
  const double e_aes2 = block_sum(ea, red);
  // mixer diff: dq = [qsh, dpat, qpat]_out - q_in
  const int mo = B.mixoff[m], ndim = nsh + 9 * nat;
  double err = 0.0;
  for (int i = tid; i < ndim; i += nt) {
    if (!TB_GUARD(11, mo + i, B.mixoff[m], B.mixoff[m + 1])) continue;
    double out;
    if (i < nsh) out = qsh_out[s0 + i];
    else if (i < nsh + 3 * nat) out = dpat_out[3 * a0 + (i - nsh)];
    else out = qpat_out[6 * a0 + (i - nsh - 3 * nat)];
    const double x = out - q_in[mo + i];
    dq[mo + i] = x;
    err += x * x;
  }
  err = block_sum(err, red);
  if (tid == 0) {
    const double elast = S.eelec[m], prev_error = S.scf_error[m];
    const double eelec = e_band + S.e_ts[m] + e_es2 + e_aes2 + e_es3;
    const double error = sqrt(err / ndim);
    S.eelec[m] = eelec;
    S.e_band[m] = e_band;
    S.e_es2[m] = e_es2;
    S.e_aes2[m] = e_aes2;
    S.e_es3[m] = e_es3;
    S.scf_error[m] = error;
    const int it = S.iscf[m] + 1;
    S.iscf[m] = it;
    bool conv = fabs(eelec - elast) < econv && error < pconv;
    if (S.phase) {
      // mixed-precision form: the mixed phase ends at the loosened test, when
      // its charge error stops falling (less than halved from the previous
      // iteration after the third: the FP32 eigenpairs no longer improve the
      // point), or after half the iteration budget; the mixer restarts from
      // the current point, then at least two FP64 iterations run and the full
      // test decides
      if (S.phase[m] == 0) {
        if ((fabs(eelec - elast) < econv_lo && error < pconv_lo) || 2 * it >= max_iter ||
            (it >= 3 && error > 0.5 * prev_error)) {
          S.phase[m] = 1;
          S.mix_iter[m] = 0;
        }
        conv = false;
      } else if (++S.n64[m] < 2) {
        conv = false;
      }
    }
    if (conv) {
      S.active[m] = 0;
    } else if (it >= max_iter) {
      S.active[m] = 0;
      S.status[m] = kStScfNotConverged;
    }
    if (!S.active[m]) atomicSub(S.n_active, 1);
  }
  // molecular dipole sum_A q_A R_A + mu_A (deterministic fixed-order sum)
  for (int k = 0; k < 3; ++k) {
    double dsum = 0.0;
    for (int a = tid; a < nat; a += nt) dsum += qat_out[a0 + a] * xyz[3 * a + k] + dpat_out[3 * (a0 + a) + k];
    dsum = block_sum(dsum, red);
    if (tid == 0) S.dipole[3 * m + k] = dsum;
  }
}

// ------------------------------------------------------------ Broyden
// Modified Broyden mixing (D. D. Johnson, PRB 38, 12807 (1988)); the update
// step `next` is missing from the reference (D19), set/diff follow
// src/scf/broyden.cu:47-72.  Runs at the start of every iteration after the
// first and leaves the new input moments in q_in.
__global__ void k_mix_next(DevBatch B, double* __restrict__ q_in, const double* __restrict__ dq,
                           double* __restrict__ dqlast, double* __restrict__ qlast, double* __restrict__ df,
                           double* __restrict__ u, double* __restrict__ amat, double* __restrict__ omega, int memory,
                           double damp, MolState S) {
  const int m = blockIdx.x;
  if (!S.active[m] || S.iscf[m] == 0) return;
  const int nat = B.aoff[m + 1] - B.aoff[m], nsh = B.soff[m + 1] - B.soff[m];
  const int n = nsh + 9 * nat, mo = B.mixoff[m];
  const long long ho = (long long)mo * memory;  // history slab of this structure
  double* q = q_in + mo;
  const double* d = dq + mo;
  double* dl = dqlast + mo;
  double* ql = qlast + mo;
  double* DF = df + ho;
  double* U = u + ho;
  double* a = amat + (long long)m * memory * memory;
  double* om = omega + (long long)m * memory;
  __shared__ double red[32];
  __shared__ double cvec[64], gvec[64], M[64 * 64];
  __shared__ int slot[64];
  __shared__ double sh_inv;
  __shared__ int sh_ok;
  const int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, wid = tid >> 5, nw = nt >> 5;
  const int iter = S.mix_iter[m] + 1;
  if (iter == 1) {
    for (int i = tid; i < n; i += nt) { dl[i] = d[i]; ql[i] = q[i]; q[i] += damp * d[i]; }
    if (tid == 0) S.mix_iter[m] = iter;
    return;
  }
  const double omega0 = 0.01, minw = 1.0, maxw = 100000.0, wfac = 0.01;
  const int itn = iter - 1;
  const int s = (itn - 1) % memory;
  const int nh = min(itn, memory);
  double p1 = 0.0, p2 = 0.0;
  for (int i = tid; i < n; i += nt) {
    const double x = d[i] - dl[i];
    DF[(long long)s * n + i] = x;
    p1 += d[i] * d[i];
    p2 += x * x;
  }
  const double nrm = sqrt(block_sum(p1, red));
  const double dn = block_sum(p2, red);
  if (tid == 0) {
    double w = nrm > wfac / maxw ? wfac / nrm : maxw;
    if (w < minw) w = minw;
    om[s] = w;
    sh_inv = 1.0 / fmax(sqrt(dn), 2.220446049250313e-16);
  }
  __syncthreads();
  const double inv = sh_inv;
  for (int i = tid; i < n; i += nt) DF[(long long)s * n + i] *= inv;
  if (tid < nh) slot[tid] = (itn - nh + tid) % memory;
  __syncthreads();
  // a(t, s) = df_t . df_s and c_t = w_t df_t . dq (one warp per history entry)
  for (int h = wid; h < nh; h += nw) {
    const int t = slot[h];
    double ad = 0.0, cd = 0.0;
    for (int i = lane; i < n; i += 32) {
      const double x = DF[(long long)t * n + i];
      ad += x * DF[(long long)s * n + i];
      cd += x * d[i];
    }
    ad = warp_sum(ad);
    cd = warp_sum(cd);
    if (lane == 0) {
      a[t * memory + s] = ad;
      a[s * memory + t] = ad;
      cvec[h] = om[t] * cd;
    }
  }
  __syncthreads();
  if (tid == 0) {
    for (int h = 0; h < nh; ++h)
      for (int k = 0; k < nh; ++k)
        M[h * nh + k] = om[slot[h]] * om[slot[k]] * a[slot[h] * memory + slot[k]] + (h == k ? omega0 * omega0 : 0.0);
    for (int h = 0; h < nh; ++h) gvec[h] = cvec[h];
    int ok = 1;
    for (int col = 0; col < nh && ok; ++col) {
      int piv = col;
      for (int r = col + 1; r < nh; ++r)
        if (fabs(M[r * nh + col]) > fabs(M[piv * nh + col])) piv = r;
      if (M[piv * nh + col] == 0.0) { ok = 0; break; }
      if (piv != col) {
        for (int k = 0; k < nh; ++k) { const double tmp = M[col * nh + k]; M[col * nh + k] = M[piv * nh + k]; M[piv * nh + k] = tmp; }
        const double tmp = gvec[col]; gvec[col] = gvec[piv]; gvec[piv] = tmp;
      }
      for (int r = col + 1; r < nh; ++r) {
        const double f = M[r * nh + col] / M[col * nh + col];
        for (int k = col; k < nh; ++k) M[r * nh + k] -= f * M[col * nh + k];
        gvec[r] -= f * gvec[col];
      }
    }
    if (ok)
      for (int r = nh - 1; r >= 0; --r) {
        double t = gvec[r];
        for (int k = r + 1; k < nh; ++k) t -= M[r * nh + k] * gvec[k];
        gvec[r] = t / M[r * nh + r];
      }
    for (int h = 0; h < nh; ++h) cvec[h] = om[slot[h]] * gvec[h];  // w_h * gamma_h
    sh_ok = ok;
  }
  __syncthreads();
  if (!sh_ok) {
    if (tid == 0) { S.status[m] = kStScfNotConverged; S.active[m] = 0; atomicSub(S.n_active, 1); }
    return;
  }
  for (int i = tid; i < n; i += nt) {
    U[(long long)s * n + i] = damp * DF[(long long)s * n + i] + inv * (q[i] - ql[i]);
  }
  __syncthreads();
  for (int i = tid; i < n; i += nt) {
    const double qi = q[i];
    dl[i] = d[i];
    ql[i] = qi;
    double v = qi + damp * d[i];
    for (int h = 0; h < nh; ++h) v -= cvec[h] * U[(long long)slot[h] * n + i];
    q[i] = v;
  }
  if (tid == 0) S.mix_iter[m] = iter;
}

TB_OOB_EXPORT(oob_scf)

// ------------------------------------------------------------ gradient
// Nuclear gradient and virial (the gradient/sigma outputs of xtb_singlepoint,
// src/xtb.cu:195-196) of the converged structures with flag[m] set, from the
// last iteration's density P, coefficients C and orbital energies:
//   dE/dR = dE_rep/dR + [shell-pair terms: P dH0 - W dS and the Mulliken
//           moments through dS, dD, dQ, k_grad_pairs_t]
//         + dE_ES2/dR + dE_AES2/dR at fixed moments + (dE/dCN) dCN/dR,
// W = C diag(f e) C^T.  Repulsion: get_repulsion_derivs (src/xtb.cu:62-91,
// quoted); the other terms differentiate the energy expression of the
// potential and energy kernels above.  Every atom sums its pair terms in a
// fixed order (no atomics): a structure's gradient is the same alone and in
// any batch.

// f e (energy-weighted occupations) and the final moments in the mixer layout
// [qsh, dpat, qpat] (input of k_potential: the potentials dE/dmoment).
__global__ void k_grad_prep(DevBatch B, const int* __restrict__ flag, const double* __restrict__ focc,
                            const double* __restrict__ w, const double* __restrict__ qsh,
                            const double* __restrict__ dpat, const double* __restrict__ qpat, double* __restrict__ fe,
                            double* __restrict__ qv) {
  const int m = blockIdx.x;
  if (!flag[m]) return;
  const int o0 = B.ooff[m], n = B.ooff[m + 1] - o0;
  const int a0 = B.aoff[m], nat = B.aoff[m + 1] - a0, s0 = B.soff[m], nsh = B.soff[m + 1] - s0;
  const int mo = B.mixoff[m];
  for (int i = threadIdx.x; i < n; i += blockDim.x) fe[o0 + i] = focc[o0 + i] * w[o0 + i];
  for (int i = threadIdx.x; i < nsh; i += blockDim.x) qv[mo + i] = qsh[s0 + i];
  for (int i = threadIdx.x; i < 3 * nat; i += blockDim.x) qv[mo + nsh + i] = dpat[3 * a0 + i];
  for (int i = threadIdx.x; i < 6 * nat; i += blockDim.x) qv[mo + nsh + 3 * nat + i] = qpat[6 * a0 + i];
}

// Sum of a neighbour pair's shell-pair items, in shell-pair order, into the
// structure's atom-pair table G[i][j] (i > j).
__global__ void k_grad_pair_reduce(DevBatch B, const int* __restrict__ npair, const int* __restrict__ pair_i,
                                   const int* __restrict__ pair_j, const int* __restrict__ flag, int maxsp,
                                   long long pair_cap, const double* __restrict__ item, double* __restrict__ G) {
  for (long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x; p < pair_cap;
       p += (long long)gridDim.x * blockDim.x) {
    int lo = 0, hi = B.nmol;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (B.poff[mid] <= p) lo = mid; else hi = mid;
    }
    const int m = lo;
    if (!flag[m] || p - B.poff[m] >= npair[m]) continue;
    const int nat = B.aoff[m + 1] - B.aoff[m];
    double g[3] = {0.0, 0.0, 0.0};
    for (int sp = 0; sp < maxsp; ++sp)
      for (int x = 0; x < 3; ++x) g[x] += item[3 * (p * maxsp + sp) + x];
    const long long gi = B.a2off[m] + (long long)pair_i[p] * nat + pair_j[p];
    if (!TB_GUARD(14, gi, B.a2off[m], B.a2off[m + 1])) continue;
    double* out = G + 3 * gi;
    for (int x = 0; x < 3; ++x) out[x] = g[x];
  }
}

// AES2 energy of the ordered pair (source i, multipole atom j), v = R_i - R_j,
// and its derivatives along v and with respect to the damping-radius sum
// (rr = (rad_i + rad_j) / (2 r)):
//   e = q_i (mu_j.v) g3 f3 + 1/2 [(mu_j.mu_i) g3 - 3 (mu_j.v)(mu_i.v) g5] f5 + q_i (Th_j : tc(v)) g5 f5.
__device__ inline void aes_pair_grad(const DevParams& P, const double* v, double radi, double radj, double qi,
                                     const double* mi, const double* mj, const double* tj, double* de,
                                     double* de_drad) {
  const double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2], r1 = sqrt(r2);
  const double g1 = 1.0 / r1, g3 = g1 * g1 * g1, g5 = g3 * g1 * g1, g7 = g5 * g1 * g1;
  const double rr = 0.5 * (radi + radj) * g1, lr = log(rr);
  const double t3 = 6.0 * exp(P.kdmp3 * lr), t5 = 6.0 * exp(P.kdmp5 * lr);
  const double f3 = 1.0 / (1.0 + t3), f5 = 1.0 / (1.0 + t5);
  const double df3 = -P.kdmp3 * t3 / rr * f3 * f3, df5 = -P.kdmp5 * t5 / rr * f5 * f5;
  const double mjv = mj[0] * v[0] + mj[1] * v[1] + mj[2] * v[2];
  const double miv = mi[0] * v[0] + mi[1] * v[1] + mi[2] * v[2];
  const double mm = mj[0] * mi[0] + mj[1] * mi[1] + mj[2] * mi[2];
  const double tv = tj[0] * v[0] * v[0] + 2.0 * tj[1] * v[0] * v[1] + tj[2] * v[1] * v[1] +
                    2.0 * tj[3] * v[0] * v[2] + 2.0 * tj[4] * v[1] * v[2] + tj[5] * v[2] * v[2];
  const double dtv[3] = {2.0 * tj[0] * v[0] + 2.0 * tj[1] * v[1] + 2.0 * tj[3] * v[2],
                         2.0 * tj[1] * v[0] + 2.0 * tj[2] * v[1] + 2.0 * tj[4] * v[2],
                         2.0 * tj[3] * v[0] + 2.0 * tj[4] * v[1] + 2.0 * tj[5] * v[2]};
  const double a_nof = qi * mjv * g3, b_nof = 0.5 * (mm * g3 - 3.0 * mjv * miv * g5), c_nof = qi * tv * g5;
  for (int k = 0; k < 3; ++k) {
    const double drr = -rr * v[k] / r2;
    const double dg3 = -3.0 * g5 * v[k], dg5 = -5.0 * g7 * v[k];
    const double da = qi * (mj[k] * g3 + mjv * dg3);
    const double db = 0.5 * (mm * dg3 - 3.0 * (mj[k] * miv + mjv * mi[k]) * g5 - 3.0 * mjv * miv * dg5);
    const double dc = qi * (dtv[k] * g5 + tv * dg5);
    de[k] = da * f3 + a_nof * df3 * drr + db * f5 + b_nof * df5 * drr + dc * f5 + c_nof * df5 * drr;
  }
  *de_drad = (a_nof * df3 + (b_nof + c_nof) * df5) * g1 * 0.5;
}

// dE/dCN per atom: its shells' dE/dse (the on-site diagonal of P plus the
// shell-pair table of k_grad_pairs_t) times dse/dCN = -kcn, and dE/d(damping
// radius) over all AES2 pairs times dmrad/dCN (get_mrad, src/coulomb.cu:387-398).
__global__ void k_grad_cn(DevParams P, DevBatch B, const int* __restrict__ flag, const double* __restrict__ Pm,
                          const double* __restrict__ ese_tab, const double* __restrict__ cn,
                          const double* __restrict__ mrad, const double* __restrict__ qat,
                          const double* __restrict__ dpat, const double* __restrict__ qpat,
                          double* __restrict__ dEdcn) {
  const int m = blockIdx.x;
  if (!flag[m]) return;
  const int a0 = B.aoff[m], nat = B.aoff[m + 1] - a0, s0 = B.soff[m], nsh = B.soff[m + 1] - s0;
  const int o0 = B.ooff[m], n = B.ooff[m + 1] - o0;
  const long long mo = B.moff[m], so = B.s2off[m];
  const int A = blockIdx.y * blockDim.x + threadIdx.x;
  if (A >= nat) return;
  const SpeciesParam& sa = P.sp[B.id[a0 + A]];
  const int isa = B.at_ish[a0 + A];
  double d = 0.0;
  for (int s = 0; s < sa.nsh; ++s) {
    const int sh = isa + s;
    double dse = 0.0;
    const int i0 = B.sh_iao[s0 + sh], na = msao(P.sh[sa.sh0 + s].ang);
    for (int x = 0; x < na; ++x) dse += Pm[mo + (long long)(i0 + x) * n + i0 + x];
    for (int b = 0; b < nsh; ++b) dse += ese_tab[so + (long long)sh * nsh + b];
    d -= P.sh[sa.sh0 + s].kcn * dse;
  }
  const double* xyz = B.xyz + 3 * a0;
  double drad = 0.0;
  for (int Bq = 0; Bq < nat; ++Bq) {
    if (Bq == A) continue;
    double de[3], dr1, dr2;
    const double v1[3] = {xyz[3 * A] - xyz[3 * Bq], xyz[3 * A + 1] - xyz[3 * Bq + 1], xyz[3 * A + 2] - xyz[3 * Bq + 2]};
    const double v2[3] = {-v1[0], -v1[1], -v1[2]};
    aes_pair_grad(P, v1, mrad[a0 + A], mrad[a0 + Bq], qat[a0 + A], dpat + 3 * (a0 + A), dpat + 3 * (a0 + Bq),
                  qpat + 6 * (a0 + Bq), de, &dr1);  // source A, multipoles on Bq
    aes_pair_grad(P, v2, mrad[a0 + Bq], mrad[a0 + A], qat[a0 + Bq], dpat + 3 * (a0 + Bq), dpat + 3 * (a0 + A),
                  qpat + 6 * (a0 + A), de, &dr2);  // source Bq, multipoles on A
    drad += dr1 + dr2;
  }
  const double t1 = exp(-P.mp_kexp * (cn[a0 + A] - sa.mp_vcn - P.mp_shift));
  d += drad * (P.mp_rmax - sa.mp_rad) * P.mp_kexp * t1 / ((1.0 + t1) * (1.0 + t1));
  dEdcn[a0 + A] = d;
}

// Gradient of atom A: every pair term with A, summed over the other atoms in
// order -- the shell-pair table G (antisymmetric), repulsion (quoted
// get_repulsion_derivs), ES2 at fixed shell charges, AES2 at fixed moments
// (A as source and as multipole atom), and the coordination-number chain.
__global__ void k_grad_atoms(DevParams P, DevBatch B, const int* __restrict__ flag, const double* __restrict__ G,
                             const double* __restrict__ dEdcn, const double* __restrict__ mrad,
                             const double* __restrict__ qsh, const double* __restrict__ qat,
                             const double* __restrict__ dpat, const double* __restrict__ qpat,
                             double* __restrict__ grad) {
  const int m = blockIdx.x;
  if (!flag[m]) return;
  const int a0 = B.aoff[m], nat = B.aoff[m + 1] - a0, s0 = B.soff[m];
  const int A = blockIdx.y * blockDim.x + threadIdx.x;
  if (A >= nat) return;
  const long long ao = B.a2off[m];
  const double* xyz = B.xyz + 3 * a0;
  const SpeciesParam& sa = P.sp[B.id[a0 + A]];
  const int isa = s0 + B.at_ish[a0 + A];
  const double ka = 10.0, kb = 20.0, rshift = 2.0;
  const double cn2 = P.cn_cutoff * P.cn_cutoff, rep2 = P.rep_cutoff * P.rep_cutoff;
  double g[3] = {0.0, 0.0, 0.0};
  for (int Bq = 0; Bq < nat; ++Bq) {
    if (Bq == A) continue;
    const double v[3] = {xyz[3 * A] - xyz[3 * Bq], xyz[3 * A + 1] - xyz[3 * Bq + 1], xyz[3 * A + 2] - xyz[3 * Bq + 2]};
    const double r2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
    if (r2 < 1.0e-12) continue;
    const double r1 = sqrt(r2);
    const SpeciesParam& sb = P.sp[B.id[a0 + Bq]];
    // shell-pair terms (H0, overlap, Mulliken moments)
    if (Bq < A) {
      const double* e = G + 3 * (ao + (long long)A * nat + Bq);
      for (int k = 0; k < 3; ++k) g[k] += e[k];
    } else {
      const double* e = G + 3 * (ao + (long long)Bq * nat + A);
      for (int k = 0; k < 3; ++k) g[k] -= e[k];
    }
    double s = 0.0;  // coefficient of v / r1
    // repulsion
    if (r2 <= rep2) {
      const double alpha = sqrt(sa.rep_alpha * sb.rep_alpha), zeff = sa.rep_zeff * sb.rep_zeff;
      const double kexp = (sa.z <= 2 && sb.z <= 2) ? P.rep_kexp_light : P.rep_kexp;
      const double r1k = pow(r1, kexp), r1r = pow(r1, P.rep_rexp);
      const double dE = zeff * exp(-alpha * r1k) / r1r;
      s += -(alpha * r1k * kexp + P.rep_rexp) * dE / r1;
    }
    // ES2: q_a q_b dgamma/dr over the shells of A and Bq
    {
      const int isb = s0 + B.at_ish[a0 + Bq];
      for (int x = 0; x < sa.nsh; ++x)
        for (int y = 0; y < sb.nsh; ++y) {
          const double gam = 0.5 * (P.sh[sa.sh0 + x].hubbard + P.sh[sb.sh0 + y].hubbard);
          double dg;
          if (P.gexp == 2.0) {
            const double b2 = r2 + 1.0 / (gam * gam);
            dg = -r1 / (b2 * sqrt(b2));
          } else {
            const double base = pow(r1, P.gexp) + pow(gam, -P.gexp);
            dg = -pow(r1, P.gexp - 1.0) * pow(base, -1.0 / P.gexp - 1.0);
          }
          s += qsh[isa + x] * qsh[isb + y] * dg;
        }
    }
    // coordination-number chain
    if (r2 <= cn2) {
      const double rc = sa.rcov + sb.rcov;
      const double ea = 1.0 / (1.0 + exp(-ka * (rc / r1 - 1.0)));
      const double eb = 1.0 / (1.0 + exp(-kb * ((rc + rshift) / r1 - 1.0)));
      const double dea = -ea * (1.0 - ea) * ka * rc / r2, deb = -eb * (1.0 - eb) * kb * (rc + rshift) / r2;
      s += (dea * eb + ea * deb) * (dEdcn[a0 + A] + dEdcn[a0 + Bq]);
    }
    for (int k = 0; k < 3; ++k) g[k] += s * v[k] / r1;
    // AES2 at fixed moments: A as source (+), A as multipole atom (-, v = R_Bq - R_A)
    double de[3], dr;
    aes_pair_grad(P, v, mrad[a0 + A], mrad[a0 + Bq], qat[a0 + A], dpat + 3 * (a0 + A), dpat + 3 * (a0 + Bq),
                  qpat + 6 * (a0 + Bq), de, &dr);
    for (int k = 0; k < 3; ++k) g[k] += de[k];
    const double vm[3] = {-v[0], -v[1], -v[2]};
    aes_pair_grad(P, vm, mrad[a0 + Bq], mrad[a0 + A], qat[a0 + Bq], dpat + 3 * (a0 + Bq), dpat + 3 * (a0 + A),
                  qpat + 6 * (a0 + A), de, &dr);
    for (int k = 0; k < 3; ++k) g[k] -= de[k];
  }
  for (int k = 0; k < 3; ++k) grad[3 * (a0 + A) + k] = g[k];
}

// Virial sigma[3][3] = sum_A g_A R_A^T per structure (fixed-order block sums).
__global__ void k_grad_sigma(DevBatch B, const int* __restrict__ flag, const double* __restrict__ grad,
                             double* __restrict__ sigma) {
  const int m = blockIdx.x;
  if (!flag[m]) return;
  __shared__ double red[32];
  const int a0 = B.aoff[m], nat = B.aoff[m + 1] - a0;
  for (int ab = 0; ab < 9; ++ab) {
    const int a = ab / 3, b = ab % 3;
    double s = 0.0;
    for (int i = threadIdx.x; i < nat; i += blockDim.x) s += grad[3 * (a0 + i) + a] * B.xyz[3 * (a0 + i) + b];
    s = block_sum(s, red);
    if (threadIdx.x == 0) sigma[9 * m + ab] = s;
    __syncthreads();
  }
}

}  // namespace tb
