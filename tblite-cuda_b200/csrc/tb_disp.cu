// D4 dispersion: dispersion_get_engrad (reference src/xtb.cu:274-277, a TODO
// there; tblite calls the dftd4 library, which the reference does not vendor).
// The published D4 model (E. Caldeweyher et al., J. Chem. Phys. 150, 154122
// (2019)) on the parameter file's D4 block, evaluated at the neutral reference
// charges -- the reference's call site comes before the SCF, so no charges
// exist there and the charge scaling of the reference polarizabilities is the
// identity:
//  * CN_A = sum_B f_EN(A, B) (1 + erf(-k0 (r_AB / Rc_AB - 1))) / 2, Rc_AB =
//    k1 (rcov_A + rcov_B), f_EN = k4 exp(-(|EN_A - EN_B| + k5)^2 / k6), r <= d4_cn_cut;
//  * weights W_A^i = exp(-wf (CN_A - CN_i)^2) / sum_j exp(-wf (CN_A - CN_j)^2);
//  * C6_AB = sum_ij W_A^i W_B^j C6ref_ij (Casimir-Polder reference C6, built
//    per calculator), C8 = C6 q_AB, q_AB = 3 sqrt(r4r2_A r4r2_B), R_AB = a1 sqrt(q_AB) + a2;
//  * two-body, r <= d4_pair_cut: E_AB = -C6 (s6 / (r^6 + R^6) + s8 q / (r^8 + R^8));
//  * three-body (Axilrod-Teller-Muto), all three distances <= d4_atm_cut:
//    E_ABC = s9 sqrt(C6_AB C6_BC C6_CA) (1 + 3 P / (8 u v w)) f / (r_AB r_BC r_CA)^3,
//    u, v, w the squared distances, P = (u+v-w)(u+w-v)(v+w-u), f = 1 / (1 + 6 t^(alp/3)),
//    t = R_AB R_BC R_CA / (r_AB r_BC r_CA).
// Each atom sums its own share of the pair and triple energies and its own
// gradient terms over the other atoms in a fixed order (no atomics), so a
// structure gives the same bits alone and in any batch.  Kernels, run once per
// batch in the setup: k_d4_weights (CN, W, dW/dCN; a thread per atom),
// k_d4_pairs (two-body; a thread per atom), k_d4_atm (three-body; a warp per
// atom), k_d4_cnchain (dE/dCN dCN/dR; a thread per atom), k_d4_energy (per
// structure).
#include <cuda_runtime.h>

#include "tb_common.cuh"
#include "tb_kernels.h"

namespace tb {

namespace {

constexpr int R4 = kD4MaxRef;

__device__ inline double d4_count(const DevParams& P, const SpeciesParam& a, const SpeciesParam& b, double r,
                                  double* dcdr) {
  const double rc = P.d4_k1 * (a.rcov + b.rcov);
  const double x = fabs(a.en - b.en) + P.d4_k5;
  const double den = P.d4_k4 * exp(-x * x / P.d4_k6);
  const double y = P.d4_k0 * (r / rc - 1.0);
  if (dcdr) *dcdr = den * (-1.0 / sqrt(M_PI)) * exp(-y * y) * P.d4_k0 / rc;
  return den * 0.5 * (1.0 + erf(-y));
}

// C6 of atoms ia, ib (batch indices) and its derivatives in CN_a, CN_b
__device__ inline double d4_c6(const DevParams& P, const SpeciesParam& sa, const SpeciesParam& sb, int za, int zb,
                               const double* W, const double* dW, int ia, int ib, double* dca, double* dcb) {
  const double* t = P.d4_c6ref + ((size_t)za * P.nsp + zb) * R4 * R4;
  double v = 0.0, da = 0.0, db = 0.0;
  for (int i = 0; i < sa.d4_nref; ++i) {
    const double wa = W[ia * R4 + i], dwa = dW[ia * R4 + i];
    for (int j = 0; j < sb.d4_nref; ++j) {
      const double r = t[i * R4 + j];
      v += wa * W[ib * R4 + j] * r;
      da += dwa * W[ib * R4 + j] * r;
      db += wa * dW[ib * R4 + j] * r;
    }
  }
  *dca = da;
  *dcb = db;
  return v;
}

__device__ inline double d4_qpair(const SpeciesParam& a, const SpeciesParam& b) {
  return 3.0 * sqrt(a.d4_r4r2 * b.d4_r4r2);
}

}  // namespace

// CN_A, W_A^i and dW_A^i / dCN_A for every atom of the batch
__global__ void k_d4_weights(DevParams P, DevBatch B, double* __restrict__ cn, double* __restrict__ W,
                             double* __restrict__ dW) {
  const int A = blockIdx.x * blockDim.x + threadIdx.x;
  if (A >= B.nat_tot) return;
  const int m = B.at_mol[A], a0 = B.aoff[m], nat = B.aoff[m + 1] - a0;
  const SpeciesParam& sa = P.sp[B.id[A]];
  double c = 0.0;
  for (int b = 0; b < nat; ++b) {
    const int Bi = a0 + b;
    if (Bi == A) continue;
    const double v0 = B.xyz[3 * A] - B.xyz[3 * Bi], v1 = B.xyz[3 * A + 1] - B.xyz[3 * Bi + 1],
                 v2 = B.xyz[3 * A + 2] - B.xyz[3 * Bi + 2];
    const double r = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
    if (r > P.d4_cn_cut || r < 1.0e-6) continue;
    c += d4_count(P, sa, P.sp[B.id[Bi]], r, nullptr);
  }
  cn[A] = c;
  double gmax = -1e300;
  for (int i = 0; i < sa.d4_nref; ++i) gmax = fmax(gmax, -P.d4_wf * (c - sa.d4_cn[i]) * (c - sa.d4_cn[i]));
  double ex[R4], sum = 0.0;
  for (int i = 0; i < sa.d4_nref; ++i) {
    ex[i] = exp(-P.d4_wf * (c - sa.d4_cn[i]) * (c - sa.d4_cn[i]) - gmax);
    sum += ex[i];
  }
  double gp = 0.0;
  for (int i = 0; i < sa.d4_nref; ++i) gp += ex[i] / sum * (-2.0 * P.d4_wf * (c - sa.d4_cn[i]));
  for (int i = 0; i < R4; ++i) {
    const double w = i < sa.d4_nref ? ex[i] / sum : 0.0;
    W[A * R4 + i] = w;
    dW[A * R4 + i] = i < sa.d4_nref ? w * (-2.0 * P.d4_wf * (c - sa.d4_cn[i]) - gp) : 0.0;
  }
}

// two-body: e_at[A] = half of A's pair energies, dEdcn[A] and the explicit
// gradient g[A] of A's pairs
__global__ void k_d4_pairs(DevParams P, DevBatch B, const double* __restrict__ W, const double* __restrict__ dW,
                           double* __restrict__ e_at, double* __restrict__ dEdcn, double* __restrict__ g) {
  const int A = blockIdx.x * blockDim.x + threadIdx.x;
  if (A >= B.nat_tot) return;
  const int m = B.at_mol[A], a0 = B.aoff[m], nat = B.aoff[m + 1] - a0;
  const int za = B.id[A];
  const SpeciesParam& sa = P.sp[za];
  double e = 0.0, de = 0.0, g0 = 0.0, g1 = 0.0, g2 = 0.0;
  for (int b = 0; b < nat; ++b) {
    const int Bi = a0 + b;
    if (Bi == A) continue;
    const double v0 = B.xyz[3 * A] - B.xyz[3 * Bi], v1 = B.xyz[3 * A + 1] - B.xyz[3 * Bi + 1],
                 v2 = B.xyz[3 * A + 2] - B.xyz[3 * Bi + 2];
    const double r = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
    if (r > P.d4_pair_cut || r < 1.0e-6) continue;
    const int zb = B.id[Bi];
    const SpeciesParam& sb = P.sp[zb];
    double dca, dcb;
    const double C6 = d4_c6(P, sa, sb, za, zb, W, dW, A, Bi, &dca, &dcb);
    const double q = d4_qpair(sa, sb), Rab = P.d4_a1 * sqrt(q) + P.d4_a2;
    const double r2 = r * r, r6 = r2 * r2 * r2, r8 = r6 * r2, R2 = Rab * Rab, R6 = R2 * R2 * R2, R8 = R6 * R2;
    const double h = P.d4_s6 / (r6 + R6) + P.d4_s8 * q / (r8 + R8);
    const double dh = -P.d4_s6 * 6.0 * r6 / r / ((r6 + R6) * (r6 + R6)) -
                      P.d4_s8 * q * 8.0 * r8 / r / ((r8 + R8) * (r8 + R8));
    e += 0.5 * (-C6 * h);
    de += -h * dca;
    const double f = -C6 * dh / r;
    g0 += f * v0; g1 += f * v1; g2 += f * v2;
  }
  e_at[A] = e;
  dEdcn[A] = de;
  g[3 * A] = g0; g[3 * A + 1] = g1; g[3 * A + 2] = g2;
}

// three-body: a warp per atom A; lane l takes the atoms B = l, l + 32, ... of
// A's structure and every C > B (B, C != A); each triple's energy goes one
// third to each atom, and A adds its own dE/dCN_A and gradient terms.  Lane
// partials are added by a fixed shuffle tree.
__global__ void k_d4_atm(DevParams P, DevBatch B, const double* __restrict__ W, const double* __restrict__ dW,
                         double* __restrict__ e_at, double* __restrict__ dEdcn, double* __restrict__ g) {
  const int A = (int)((blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5);
  const int lane = threadIdx.x & 31;
  if (A >= B.nat_tot || P.d4_s9 == 0.0) return;
  const int m = B.at_mol[A], a0 = B.aoff[m], nat = B.aoff[m + 1] - a0;
  const int za = B.id[A];
  const SpeciesParam& sa = P.sp[za];
  const double xa = B.xyz[3 * A], ya = B.xyz[3 * A + 1], zaa = B.xyz[3 * A + 2];
  const double cut = P.d4_atm_cut, p = P.d4_alp / 3.0;
  double e = 0.0, de = 0.0, g0 = 0.0, g1 = 0.0, g2 = 0.0;
  for (int b = lane; b < nat; b += 32) {
    const int Bi = a0 + b;
    if (Bi == A) continue;
    const double vab0 = xa - B.xyz[3 * Bi], vab1 = ya - B.xyz[3 * Bi + 1], vab2 = zaa - B.xyz[3 * Bi + 2];
    const double rab = sqrt(vab0 * vab0 + vab1 * vab1 + vab2 * vab2);
    if (rab > cut || rab < 1.0e-6) continue;
    const int zb = B.id[Bi];
    const SpeciesParam& sb = P.sp[zb];
    double dab_a, dab_b;
    const double cab = d4_c6(P, sa, sb, za, zb, W, dW, A, Bi, &dab_a, &dab_b);
    const double Rab = P.d4_a1 * sqrt(d4_qpair(sa, sb)) + P.d4_a2;
    for (int cc = b + 1; cc < nat; ++cc) {
      const int Ci = a0 + cc;
      if (Ci == A) continue;
      const double vca0 = B.xyz[3 * Ci] - xa, vca1 = B.xyz[3 * Ci + 1] - ya, vca2 = B.xyz[3 * Ci + 2] - zaa;
      const double rca = sqrt(vca0 * vca0 + vca1 * vca1 + vca2 * vca2);
      if (rca > cut || rca < 1.0e-6) continue;
      const double vbc0 = B.xyz[3 * Bi] - B.xyz[3 * Ci], vbc1 = B.xyz[3 * Bi + 1] - B.xyz[3 * Ci + 1],
                   vbc2 = B.xyz[3 * Bi + 2] - B.xyz[3 * Ci + 2];
      const double rbc = sqrt(vbc0 * vbc0 + vbc1 * vbc1 + vbc2 * vbc2);
      if (rbc > cut || rbc < 1.0e-6) continue;
      const int zc = B.id[Ci];
      const SpeciesParam& sc = P.sp[zc];
      double dbc_b, dbc_c, dca_c, dca_a;
      const double cbc = d4_c6(P, sb, sc, zb, zc, W, dW, Bi, Ci, &dbc_b, &dbc_c);
      const double cca = d4_c6(P, sc, sa, zc, za, W, dW, Ci, A, &dca_c, &dca_a);
      const double K = P.d4_s9 * sqrt(cab * cbc * cca);
      const double u = rab * rab, v = rbc * rbc, w = rca * rca;
      const double f1 = u + v - w, f2 = u + w - v, f3 = v + w - u;
      const double Pp = f1 * f2 * f3, uvw = u * v * w;
      const double ang = 1.0 + 3.0 * Pp / (8.0 * uvw);
      const double r3 = rab * rbc * rca, r9 = r3 * r3 * r3;
      const double Rbc = P.d4_a1 * sqrt(d4_qpair(sb, sc)) + P.d4_a2, Rca = P.d4_a1 * sqrt(d4_qpair(sc, sa)) + P.d4_a2;
      const double tp = pow(Rab * Rbc * Rca / r3, p);
      const double fd = 1.0 / (1.0 + 6.0 * tp);
      const double E = K * ang * fd / r9;
      e += E / 3.0;
      de += 0.5 * E * (dab_a / cab + dca_a / cca);
      // dE / dr_AB and dE / dr_CA (the distances that move with A)
      const double pre = 3.0 / (8.0 * uvw);
      const double dang_u = pre * ((f2 * f3 + f1 * f3 - f1 * f2) - Pp / u);
      const double dang_w = pre * ((-f2 * f3 + f1 * f3 + f1 * f2) - Pp / w);
      const double dfd = 6.0 * p * tp * fd * fd;
      const double dEab = K * ((dang_u * 2.0 * rab) * fd / r9 + ang * (dfd / rab) / r9 - 3.0 * ang * fd / (r9 * rab));
      const double dEca = K * ((dang_w * 2.0 * rca) * fd / r9 + ang * (dfd / rca) / r9 - 3.0 * ang * fd / (r9 * rca));
      // A's gradient: dE/dr_AB (R_A - R_B)/r_AB + dE/dr_CA (R_A - R_C)/r_CA
      g0 += dEab * vab0 / rab - dEca * vca0 / rca;
      g1 += dEab * vab1 / rab - dEca * vca1 / rca;
      g2 += dEab * vab2 / rab - dEca * vca2 / rca;
    }
  }
  e = warp_sum(e);
  de = warp_sum(de);
  g0 = warp_sum(g0);
  g1 = warp_sum(g1);
  g2 = warp_sum(g2);
  if (lane == 0) {
    e_at[A] += e;
    dEdcn[A] += de;
    g[3 * A] += g0; g[3 * A + 1] += g1; g[3 * A + 2] += g2;
  }
}

// coordination-number chain: g_A += sum_B (dE/dCN_A + dE/dCN_B) dcount_AB/dr (R_A - R_B)/r
__global__ void k_d4_cnchain(DevParams P, DevBatch B, const double* __restrict__ dEdcn, double* __restrict__ g) {
  const int A = blockIdx.x * blockDim.x + threadIdx.x;
  if (A >= B.nat_tot) return;
  const int m = B.at_mol[A], a0 = B.aoff[m], nat = B.aoff[m + 1] - a0;
  const SpeciesParam& sa = P.sp[B.id[A]];
  double g0 = 0.0, g1 = 0.0, g2 = 0.0;
  for (int b = 0; b < nat; ++b) {
    const int Bi = a0 + b;
    if (Bi == A) continue;
    const double v0 = B.xyz[3 * A] - B.xyz[3 * Bi], v1 = B.xyz[3 * A + 1] - B.xyz[3 * Bi + 1],
                 v2 = B.xyz[3 * A + 2] - B.xyz[3 * Bi + 2];
    const double r = sqrt(v0 * v0 + v1 * v1 + v2 * v2);
    if (r > P.d4_cn_cut || r < 1.0e-6) continue;
    double dcdr;
    d4_count(P, sa, P.sp[B.id[Bi]], r, &dcdr);
    const double f = (dEdcn[A] + dEdcn[Bi]) * dcdr / r;
    g0 += f * v0; g1 += f * v1; g2 += f * v2;
  }
  g[3 * A] += g0; g[3 * A + 1] += g1; g[3 * A + 2] += g2;
}

// per-structure dispersion energy: the atoms' shares in order
__global__ void k_d4_energy(DevBatch B, const double* __restrict__ e_at, double* __restrict__ e_disp) {
  const int m = blockIdx.x;
  if (threadIdx.x != 0) return;
  double s = 0.0;
  for (int a = B.aoff[m]; a < B.aoff[m + 1]; ++a) s += e_at[a];
  e_disp[m] = s;
}

// the dispersion gradient into the total gradient of the flagged structures
__global__ void k_d4_add_grad(DevBatch B, const int* __restrict__ flag, const double* __restrict__ gd,
                              double* __restrict__ grad) {
  const int A = blockIdx.x * blockDim.x + threadIdx.x;
  if (A >= B.nat_tot || !flag[B.at_mol[A]]) return;
  for (int k = 0; k < 3; ++k) grad[3 * A + k] += gd[3 * A + k];
}

cudaError_t launch_dispersion(const DevParams& P, const DevBatch& B, int nmol, double* cn, double* W, double* dW,
                              double* e_at, double* dEdcn, double* g, double* e_disp, cudaStream_t st) {
  const int na = B.nat_tot, t = 128;
  k_d4_weights<<<(na + t - 1) / t, t, 0, st>>>(P, B, cn, W, dW);
  k_d4_pairs<<<(na + t - 1) / t, t, 0, st>>>(P, B, W, dW, e_at, dEdcn, g);
  k_d4_atm<<<(int)(((long long)na * 32 + t - 1) / t), t, 0, st>>>(P, B, W, dW, e_at, dEdcn, g);
  k_d4_cnchain<<<(na + t - 1) / t, t, 0, st>>>(P, B, dEdcn, g);
  k_d4_energy<<<nmol, 32, 0, st>>>(B, e_at, e_disp);
  return cudaGetLastError();
}

}  // namespace tb
