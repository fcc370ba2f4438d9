// Setup kernels of the singlepoint (run once per structure batch): coordination
// numbers, multipole damping radii, self-energies, repulsion, the half
// neighbour list, and the overlap/dipole/quadrupole/H0 integral matrices.
//
// Layout: every structure of a batch owns contiguous slices of the packed
// atom/shell/AO vectors and an N x N slice (N = nao) of each matrix arena;
// D and Q are [3][N][N] / [6][N][N] planar per structure.
#include "tb_common.cuh"
#include "tb_kernels.h"

#include <algorithm>

namespace tb {

// ---------------------------------------------------------------- atoms
// GFN double-exponential counting function (published GFN2-xTB method; the
// reference calls exp_count without quoting it, src/coulomb.cu:220-222).
__device__ inline double exp_count(double k, double r, double r0) {
  return 1.0 / (1.0 + exp(-k * (r0 / r - 1.0)));
}

// One thread per atom: CN (ncoord_dexp, src/coulomb.cu:173-246), repulsion
// energy share (get_repulsion_derivs, src/xtb.cu:62-91), multipole damping
// radius (get_mrad, src/coulomb.cu:387-398) and shell self-energies
// (get_selfenergy, src/h0.cu:137-170).
__global__ void k_atoms(DevParams P, DevBatch B, double* __restrict__ cn, double* __restrict__ mrad,
                        double* __restrict__ erep, double* __restrict__ se) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  if (a >= B.nat_tot) return;
  const int m = B.at_mol[a];
  const int a0 = B.aoff[m], a1 = B.aoff[m + 1];
  const double xa = B.xyz[3 * a], ya = B.xyz[3 * a + 1], za = B.xyz[3 * a + 2];
  const SpeciesParam si = P.sp[B.id[a]];
  const double ka = 10.0, kb = 20.0, rshift = 2.0;
  const double cn2 = P.cn_cutoff * P.cn_cutoff, rep2 = P.rep_cutoff * P.rep_cutoff;
  double c = 0.0, e = 0.0;
  for (int b = a0; b < a1; ++b) {
    if (b == a) continue;
    const double dx = xa - B.xyz[3 * b], dy = ya - B.xyz[3 * b + 1], dz = za - B.xyz[3 * b + 2];
    const double r2 = dx * dx + dy * dy + dz * dz;
    if (r2 < 1.0e-12) continue;
    const SpeciesParam& sj = P.sp[B.id[b]];
    const double r1 = sqrt(r2);
    if (r2 <= cn2) {
      const double rc = si.rcov + sj.rcov;
      c += exp_count(ka, r1, rc) * exp_count(kb, r1, rc + rshift);
    }
    if (r2 <= rep2) {
      const double alpha = sqrt(si.rep_alpha * sj.rep_alpha);
      const double zeff = si.rep_zeff * sj.rep_zeff;
      const double kexp = (si.z <= 2 && sj.z <= 2) ? P.rep_kexp_light : P.rep_kexp;
      const double r1k = pow(r1, kexp);
      const double r1r = pow(r1, P.rep_rexp);
      e += 0.5 * zeff * exp(-alpha * r1k) / r1r;
    }
  }
  cn[a] = c;
  erep[a] = e;
  const double t1 = exp(-P.mp_kexp * (c - si.mp_vcn - P.mp_shift));
  mrad[a] = si.mp_rad + (P.mp_rmax - si.mp_rad) / (1.0 + t1);
  const int s0 = B.soff[m] + B.at_ish[a];
  for (int s = 0; s < si.nsh; ++s) {
    const ShellParam& sh = P.sh[si.sh0 + s];
    se[s0 + s] = sh.selfenergy - sh.kcn * c;
  }
}

// ---------------------------------------------------------------- neighbour list
// Half list of generate() (src/adjlist.cu:15-44): for atom i all j < i with
// eps <= r2 <= cutoff^2, j ascending.  r2 is evaluated x, y, z in that order
// with explicit round-to-nearest operations (no contraction) so that the list
// is bit-identical to the FP64 restatement.
__device__ inline bool adj_keep(const double* xyz, int i, int j, double cutoff2) {
  const double v0 = __dsub_rn(xyz[3 * i + 0], xyz[3 * j + 0]);
  const double v1 = __dsub_rn(xyz[3 * i + 1], xyz[3 * j + 1]);
  const double v2 = __dsub_rn(xyz[3 * i + 2], xyz[3 * j + 2]);
  double r2 = __dmul_rn(v0, v0);
  r2 = __dadd_rn(r2, __dmul_rn(v1, v1));
  r2 = __dadd_rn(r2, __dmul_rn(v2, v2));
  return !(r2 < 2.220446049250313e-16 || r2 > cutoff2);
}

// one warp per atom: number of kept j < i
__global__ void k_adj_count(DevBatch B, double cutoff, int* __restrict__ cnt) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= B.nat_tot) return;
  const int a = warp, m = B.at_mol[a], a0 = B.aoff[m];
  const double c2 = cutoff * cutoff;
  int n = 0;
  for (int b = a0 + lane; b < a; b += 32) n += adj_keep(B.xyz, a, b, c2) ? 1 : 0;
  for (int o = 16; o > 0; o >>= 1) n += __shfl_xor_sync(0xffffffffu, n, o);
  if (lane == 0) cnt[a] = n;
}

// one block per structure: exclusive scan of the counts -> inl (absolute pair
// offsets inside the structure's pair slice), npair per structure.
__global__ void k_adj_scan(DevBatch B, const int* __restrict__ cnt, long long* __restrict__ inl,
                           int* __restrict__ npair) {
  const int m = blockIdx.x;
  const int a0 = B.aoff[m], nat = B.aoff[m + 1] - a0;
  __shared__ long long carry;
  __shared__ int wsum[32];
  if (threadIdx.x == 0) carry = B.poff[m];
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int base = 0; base < nat; base += blockDim.x) {
    const int i = base + threadIdx.x;
    const int v = i < nat ? cnt[a0 + i] : 0;
    int x = v;  // inclusive warp scan
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) wsum[wid] = x;
    __syncthreads();
    int off = 0;
    for (int w = 0; w < wid; ++w) off += wsum[w];
    if (i < nat) inl[a0 + i] = carry + off + x - v;
    __syncthreads();
    if (threadIdx.x == 0) {
      int tot = 0;
      for (int w = 0; w < nw; ++w) tot += wsum[w];
      carry += tot;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) npair[m] = (int)(carry - B.poff[m]);
}

// one warp per atom: write kept j (local indices) in ascending order
__global__ void k_adj_fill(DevBatch B, double cutoff, const long long* __restrict__ inl,
                           int* __restrict__ pair_i, int* __restrict__ pair_j) {
  const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (warp >= B.nat_tot) return;
  const int a = warp, m = B.at_mol[a], a0 = B.aoff[m];
  const double c2 = cutoff * cutoff;
  long long pos = inl[a];
  for (int base = a0; base < a; base += 32) {
    const int b = base + lane;
    const bool keep = b < a && adj_keep(B.xyz, a, b, c2);
    const unsigned mask = __ballot_sync(0xffffffffu, keep);
    if (keep) {
      const int r = __popc(mask & ((1u << lane) - 1u));
      pair_i[pos + r] = a - a0;
      pair_j[pos + r] = b - a0;
    }
    pos += __popc(mask);
  }
}

// ---------------------------------------------------------------- integrals
// lx ("x (+1), y (-1), z (0)" sorting, src/integral/overlap.h:62-86):
// p = (y, z, x); d = (xx, yy, zz, xy, xz, yz).
__device__ constexpr int c_lx[10][3] = {{0, 0, 0}, {0, 1, 0}, {0, 0, 1}, {1, 0, 0}, {2, 0, 0},
                                {0, 2, 0}, {0, 0, 2}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}};

// 1-D overlap, dipole and quadrupole moments about centre i for one Cartesian
// direction: horizontal_shift + form_product + the moment loop of
// multipole_3d (src/integral/multipole.cu:411-457, quoted Fortran).
__device__ inline void moments_1d(int li, int lj, double rpi, double rpj, const double* s1d, double* v) {
  double vi[3] = {0, 0, 0}, vj[3] = {0, 0, 0};
  vi[li] = 1.0;
  vj[lj] = 1.0;
  if (li == 1) vi[0] += rpi * vi[1];
  if (li == 2) { vi[0] += rpi * rpi * vi[2]; vi[1] += 2.0 * rpi * vi[2]; }
  if (lj == 1) vj[0] += rpj * vj[1];
  if (lj == 2) { vj[0] += rpj * rpj * vj[2]; vj[1] += 2.0 * rpj * vj[2]; }
  double vv[5] = {0, 0, 0, 0, 0};
  for (int x = 0; x <= li; ++x)
    for (int y = 0; y <= lj; ++y) vv[x + y] += vi[x] * vj[y];
  double v0 = 0.0, v1 = 0.0, v2 = 0.0;
  for (int l = 0; l <= li + lj; ++l) {
    v0 += s1d[l] * vv[l];
    v1 += (s1d[l + 1] + rpi * s1d[l]) * vv[l];
    v2 += (s1d[l + 2] + 2.0 * rpi * s1d[l + 1] + rpi * rpi * s1d[l]) * vv[l];
  }
  v[0] = v0; v[1] = v1; v[2] = v2;
}

// Cartesian -> spherical for one index (dtrafo of src/integral/trafo.h:6-107).
template <int L>
__device__ inline void cart_to_sph(const double* c, double* s) {
  if (L < 2) {
#pragma unroll
    for (int i = 0; i < mlao(L); ++i) s[i] = c[i];
  } else {
    const double s3 = 1.7320508075688772, s3_4 = 0.8660254037844386;
    s[0] = c[2] - 0.5 * (c[0] + c[1]);
    s[1] = s3 * c[4];
    s[2] = s3 * c[5];
    s[3] = s3_4 * (c[0] - c[1]);
    s[4] = s3 * c[3];
  }
}

// transform0(lj, li, cart[mli][mlj]) -> sphr[msi][msj]
template <int LI, int LJ>
__device__ inline void transform0(const double* cart, double* sphr) {
  constexpr int MI = (LI + 1) * (LI + 2) / 2, MJ = (LJ + 1) * (LJ + 2) / 2;
  constexpr int SI = 2 * LI + 1, SJ = 2 * LJ + 1;
  double tmp[MI][SJ];
#pragma unroll
  for (int a = 0; a < MI; ++a) cart_to_sph<LJ>(cart + a * MJ, tmp[a]);
#pragma unroll
  for (int b = 0; b < SJ; ++b) {
    double col[MI], out[SI];
#pragma unroll
    for (int a = 0; a < MI; ++a) col[a] = tmp[a][b];
    cart_to_sph<LI>(col, out);
#pragma unroll
    for (int a = 0; a < SI; ++a) sphr[a * SJ + b] = out[a];
  }
}

// multipole_cgto(cgtoj, cgtoi, r2, vec, intcut) (src/integral/multipole.h:48-120,
// quoted Fortran): blocks s[SI][SJ], d[SI][SJ][3], q[SI][SJ][6] with the moment
// operator on centre i; vec = R_i - R_j.
template <int LI, int LJ>
__device__ void multipole_cgto(const ShellParam* __restrict__ ci, const ShellParam* __restrict__ cj, double r2,
                               const double* vec, double intcut, double* s, double* d, double* q) {
  constexpr int MI = (LI + 1) * (LI + 2) / 2, MJ = (LJ + 1) * (LJ + 2) / 2;
  constexpr int SI = 2 * LI + 1, SJ = 2 * LJ + 1;
  double s3d[MI * MJ], d3d[3][MI * MJ], q3d[6][MI * MJ];
#pragma unroll
  for (int x = 0; x < MI * MJ; ++x) {
    s3d[x] = 0.0;
#pragma unroll
    for (int k = 0; k < 3; ++k) d3d[k][x] = 0.0;
#pragma unroll
    for (int k = 0; k < 6; ++k) q3d[k][x] = 0.0;
  }
  const double sqrtpi3 = 5.568327996831708;
  const int npi = ci->nprim, npj = cj->nprim;
  for (int ip = 0; ip < npi; ++ip) {
    const double ai = ci->alpha[ip], cci = ci->coeff[ip];
    for (int jp = 0; jp < npj; ++jp) {
      const double aj = cj->alpha[jp];
      const double eab = ai + aj;
      const double oab = 1.0 / eab;
      const double est = ai * aj * r2 * oab;
      if (est > intcut) continue;
      const double pre = exp(-est) * sqrtpi3 * oab * sqrt(oab);
      const double cc = cci * cj->coeff[jp] * pre;
      double rpi[3], rpj[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) { rpi[k] = -vec[k] * aj * oab; rpj[k] = vec[k] * ai * oab; }
      double s1d[LI + LJ + 3];
      const double h = 0.5 * oab;
      s1d[0] = 1.0;
#pragma unroll
      for (int l = 1; l < LI + LJ + 3; ++l) s1d[l] = 0.0;
      if (LI + LJ + 2 >= 2) s1d[2] = h;
      if (LI + LJ + 2 >= 4) s1d[4] = 3.0 * h * h;
      if (LI + LJ + 2 >= 6) s1d[6] = 15.0 * h * h * h;
      // 1-D moment tables V[k][li][lj][0..2] shared by all Cartesian pairs
      double V[3][LI + 1][LJ + 1][3];
#pragma unroll
      for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int x = 0; x <= LI; ++x)
#pragma unroll
          for (int y = 0; y <= LJ; ++y) moments_1d(x, y, rpi[k], rpj[k], s1d, V[k][x][y]);
#pragma unroll
      for (int a = 0; a < MI; ++a) {
#pragma unroll
        for (int b = 0; b < MJ; ++b) {
          const double* vx = V[0][c_lx[lmap(LI) + a][0]][c_lx[lmap(LJ) + b][0]];
          const double* vy = V[1][c_lx[lmap(LI) + a][1]][c_lx[lmap(LJ) + b][1]];
          const double* vz = V[2][c_lx[lmap(LI) + a][2]][c_lx[lmap(LJ) + b][2]];
          const int x = a * MJ + b;
          s3d[x] += cc * (vx[0] * vy[0] * vz[0]);
          d3d[0][x] += cc * (vx[1] * vy[0] * vz[0]);
          d3d[1][x] += cc * (vx[0] * vy[1] * vz[0]);
          d3d[2][x] += cc * (vx[0] * vy[0] * vz[1]);
          q3d[0][x] += cc * (vx[2] * vy[0] * vz[0]);
          q3d[1][x] += cc * (vx[1] * vy[1] * vz[0]);
          q3d[2][x] += cc * (vx[0] * vy[2] * vz[0]);
          q3d[3][x] += cc * (vx[1] * vy[0] * vz[1]);
          q3d[4][x] += cc * (vx[0] * vy[1] * vz[1]);
          q3d[5][x] += cc * (vx[0] * vy[0] * vz[2]);
        }
      }
    }
  }
  double tmp[SI * SJ];
  transform0<LI, LJ>(s3d, s);
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    transform0<LI, LJ>(d3d[k], tmp);
#pragma unroll
    for (int x = 0; x < SI * SJ; ++x) d[3 * x + k] = tmp[x];
  }
#pragma unroll
  for (int k = 0; k < 6; ++k) {
    transform0<LI, LJ>(q3d[k], tmp);
#pragma unroll
    for (int x = 0; x < SI * SJ; ++x) q[6 * x + k] = tmp[x];
  }
#pragma unroll
  for (int x = 0; x < SI * SJ; ++x) {
    double* qq = q + 6 * x;
    const double tr = 0.5 * (qq[0] + qq[2] + qq[5]);
    qq[0] = 1.5 * qq[0] - tr; qq[1] = 1.5 * qq[1]; qq[2] = 1.5 * qq[2] - tr;
    qq[3] = 1.5 * qq[3]; qq[4] = 1.5 * qq[4]; qq[5] = 1.5 * qq[5] - tr;
  }
}

// shift_operator (src/h0.cu:201-250, quoted Fortran).
__device__ inline void shift_operator(const double* vec, double s, const double* di, const double* qi,
                                      double* dj, double* qj) {
  dj[0] = di[0] + vec[0] * s;
  dj[1] = di[1] + vec[1] * s;
  dj[2] = di[2] + vec[2] * s;
  qj[0] = 2 * vec[0] * di[0] + vec[0] * vec[0] * s;
  qj[2] = 2 * vec[1] * di[1] + vec[1] * vec[1] * s;
  qj[5] = 2 * vec[2] * di[2] + vec[2] * vec[2] * s;
  qj[1] = vec[0] * di[1] + vec[1] * di[0] + vec[0] * vec[1] * s;
  qj[3] = vec[0] * di[2] + vec[2] * di[0] + vec[0] * vec[2] * s;
  qj[4] = vec[1] * di[2] + vec[2] * di[1] + vec[1] * vec[2] * s;
  const double tr = 0.5 * (qj[0] + qj[2] + qj[5]);
  qj[0] = qi[0] + 1.5 * qj[0] - tr;
  qj[1] = qi[1] + 1.5 * qj[1];
  qj[2] = qi[2] + 1.5 * qj[2] - tr;
  qj[3] = qi[3] + 1.5 * qj[3];
  qj[4] = qi[4] + 1.5 * qj[4];
  qj[5] = qi[5] + 1.5 * qj[5] - tr;
}

// Scatter one shell-pair block into the structure's matrices (the assembly
// loop of get_hamiltonian, src/h0.cu:306-477, quoted Fortran).  Off-site pairs
// (onsite=false) also write the transposed block with the operator shifted to
// centre j; on-site blocks carry no H0 (the diagonal is added separately).
template <int LI, int LJ>
__device__ void scatter_block(const MatOut& out, long long mo, int n, int ii, int jj, bool onsite, double hij,
                              const double* vec, const double* s, const double* d, const double* q) {
  constexpr int SI = 2 * LI + 1, SJ = 2 * LJ + 1;
  const long long nn = (long long)n * n;
#pragma unroll
  for (int iao = 0; iao < SI; ++iao) {
#pragma unroll
    for (int jao = 0; jao < SJ; ++jao) {
      const int ij = iao * SJ + jao;
      const long long mu = jj + jao, nu = ii + iao;
      const long long e1 = mu * n + nu;
      if (!TB_GUARD(1, e1, 0, nn)) continue;
      out.S[mo + e1] = s[ij];
#pragma unroll
      for (int k = 0; k < 3; ++k) out.D[3 * mo + k * nn + e1] = d[3 * ij + k];
#pragma unroll
      for (int k = 0; k < 6; ++k) out.Q[6 * mo + k * nn + e1] = q[6 * ij + k];
      if (!onsite) {
        out.H0[mo + e1] = s[ij] * hij;
        double dj[3], qj[6];
        shift_operator(vec, s[ij], d + 3 * ij, q + 6 * ij, dj, qj);
        const long long e2 = nu * n + mu;
        if (!TB_GUARD(2, e2, 0, nn)) continue;
        out.S[mo + e2] = s[ij];
        out.H0[mo + e2] = s[ij] * hij;
#pragma unroll
        for (int k = 0; k < 3; ++k) out.D[3 * mo + k * nn + e2] = dj[k];
#pragma unroll
        for (int k = 0; k < 6; ++k) out.Q[6 * mo + k * nn + e2] = qj[k];
      }
    }
  }
}

template <int LI, int LJ>
__device__ void pair_block(const DevParams& P, const MatOut& out, long long mo, int n, int ii, int jj, bool onsite,
                           double hij, double r2, const double* vec, const ShellParam* ci, const ShellParam* cj) {
  constexpr int SI = 2 * LI + 1, SJ = 2 * LJ + 1;
  double s[SI * SJ], d[3 * SI * SJ], q[6 * SI * SJ];
  multipole_cgto<LI, LJ>(ci, cj, r2, vec, P.intcut, s, d, q);
  scatter_block<LI, LJ>(out, mo, n, ii, jj, onsite, hij, vec, s, d, q);
}

// Item offsets of class c in the sorted list and in the block records.
__device__ inline void sp_bases(const int* cls, int c, int* off, long long* rbase) {
  int o = 0;
  long long r = 0;
  for (int k = 0; k < c; ++k) {
    o += cls[k];
    r += (long long)cls[k] * sp_record(k / (kMaxL + 1), k % (kMaxL + 1));
  }
  *off = o;
  *rbase = r;
}

// Shell-pair items of the half neighbour list sorted by (li, lj) class
// c = 3 li + lj, one thread per pair slot.  Pass 0 adds each class's item
// count to cls[c]; pass 1 places the items into list, class c after the
// counts of the classes below it, through the cursors cls[16 + c], and
// records each item's index in idx[p * maxsp + sp].  An item is (pair slot,
// structure << 8 | shell pair).  The order inside a class follows the
// atomics and changes no result: every block has its own record.
__global__ void k_sp_classify(DevParams P, DevBatch B, const int* __restrict__ npair, const int* __restrict__ pair_i,
                              const int* __restrict__ pair_j, long long pair_cap, int maxsp, int pass, SpLists W) {
  constexpr int NC = (kMaxL + 1) * (kMaxL + 1), MS = kMaxShPerAtom * kMaxShPerAtom;
  __shared__ int scnt[NC], sbase[NC];
  if (threadIdx.x < NC) scnt[threadIdx.x] = 0;
  __syncthreads();
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  int m = 0, nsp = 0, nshj = 1;
  int cl[MS], loc[MS];
  if (p < pair_cap) {
    int lo = 0, hi = B.nmol;  // structure owning pair slot p
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (B.poff[mid] <= p) lo = mid; else hi = mid;
    }
    m = lo;
    if (p - B.poff[m] < npair[m]) {
      const int a0 = B.aoff[m];
      const SpeciesParam& spi = P.sp[B.id[a0 + pair_i[p]]];
      const SpeciesParam& spj = P.sp[B.id[a0 + pair_j[p]]];
      nshj = spj.nsh;
      nsp = spi.nsh * spj.nsh;
      for (int sp = 0; sp < nsp; ++sp) {
        cl[sp] = (kMaxL + 1) * P.sh[spi.sh0 + sp / nshj].ang + P.sh[spj.sh0 + sp % nshj].ang;
        loc[sp] = atomicAdd(&scnt[cl[sp]], 1);
      }
    }
  }
  __syncthreads();
  if (threadIdx.x < NC && scnt[threadIdx.x] > 0) {
    if (pass == 0) atomicAdd(&W.cls[threadIdx.x], scnt[threadIdx.x]);
    else sbase[threadIdx.x] = atomicAdd(&W.cls[16 + threadIdx.x], scnt[threadIdx.x]);
  }
  if (pass == 0) return;
  __syncthreads();
  for (int sp = 0; sp < nsp; ++sp) {
    int off;
    long long rb;
    sp_bases(W.cls, cl[sp], &off, &rb);
    const int g = off + sbase[cl[sp]] + loc[sp];
    if (!TB_GUARD(4, g, 0, W.items) || !TB_GUARD(5, p * maxsp + sp, 0, pair_cap * maxsp)) continue;
    W.list[g] = make_int2((int)p, (m << 8) | sp);
    W.idx[p * maxsp + sp] = g;
  }
}

// Pair slot of every kept atom pair i > j of a structure, at a2off + i nat + j
// and at a2off + j nat + i, so that a row of the table is read contiguously
// (the table is cleared to -1 first: atom pairs beyond the cutoff).
__global__ void k_sp_pairtab(DevBatch B, const int* __restrict__ npair, const int* __restrict__ pair_i,
                             const int* __restrict__ pair_j, long long pair_cap, int* __restrict__ tab) {
  const long long p = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (p >= pair_cap) return;
  int lo = 0, hi = B.nmol;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (B.poff[mid] <= p) lo = mid; else hi = mid;
  }
  const int m = lo;
  if (p - B.poff[m] >= npair[m]) return;
  const int nat = B.aoff[m + 1] - B.aoff[m];
  const long long x = B.a2off[m] + (long long)pair_i[p] * nat + pair_j[p];
  const long long y = B.a2off[m] + (long long)pair_j[p] * nat + pair_i[p];
  if (TB_GUARD(6, x, B.a2off[m], B.a2off[m + 1])) tab[x] = (int)p;
  if (TB_GUARD(6, y, B.a2off[m], B.a2off[m + 1])) tab[y] = (int)p;
}

// Off-site shell pairs of angular momenta (LI, LJ): one thread per item of
// the class's list (k_sp_classify), grid stride; the block goes to the
// item's record, which consecutive threads write side by side.  One
// instantiation per (li, lj) keeps the register budget of the s/p kernels
// independent of the d-shell ones.
template <int LI, int LJ>
__global__ void k_integrals_t(DevParams P, DevBatch B, const int* __restrict__ pair_i, const int* __restrict__ pair_j,
                              const double* __restrict__ se, SpLists W) {
  constexpr int C = (kMaxL + 1) * LI + LJ, SIJ = (2 * LI + 1) * (2 * LJ + 1), R = sp_record(LI, LJ);
  int off;
  long long rbase;
  sp_bases(W.cls, C, &off, &rbase);
  const int cnt = W.cls[C];
  for (int it = blockIdx.x * blockDim.x + threadIdx.x; it < cnt; it += gridDim.x * blockDim.x) {
    const int2 e = W.list[off + it];
    const int p = e.x, m = e.y >> 8, sp = e.y & 255;
    const int a0 = B.aoff[m];
    const int iat = pair_i[p], jat = pair_j[p];
    const SpeciesParam& spi = P.sp[B.id[a0 + iat]];
    const SpeciesParam& spj = P.sp[B.id[a0 + jat]];
    const int ish = sp / spj.nsh, jsh = sp % spj.nsh;
    const int ti = spi.sh0 + ish, tj = spj.sh0 + jsh;
    const ShellParam* ci = P.sh + ti;
    const ShellParam* cj = P.sh + tj;
    const int is = B.soff[m] + B.at_ish[a0 + iat], js = B.soff[m] + B.at_ish[a0 + jat];
    const double vec[3] = {B.xyz[3 * (a0 + iat)] - B.xyz[3 * (a0 + jat)],
                           B.xyz[3 * (a0 + iat) + 1] - B.xyz[3 * (a0 + jat) + 1],
                           B.xyz[3 * (a0 + iat) + 2] - B.xyz[3 * (a0 + jat) + 2]};
    const double r2 = vec[0] * vec[0] + vec[1] * vec[1] + vec[2] * vec[2];
    const double rr = sqrt(sqrt(r2) / (spj.rad + spi.rad));
    const double shpoly = (1.0 + ci->shpoly * rr) * (1.0 + cj->shpoly * rr);
    const double hij = 0.5 * (se[is + ish] + se[js + jsh]) * P.hscale[ti * P.nshtype + tj] * shpoly;
    double sb[SIJ], db[3 * SIJ], qb[6 * SIJ];
    multipole_cgto<LI, LJ>(ci, cj, r2, vec, P.intcut, sb, db, qb);
    const long long r0 = rbase + (long long)it * R;
    if (!TB_GUARD(7, r0 + R - 1, 0, W.rec_len)) continue;
    double* rec = W.rec + r0;
#pragma unroll
    for (int x = 0; x < SIJ; ++x) rec[x] = sb[x];
    rec[SIJ] = hij;
#pragma unroll
    for (int x = 0; x < 3 * SIJ; ++x) rec[SIJ + 1 + x] = db[x];
#pragma unroll
    for (int x = 0; x < 6 * SIJ; ++x) rec[4 * SIJ + 1 + x] = qb[x];
  }
}

constexpr int kAsmCols = 4;  // columns per lane and round in k_sp_assemble

// Dense S, H0, D, Q of every structure from the block records, one warp per
// AO row, lanes over the columns: each row of the eleven planes is written
// once, contiguously, zeros included (atom pairs beyond the cutoff, and the
// on-site blocks, which k_onsite_t writes afterwards).  Element (r, c) with
// atoms A = atom(r) != Bt = atom(c) belongs to the half-list pair i =
// max(A, Bt), j = min(A, Bt) (get_hamiltonian's assembly loop,
// src/h0.cu:306-477, quoted Fortran): for A < Bt it is the block's element
// [c - first AO of i's shell][r - first AO of j's shell] as computed (operator
// on centre i); for A > Bt the transposed element [r ...][c ...] with the
// dipole and quadrupole operators shifted to centre j (shift_operator).
__global__ void k_sp_assemble(DevParams P, DevBatch B, SpLists W, MatOut out, int maxsp) {
  constexpr int NC = (kMaxL + 1) * (kMaxL + 1);
  __shared__ int s_off[NC];
  __shared__ long long s_rbase[NC];
  if (threadIdx.x < NC) sp_bases(W.cls, threadIdx.x, &s_off[threadIdx.x], &s_rbase[threadIdx.x]);
  __syncthreads();
  const int lane = threadIdx.x & 31;
  const long long row = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  if (row >= B.nao_tot) return;
  int lo = 0, hi = B.nmol;  // structure owning AO row `row`
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (B.ooff[mid] <= row) lo = mid; else hi = mid;
  }
  const int m = lo, o0 = B.ooff[m], n = B.ooff[m + 1] - o0, r = (int)(row - o0);
  const int a0 = B.aoff[m], nat = B.aoff[m + 1] - a0, s0 = B.soff[m];
  const long long mo = B.moff[m], nn = (long long)n * n;
  const int A = B.ao_at[o0 + r], shA = B.ao_sh[o0 + r];
  // the row's own atom and shell, once per warp
  const int ishA = shA - B.at_ish[a0 + A], nshA = P.sp[B.id[a0 + A]].nsh;
  const int lA = P.sh[B.sh_type[s0 + shA]].ang, aoA = r - B.sh_iao[s0 + shA];
  const double xA[3] = {B.xyz[3 * (a0 + A)], B.xyz[3 * (a0 + A) + 1], B.xyz[3 * (a0 + A) + 2]};
  const int* trow = W.tab + B.a2off[m] + (long long)A * nat;
  // kAsmCols columns per lane and round: their index chains (pair table ->
  // item index -> record) are resolved first, all through the read-only
  // path, so that several chains are in flight at once
  constexpr int U = kAsmCols;
  for (int cb = lane; cb < n; cb += 32 * U) {
    const double* rec[U];
    int ij[U], sij[U], bt[U];
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int c = cb + 32 * u;
      rec[u] = nullptr;
      ij[u] = sij[u] = 0;
      bt[u] = A;
      if (c >= n) continue;
      const int Bt = __ldg(B.ao_at + o0 + c);
      bt[u] = Bt;
      if (Bt == A) continue;
      const int p = __ldg(trow + Bt);
      if (p < 0) continue;
      const bool tr = A > Bt;  // row atom is the pair's i
      const int shB = __ldg(B.ao_sh + o0 + c);
      const int ishB = shB - __ldg(B.at_ish + a0 + Bt), nshB = P.sp[__ldg(B.id + a0 + Bt)].nsh;
      const int lB = P.sh[__ldg(B.sh_type + s0 + shB)].ang, aoB = c - __ldg(B.sh_iao + s0 + shB);
      const int li = tr ? lA : lB, lj = tr ? lB : lA;
      const int SJ = 2 * lj + 1;
      const int iao = tr ? aoA : aoB, jao = tr ? aoB : aoA;
      const int sp = tr ? ishA * nshB + ishB : ishB * nshA + ishA;
      const int g = __ldg(W.idx + (long long)p * maxsp + sp);
      const int cl = (kMaxL + 1) * li + lj;
      rec[u] = W.rec + s_rbase[cl] + (long long)(g - s_off[cl]) * sp_record(li, lj);
      ij[u] = iao * SJ + jao;
      sij[u] = (2 * li + 1) * SJ;
    }
#pragma unroll
    for (int u = 0; u < U; ++u) {
      const int c = cb + 32 * u;
      if (c >= n) continue;
      const long long e = (long long)r * n + c;
      if (!TB_GUARD(8, e, 0, nn)) continue;
      double sv = 0.0, hv = 0.0, dv[3] = {0.0, 0.0, 0.0}, qv[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
      if (rec[u]) {
        const int SIJ = sij[u];
        sv = __ldg(rec[u] + ij[u]);
        hv = sv * __ldg(rec[u] + SIJ);
        double d[3], q[6];
#pragma unroll
        for (int k = 0; k < 3; ++k) d[k] = __ldg(rec[u] + SIJ + 1 + 3 * ij[u] + k);
#pragma unroll
        for (int k = 0; k < 6; ++k) q[k] = __ldg(rec[u] + 4 * SIJ + 1 + 6 * ij[u] + k);
        if (A > bt[u]) {
          const int Bt = bt[u];
          const double vec[3] = {xA[0] - B.xyz[3 * (a0 + Bt)], xA[1] - B.xyz[3 * (a0 + Bt) + 1],
                                 xA[2] - B.xyz[3 * (a0 + Bt) + 2]};
          shift_operator(vec, sv, d, q, dv, qv);
        } else {
#pragma unroll
          for (int k = 0; k < 3; ++k) dv[k] = d[k];
#pragma unroll
          for (int k = 0; k < 6; ++k) qv[k] = q[k];
        }
      }
      out.S[mo + e] = sv;
      out.H0[mo + e] = hv;
#pragma unroll
      for (int k = 0; k < 3; ++k) out.D[3 * mo + k * nn + e] = dv[k];
#pragma unroll
      for (int k = 0; k < 6; ++k) out.Q[6 * mo + k * nn + e] = qv[k];
    }
  }
}

// On-site blocks (the same-atom step missing from the reference, D8): one
// thread per (atom, shell pair); the diagonal of H0 gets the self-energies.
template <int LI, int LJ>
__global__ void k_onsite_t(DevParams P, DevBatch B, const double* __restrict__ se, MatOut out, int maxsp) {
  const long long it = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (it >= (long long)B.nat_tot * maxsp) return;
  const int a = (int)(it / maxsp), sp = (int)(it % maxsp);
  const int m = B.at_mol[a];
  const SpeciesParam& spa = P.sp[B.id[a]];
  if (sp >= spa.nsh * spa.nsh) return;
  const int ish = sp / spa.nsh, jsh = sp % spa.nsh;
  const ShellParam* ci = P.sh + spa.sh0 + ish;
  const ShellParam* cj = P.sh + spa.sh0 + jsh;
  if (ci->ang != LI || cj->ang != LJ) return;
  const int n = B.ooff[m + 1] - B.ooff[m];
  const long long mo = B.moff[m];
  const int is = B.soff[m] + B.at_ish[a];
  const int ii = B.sh_iao[is + ish], jj = B.sh_iao[is + jsh];
  const double vec[3] = {0.0, 0.0, 0.0};
  pair_block<LI, LJ>(P, out, mo, n, ii, jj, true, 0.0, 0.0, vec, ci, cj);
  if (ish == jsh) {
    for (int x = 0; x < msao(LI); ++x)
      if (TB_GUARD(3, ii + x, 0, n)) out.H0[mo + (long long)(ii + x) * n + ii + x] = se[is + ish];
  }
}

// The integral setup: shell-pair items sorted into (li, lj) classes, the
// pair table, the off-site blocks of every class present in `lmask` (bit l
// set when the parameter set has shells of angular momentum l) into their
// records, the dense planes from the records, then the on-site blocks.
cudaError_t launch_integrals(const DevParams& P, const DevBatch& B, const int* npair, const int* pair_i,
                             const int* pair_j, const double* se, const MatOut& out, int maxsp, long long pair_cap,
                             int lmask, const SpLists& W, cudaStream_t st, int64_t* launches) {
  const int grid = (int)std::max(1LL, std::min((W.items + 127) / 128, 148LL * 32));
  const int ogrid = (int)std::max(1LL, ((long long)B.nat_tot * maxsp + 127) / 128);
  const int cgrid = (int)std::max(1LL, (pair_cap + 255) / 256);
  const int agrid = (int)std::max(1LL, ((long long)B.nao_tot * 32 + 255) / 256);
  cudaError_t e = cudaMemsetAsync(W.cls, 0, 32 * sizeof(int), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(W.tab, 0xff, (size_t)W.tab_len * sizeof(int), st);
  if (e != cudaSuccess) return e;
  for (int pass = 0; pass < 2; ++pass)
    k_sp_classify<<<cgrid, 256, 0, st>>>(P, B, npair, pair_i, pair_j, pair_cap, maxsp, pass, W);
  k_sp_pairtab<<<cgrid, 256, 0, st>>>(B, npair, pair_i, pair_j, pair_cap, W.tab);
  *launches += 3;
#define TB_LAUNCH_PAIR(A, C)                                                           \
  if ((lmask >> A & 1) && (lmask >> C & 1)) {                                          \
    k_integrals_t<A, C><<<grid, 128, 0, st>>>(P, B, pair_i, pair_j, se, W);            \
    *launches += 1;                                                                    \
  }
  TB_LAUNCH_PAIR(0, 0) TB_LAUNCH_PAIR(0, 1) TB_LAUNCH_PAIR(1, 0) TB_LAUNCH_PAIR(1, 1)
  TB_LAUNCH_PAIR(0, 2) TB_LAUNCH_PAIR(2, 0) TB_LAUNCH_PAIR(1, 2) TB_LAUNCH_PAIR(2, 1) TB_LAUNCH_PAIR(2, 2)
#undef TB_LAUNCH_PAIR
  k_sp_assemble<<<agrid, 256, 0, st>>>(P, B, W, out, maxsp);
  *launches += 1;
#define TB_LAUNCH_ONSITE(A, C)                                                         \
  if ((lmask >> A & 1) && (lmask >> C & 1)) {                                          \
    k_onsite_t<A, C><<<ogrid, 128, 0, st>>>(P, B, se, out, maxsp);                     \
    *launches += 1;                                                                    \
  }
  TB_LAUNCH_ONSITE(0, 0) TB_LAUNCH_ONSITE(0, 1) TB_LAUNCH_ONSITE(1, 0) TB_LAUNCH_ONSITE(1, 1)
  TB_LAUNCH_ONSITE(0, 2) TB_LAUNCH_ONSITE(2, 0) TB_LAUNCH_ONSITE(1, 2) TB_LAUNCH_ONSITE(2, 1)
  TB_LAUNCH_ONSITE(2, 2)
#undef TB_LAUNCH_ONSITE
  return cudaGetLastError();
}

// ---------------------------------------------------------------- gradient
// Nuclear gradient, off-site shell pairs (the integral part of the gradient
// output of xtb_singlepoint, src/xtb.cu:195-196).  The blocks of a shell pair
// depend on vec = R_i - R_j only; with the moment operator on centre i,
// d/dvec <phi_j|O_i|phi_i> = <d_r phi_j|O_i|phi_i>: the j function's Cartesian
// power l along the direction is replaced by l x^(l-1) - 2 a x^(l+1) (the
// construction of the quoted multipole_grad_3d, src/multipole.cu:326-421,
// which differentiates the i function with the operator on j).

// 1-D moments of order 0..2 about centre i, powers li <= 2 and lj <= 3.
__device__ inline void moments_1d_ext(int li, int lj, double rpi, double rpj, const double* s1d, double* v) {
  double vi[3] = {0, 0, 0}, vj[4] = {0, 0, 0, 0};
  vi[li] = 1.0;
  vj[lj] = 1.0;
  if (li == 1) vi[0] += rpi;
  if (li == 2) { vi[0] += rpi * rpi; vi[1] += 2.0 * rpi; }
  if (lj == 1) vj[0] += rpj;
  if (lj == 2) { vj[0] += rpj * rpj; vj[1] += 2.0 * rpj; }
  if (lj == 3) { vj[0] += rpj * rpj * rpj; vj[1] += 3.0 * rpj * rpj; vj[2] += 3.0 * rpj; }
  double vv[6] = {0, 0, 0, 0, 0, 0};
  for (int x = 0; x <= li; ++x)
    for (int y = 0; y <= lj; ++y) vv[x + y] += vi[x] * vj[y];
  double v0 = 0.0, v1 = 0.0, v2 = 0.0;
  for (int l = 0; l <= li + lj; ++l) {
    v0 += s1d[l] * vv[l];
    v1 += (s1d[l + 1] + rpi * s1d[l]) * vv[l];
    v2 += (s1d[l + 2] + 2.0 * rpi * s1d[l + 1] + rpi * rpi * s1d[l]) * vv[l];
  }
  v[0] = v0; v[1] = v1; v[2] = v2;
}

// Values (t = 0) and vec derivatives (t = 1..3) of one shell pair's blocks:
// s[t][SI*SJ], d[t][3*SI*SJ], q[t][6*SI*SJ] (spherical, quadrupole traceless).
template <int LI, int LJ>
__device__ void multipole_cgto_grad(const ShellParam* __restrict__ ci, const ShellParam* __restrict__ cj, double r2,
                                    const double* vec, double intcut, double (*s)[(2 * LI + 1) * (2 * LJ + 1)],
                                    double (*d)[3 * (2 * LI + 1) * (2 * LJ + 1)],
                                    double (*q)[6 * (2 * LI + 1) * (2 * LJ + 1)]) {
  constexpr int MI = (LI + 1) * (LI + 2) / 2, MJ = (LJ + 1) * (LJ + 2) / 2;
  constexpr int SI = 2 * LI + 1, SJ = 2 * LJ + 1;
  double c3[4][10][MI * MJ];  // [t][s, d(3), q(6)][cartesian pair]
  for (int t = 0; t < 4; ++t)
    for (int k = 0; k < 10; ++k)
      for (int x = 0; x < MI * MJ; ++x) c3[t][k][x] = 0.0;
  const double sqrtpi3 = 5.568327996831708;
  for (int ip = 0; ip < ci->nprim; ++ip) {
    const double ai = ci->alpha[ip], cci = ci->coeff[ip];
    for (int jp = 0; jp < cj->nprim; ++jp) {
      const double aj = cj->alpha[jp];
      const double eab = ai + aj, oab = 1.0 / eab;
      const double est = ai * aj * r2 * oab;
      if (est > intcut) continue;
      const double cc = cci * cj->coeff[jp] * exp(-est) * sqrtpi3 * oab * sqrt(oab);
      double rpi[3], rpj[3];
      for (int k = 0; k < 3; ++k) { rpi[k] = -vec[k] * aj * oab; rpj[k] = vec[k] * ai * oab; }
      const double h = 0.5 * oab;
      double s1d[8] = {1.0, 0.0, h, 0.0, 3.0 * h * h, 0.0, 15.0 * h * h * h, 0.0};
      for (int a = 0; a < MI; ++a) {
        for (int b = 0; b < MJ; ++b) {
          const int* la = c_lx[lmap(LI) + a];
          const int* lb = c_lx[lmap(LJ) + b];
          double v[3][3], g[3][3];
          for (int k = 0; k < 3; ++k) {
            moments_1d_ext(la[k], lb[k], rpi[k], rpj[k], s1d, v[k]);
            double up[3], dn[3] = {0.0, 0.0, 0.0};
            moments_1d_ext(la[k], lb[k] + 1, rpi[k], rpj[k], s1d, up);
            if (lb[k] > 0) moments_1d_ext(la[k], lb[k] - 1, rpi[k], rpj[k], s1d, dn);
            for (int o = 0; o < 3; ++o) g[k][o] = lb[k] * dn[o] - 2.0 * aj * up[o];
          }
          const int x = a * MJ + b;
          for (int t = 0; t < 4; ++t) {
            const double* fx = (t == 1) ? g[0] : v[0];
            const double* fy = (t == 2) ? g[1] : v[1];
            const double* fz = (t == 3) ? g[2] : v[2];
            c3[t][0][x] += cc * (fx[0] * fy[0] * fz[0]);
            c3[t][1][x] += cc * (fx[1] * fy[0] * fz[0]);
            c3[t][2][x] += cc * (fx[0] * fy[1] * fz[0]);
            c3[t][3][x] += cc * (fx[0] * fy[0] * fz[1]);
            c3[t][4][x] += cc * (fx[2] * fy[0] * fz[0]);
            c3[t][5][x] += cc * (fx[1] * fy[1] * fz[0]);
            c3[t][6][x] += cc * (fx[0] * fy[2] * fz[0]);
            c3[t][7][x] += cc * (fx[1] * fy[0] * fz[1]);
            c3[t][8][x] += cc * (fx[0] * fy[1] * fz[1]);
            c3[t][9][x] += cc * (fx[0] * fy[0] * fz[2]);
          }
        }
      }
    }
  }
  for (int t = 0; t < 4; ++t) {
    double tmp[SI * SJ];
    transform0<LI, LJ>(c3[t][0], s[t]);
    for (int k = 0; k < 3; ++k) {
      transform0<LI, LJ>(c3[t][1 + k], tmp);
      for (int x = 0; x < SI * SJ; ++x) d[t][3 * x + k] = tmp[x];
    }
    for (int k = 0; k < 6; ++k) {
      transform0<LI, LJ>(c3[t][4 + k], tmp);
      for (int x = 0; x < SI * SJ; ++x) q[t][6 * x + k] = tmp[x];
    }
    for (int x = 0; x < SI * SJ; ++x) {
      double* qq = q[t] + 6 * x;
      const double tr = 0.5 * (qq[0] + qq[2] + qq[5]);
      qq[0] = 1.5 * qq[0] - tr; qq[1] = 1.5 * qq[1]; qq[2] = 1.5 * qq[2] - tr;
      qq[3] = 1.5 * qq[3]; qq[4] = 1.5 * qq[4]; qq[5] = 1.5 * qq[5] - tr;
    }
  }
}

// Derivative along vec_x of shift_operator's output (dj, qj) from the
// derivatives ds, ddi[3], dqi[6] of its inputs along x.
__device__ inline void shift_operator_grad(const double* vec, int x, double s, const double* di, double ds,
                                           const double* ddi, const double* dqi, double* ddj, double* dqj) {
  double e[3] = {0.0, 0.0, 0.0};
  e[x] = 1.0;
  for (int k = 0; k < 3; ++k) ddj[k] = ddi[k] + e[k] * s + vec[k] * ds;
  const int pa[6] = {0, 0, 1, 0, 1, 2}, pb[6] = {0, 1, 1, 2, 2, 2};
  double dt[6];
  for (int c = 0; c < 6; ++c) {
    const int a = pa[c], b = pb[c];
    if (a == b)
      dt[c] = 2.0 * e[a] * di[a] + 2.0 * vec[a] * ddi[a] + 2.0 * vec[a] * e[a] * s + vec[a] * vec[a] * ds;
    else
      dt[c] = e[a] * di[b] + vec[a] * ddi[b] + e[b] * di[a] + vec[b] * ddi[a] + (e[a] * vec[b] + vec[a] * e[b]) * s +
              vec[a] * vec[b] * ds;
  }
  const double tr = 0.5 * (dt[0] + dt[2] + dt[5]);
  dqj[0] = dqi[0] + 1.5 * dt[0] - tr;
  dqj[1] = dqi[1] + 1.5 * dt[1];
  dqj[2] = dqi[2] + 1.5 * dt[2] - tr;
  dqj[3] = dqi[3] + 1.5 * dt[3];
  dqj[4] = dqi[4] + 1.5 * dt[4];
  dqj[5] = dqi[5] + 1.5 * dt[5] - tr;
}

// One thread per (neighbour pair, shell pair) as k_integrals_t, structures
// with flag[m] set.  dE/dvec of the pair's blocks:
//   2 P (h_ij - (v_mu + v_nu)/2) dS - 2 W dS + 2 P S dh_ij (shpoly(rr))
//   - P (vdp(i) dD_i + vqp(i) dQ_i + vdp(j) dD_j + vqp(j) dQ_j),
// D_j, Q_j the operator shifted to centre j (shift_operator); written to
// item[p * maxsp + sp][3].  ese = sum P S hscale shpoly is dE/dse of both
// shells (written to the structure's shell-pair table at (i, j) and (j, i)).
template <int LI, int LJ>
__global__ void k_grad_pairs_t(DevParams P, DevBatch B, const int* __restrict__ npair, const int* __restrict__ pair_i,
                               const int* __restrict__ pair_j, const double* __restrict__ se,
                               const double* __restrict__ Pm, const double* __restrict__ Wm,
                               const double* __restrict__ vsh, const double* __restrict__ vat,
                               const double* __restrict__ vdp, const double* __restrict__ vqp,
                               const int* __restrict__ flag, int maxsp, long long total_items,
                               double* __restrict__ item, double* __restrict__ ese_tab) {
  constexpr int SI = 2 * LI + 1, SJ = 2 * LJ + 1;
  for (long long it = blockIdx.x * (long long)blockDim.x + threadIdx.x; it < total_items;
       it += (long long)gridDim.x * blockDim.x) {
    const long long p = it / maxsp;
    const int sp = (int)(it % maxsp);
    int lo = 0, hi = B.nmol;
    while (hi - lo > 1) {
      const int mid = (lo + hi) >> 1;
      if (B.poff[mid] <= p) lo = mid; else hi = mid;
    }
    const int m = lo;
    if (!flag[m] || p - B.poff[m] >= npair[m]) continue;
    const int a0 = B.aoff[m];
    const int iat = pair_i[p], jat = pair_j[p];
    const SpeciesParam& spi = P.sp[B.id[a0 + iat]];
    const SpeciesParam& spj = P.sp[B.id[a0 + jat]];
    if (sp >= spi.nsh * spj.nsh) continue;
    const int ish = sp / spj.nsh, jsh = sp % spj.nsh;
    const int ti = spi.sh0 + ish, tj = spj.sh0 + jsh;
    const ShellParam* ci = P.sh + ti;
    const ShellParam* cj = P.sh + tj;
    if (ci->ang != LI || cj->ang != LJ) continue;
    const int n = B.ooff[m + 1] - B.ooff[m], o0 = B.ooff[m], s0 = B.soff[m];
    const long long mo = B.moff[m];
    const int is = s0 + B.at_ish[a0 + iat], js = s0 + B.at_ish[a0 + jat];
    const int ii = B.sh_iao[is + ish], jj = B.sh_iao[js + jsh];
    const double vec[3] = {B.xyz[3 * (a0 + iat)] - B.xyz[3 * (a0 + jat)],
                           B.xyz[3 * (a0 + iat) + 1] - B.xyz[3 * (a0 + jat) + 1],
                           B.xyz[3 * (a0 + iat) + 2] - B.xyz[3 * (a0 + jat) + 2]};
    const double r2 = vec[0] * vec[0] + vec[1] * vec[1] + vec[2] * vec[2];
    const double r1 = sqrt(r2), radsum = spj.rad + spi.rad;
    const double rr = sqrt(r1 / radsum);
    const double shpoly = (1.0 + ci->shpoly * rr) * (1.0 + cj->shpoly * rr);
    const double dshpoly = ci->shpoly * (1.0 + cj->shpoly * rr) + cj->shpoly * (1.0 + ci->shpoly * rr);
    const double hs = P.hscale[ti * P.nshtype + tj];
    const double sesum = 0.5 * (se[is + ish] + se[js + jsh]);
    const double hij = sesum * hs * shpoly;
    double s[4][SI * SJ], d[4][3 * SI * SJ], q[4][6 * SI * SJ];
    multipole_cgto_grad<LI, LJ>(ci, cj, r2, vec, P.intcut, s, d, q);
    const double* vdi = vdp + 3 * (a0 + iat);
    const double* vdj = vdp + 3 * (a0 + jat);
    const double* vqi = vqp + 6 * (a0 + iat);
    const double* vqj = vqp + 6 * (a0 + jat);
    double gx[3] = {0.0, 0.0, 0.0}, ese = 0.0;
    for (int iao = 0; iao < SI; ++iao) {
      const int nu = ii + iao;
      const double vnu = vsh[s0 + B.ao_sh[o0 + nu]] + vat[a0 + B.ao_at[o0 + nu]];
      for (int jao = 0; jao < SJ; ++jao) {
        const int ij = iao * SJ + jao;
        const int mu = jj + jao;
        const long long e1 = mo + (long long)mu * n + nu;
        if (!TB_GUARD(12, e1, mo, mo + (long long)n * n)) continue;
        const double pij = Pm[e1], wij = Wm[e1];
        const double vmu = vsh[s0 + B.ao_sh[o0 + mu]] + vat[a0 + B.ao_at[o0 + mu]];
        ese += pij * s[0][ij] * hs * shpoly;
        for (int x = 0; x < 3; ++x) {
          const double drr = 0.5 / rr / radsum * vec[x] / r1;
          double g = 2.0 * pij * (hij - 0.5 * (vmu + vnu)) * s[1 + x][ij] - 2.0 * wij * s[1 + x][ij];
          g += 2.0 * pij * s[0][ij] * sesum * hs * dshpoly * drr;
          double ddj[3], dqj[6];
          shift_operator_grad(vec, x, s[0][ij], d[0] + 3 * ij, s[1 + x][ij], d[1 + x] + 3 * ij, q[1 + x] + 6 * ij,
                              ddj, dqj);
          for (int k = 0; k < 3; ++k) g -= pij * (vdi[k] * d[1 + x][3 * ij + k] + vdj[k] * ddj[k]);
          for (int c = 0; c < 6; ++c) g -= pij * (vqi[c] * q[1 + x][6 * ij + c] + vqj[c] * dqj[c]);
          gx[x] += g;
        }
      }
    }
    for (int x = 0; x < 3; ++x) item[3 * it + x] = gx[x];
    const int nsh = B.soff[m + 1] - s0;
    const long long so = B.s2off[m];
    const long long x1 = so + (long long)(is - s0 + ish) * nsh + (js - s0 + jsh);
    const long long x2 = so + (long long)(js - s0 + jsh) * nsh + (is - s0 + ish);
    if (TB_GUARD(13, x1, so, B.s2off[m + 1])) ese_tab[x1] = ese;
    if (TB_GUARD(13, x2, so, B.s2off[m + 1])) ese_tab[x2] = ese;
  }
}

TB_OOB_EXPORT(oob_setup)

cudaError_t launch_grad_pairs(const DevParams& P, const DevBatch& B, const int* npair, const int* pair_i,
                              const int* pair_j, const double* se, const double* Pm, const double* Wm,
                              const double* vsh, const double* vat, const double* vdp, const double* vqp,
                              const int* flag, int maxsp, long long items, int lmask, double* item, double* ese_tab,
                              cudaStream_t st) {
  const int grid = (int)std::max(1LL, std::min((items + 127) / 128, 148LL * 16));
#define TB_LAUNCH_GRAD(A, C)                                                                                   \
  if ((lmask >> A & 1) && (lmask >> C & 1))                                                                    \
    k_grad_pairs_t<A, C><<<grid, 128, 0, st>>>(P, B, npair, pair_i, pair_j, se, Pm, Wm, vsh, vat, vdp, vqp, flag, \
                                               maxsp, items, item, ese_tab);
  TB_LAUNCH_GRAD(0, 0) TB_LAUNCH_GRAD(0, 1) TB_LAUNCH_GRAD(1, 0) TB_LAUNCH_GRAD(1, 1)
  TB_LAUNCH_GRAD(0, 2) TB_LAUNCH_GRAD(2, 0) TB_LAUNCH_GRAD(1, 2) TB_LAUNCH_GRAD(2, 1) TB_LAUNCH_GRAD(2, 2)
#undef TB_LAUNCH_GRAD
  return cudaGetLastError();
}

}  // namespace tb
