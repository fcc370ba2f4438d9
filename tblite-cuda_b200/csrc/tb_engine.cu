// Host side of the tblite-b200 engine: parameter file, calculator, structure
// batches (workspace layout in one device allocation), kernel orchestration
// of xtb_singlepoint (reference src/xtb.cu:188-434) and the C ABI declared in
// include/tblite_b200.h.  No computation of the singlepoint happens on the
// host: it only builds index maps (the basis_type bookkeeping of
// src/basis/type.h:56-73) and launches kernels.
#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cctype>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <fstream>
#include <map>
#include <memory>
#include <mutex>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "../../include/tblite_b200.h"
#include "tb_common.cuh"
#include "tb_kernels.h"

using namespace tb;

// NVTX ranges per phase of a run (setup, SCF loop, read-outs, serving steps):
// named spans on the host timeline for Nsight tools; without a tool attached
// a push/pop is a no-op call.
struct NvtxRange {
  explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange&) = delete;
  NvtxRange& operator=(const NvtxRange&) = delete;
};

namespace {

thread_local std::string g_err;

tb_status fail(tb_status st, const std::string& msg) {
  g_err = msg;
  return st;
}

#define TB_CUDA(call)                                                                        \
  do {                                                                                       \
    cudaError_t e_ = (call);                                                                 \
    if (e_ != cudaSuccess)                                                                   \
      return fail(TB_CUDA_ERROR, std::string(#call) + ": " + cudaGetErrorString(e_));        \
  } while (0)

// ------------------------------------------------------------ parameters
struct HostParams {
  std::map<std::string, double> g;
  double kshell[3][3] = {{0}};
  std::map<std::pair<int, int>, double> kpair;
  std::vector<SpeciesParam> sp;
  std::vector<ShellParam> sh;
  std::vector<std::string> sym;
  double min_alpha = 1e300;
  // D4 block: frequency grid, quadrature weights, per species the reference
  // polarizabilities alpha(i w) on the grid (empty grid: no dispersion)
  std::vector<double> d4_freq, d4_wts;
  std::vector<std::vector<std::vector<double>>> d4_alpha;
  double glob(const char* k, double dflt = 0.0) const {
    auto it = g.find(k);
    return it == g.end() ? dflt : it->second;
  }
};

bool parse_params(const char* path, HostParams& P, std::string& err) {
  std::ifstream f(path);
  if (!f) { err = std::string("cannot open parameter file ") + path; return false; }
  std::string line;
  int cur = -1, csh = -1;
  bool fmt = false;
  std::vector<std::vector<ShellParam>> shells;
  std::vector<std::tuple<std::string, std::string, double>> kp;
  int lineno = 0;
  while (std::getline(f, line)) {
    ++lineno;
    auto h = line.find('#');
    if (h != std::string::npos) line = line.substr(0, h);
    std::istringstream is(line);
    std::string key;
    if (!(is >> key)) continue;
    auto bad = [&](const std::string& m) { err = m + " (line " + std::to_string(lineno) + ")"; return false; };
    if (key == "format") { std::string n; int v = 0; is >> n >> v; fmt = n == "tblite-b200-params" && v == 1; continue; }
    if (key == "name") continue;
    if (csh >= 0) {
      ShellParam& s = shells[cur][csh];
      if (key == "end") { csh = -1; continue; }
      if (key == "alpha") { for (int i = 0; i < s.nprim; ++i) is >> s.alpha[i]; if (!is) return bad("short alpha"); continue; }
      if (key == "coeff") { for (int i = 0; i < s.nprim; ++i) is >> s.coeff[i]; if (!is) return bad("short coeff"); continue; }
      double v; if (!(is >> v)) return bad("missing value for " + key);
      if (key == "selfenergy") s.selfenergy = v;
      else if (key == "kcn") s.kcn = v;
      else if (key == "shpoly") s.shpoly = v;
      else if (key == "refocc") s.refocc = v;
      else if (key == "hubbard") s.hubbard = v;
      else if (key == "hubbard_deriv") s.hubbard_deriv = v;
      else if (key == "slater") s.slater = v;
      else return bad("unknown shell key " + key);
      continue;
    }
    if (cur >= 0) {
      SpeciesParam& e = P.sp[cur];
      if (key == "end") { cur = -1; continue; }
      if (key == "shell") {
        ShellParam s{};
        s.slater = 1.0;
        if (!(is >> s.ang >> s.nprim)) return bad("bad shell line");
        if (s.ang < 0 || s.ang > kMaxL || s.nprim < 1 || s.nprim > kMaxPrim) return bad("unsupported shell");
        if ((int)shells[cur].size() >= kMaxShPerAtom) return bad("too many shells");
        shells[cur].push_back(s);
        csh = (int)shells[cur].size() - 1;
        continue;
      }
      if (key == "d4_ref") {
        double cn = 0;
        std::vector<double> a(P.d4_freq.size());
        is >> cn;
        for (double& x : a) is >> x;
        if (P.d4_freq.empty() || !is) return bad("d4_ref before d4freq, or short");
        if (e.d4_nref >= kD4MaxRef) return bad("more than " + std::to_string(kD4MaxRef) + " D4 references");
        e.d4_cn[e.d4_nref++] = cn;
        P.d4_alpha[cur].push_back(a);
        continue;
      }
      double v; if (!(is >> v)) return bad("missing value for " + key);
      if (key == "rad") e.rad = v;
      else if (key == "d4_r4r2") e.d4_r4r2 = v;
      else if (key == "rcov") e.rcov = v;
      else if (key == "en") e.en = v;
      else if (key == "rep_alpha") e.rep_alpha = v;
      else if (key == "rep_zeff") e.rep_zeff = v;
      else if (key == "mp_rad") e.mp_rad = v;
      else if (key == "mp_vcn") e.mp_vcn = v;
      else if (key == "dkernel") e.dkernel = v;
      else if (key == "qkernel") e.qkernel = v;
      else return bad("unknown element key " + key);
      continue;
    }
    if (key == "global") { std::string k; double v; if (!(is >> k >> v)) return bad("bad global"); P.g[k] = v; continue; }
    if (key == "d4freq" || key == "d4wts") {
      int nf = 0;
      std::vector<double>& dst = key == "d4freq" ? P.d4_freq : P.d4_wts;
      if (!(is >> nf) || nf <= 0 || nf > 256) return bad("bad " + key);
      dst.resize(nf);
      for (double& x : dst) is >> x;
      if (!is) return bad("short " + key);
      continue;
    }
    if (key == "kshell") { int a, b; double v; if (!(is >> a >> b >> v) || a < 0 || b < 0 || a > 2 || b > 2) return bad("bad kshell"); P.kshell[a][b] = P.kshell[b][a] = v; continue; }
    if (key == "kpair") { std::string a, b; double v; if (!(is >> a >> b >> v)) return bad("bad kpair"); kp.emplace_back(a, b, v); continue; }
    if (key == "element") {
      SpeciesParam e{};
      std::string sym;
      if (!(is >> sym >> e.z)) return bad("bad element line");
      P.sp.push_back(e);
      P.sym.push_back(sym);
      P.d4_alpha.emplace_back();
      shells.emplace_back();
      cur = (int)P.sp.size() - 1;
      continue;
    }
    return bad("unknown key " + key);
  }
  if (!fmt) { err = "missing or unsupported 'format' line"; return false; }
  if (P.sp.empty()) { err = "no elements"; return false; }
  if (!P.d4_freq.empty()) {
    if (P.d4_wts.size() != P.d4_freq.size()) { err = "d4wts and d4freq differ in length"; return false; }
    for (size_t i = 0; i < P.sp.size(); ++i)
      if (P.sp[i].d4_nref == 0) { err = "element " + P.sym[i] + " has no d4_ref"; return false; }
  }
  for (size_t i = 0; i < P.sp.size(); ++i) {
    P.sp[i].nsh = (int)shells[i].size();
    P.sp[i].sh0 = (int)P.sh.size();
    for (size_t s = 0; s < shells[i].size(); ++s) {
      shells[i][s].species = (int)i;
      shells[i][s].local = (int)s;
      P.sh.push_back(shells[i][s]);
      for (int k = 0; k < shells[i][s].nprim; ++k) P.min_alpha = std::min(P.min_alpha, shells[i][s].alpha[k]);
    }
  }
  for (auto& t : kp) {
    int a = -1, b = -1;
    for (size_t i = 0; i < P.sym.size(); ++i) { if (P.sym[i] == std::get<0>(t)) a = (int)i; if (P.sym[i] == std::get<1>(t)) b = (int)i; }
    if (a < 0 || b < 0) { err = "kpair names an unknown element"; return false; }
    P.kpair[{a, b}] = P.kpair[{b, a}] = std::get<2>(t);
  }
  return true;
}

// hscale(jsh, ish, jzp, izp) by shell type: GFN2-shaped preprocessing of the
// parameter file (the reference's gfn2_h0spec is empty, src/h0.h:42-48).
double hscale_of(const HostParams& P, int ti, int tj) {
  const ShellParam& a = P.sh[ti];
  const ShellParam& b = P.sh[tj];
  const double den = P.sp[a.species].en - P.sp[b.species].en;
  const double zij = std::pow(2.0 * std::sqrt(a.slater * b.slater) / (a.slater + b.slater), P.glob("wexp"));
  auto it = P.kpair.find({a.species, b.species});
  const double kp = it == P.kpair.end() ? 1.0 : it->second;
  return P.kshell[a.ang][b.ang] * kp * (1.0 + P.glob("enscale") * den * den) * zij;
}

double integral_cutoff(double acc) {
  // src/basis/type.cu:17-30 (quoted): clip(acc, min_acc=1e3, max_acc=1e-4)
  // always yields 1e-4, so intcut = 25 for every accuracy (reproduced literally).
  auto clip = [](double v, double lo, double hi) { return std::min(std::max(v, lo), hi); };
  return clip(25.0 - 10.0 * std::log10(clip(acc, 1.0e+3, 1.0e-4)), 5.0, 25.0);
}

// ------------------------------------------------------------ device arena
struct Arena {
  char* base = nullptr;
  size_t cap = 0;
  ~Arena() { if (base) cudaFree(base); }
  cudaError_t reserve(size_t bytes) {
    if (bytes <= cap) return cudaSuccess;
    if (base) { cudaFree(base); base = nullptr; cap = 0; }
    cudaError_t e = cudaMalloc(&base, bytes);
    if (e == cudaSuccess) cap = bytes;
    return e;
  }
};

struct Layout {
  size_t total = 0;
  size_t add(size_t bytes) {
    const size_t off = (total + 255) & ~size_t(255);
    total = off + bytes;
    return off;
  }
};

// The structures of each k_trid_smem class (cluster size), largest first:
// every in-house structure of max(min_n, kTridMin)..kTridClassMax[last] AOs
// (min_n = 0: none), so that k_syev can take DevBatch::trid_min/trid_max as
// the rule.
struct TridPlan {
  std::vector<int> list;
  int off[kTridClasses + 1] = {0};
  int nmax[kTridClasses] = {0};
  int trid_min = 0, trid_max = 0;
  void build(const std::vector<int>& n, const std::vector<char>& in_house, int min_n) {
    list.clear();
    for (int c = 0; c <= kTridClasses; ++c) off[c] = 0;
    for (int c = 0; c < kTridClasses; ++c) nmax[c] = 0;
    trid_min = min_n > 0 ? std::max(min_n, kTridMin) : 0;
    trid_max = min_n > 0 ? kTridClassMax[kTridClasses - 1] : 0;
    if (min_n <= 0) return;
    std::vector<std::vector<int>> cls(kTridClasses);
    for (int m = 0; m < (int)n.size(); ++m) {
      const int c = in_house[m] && n[m] >= trid_min ? trid_class_of(n[m]) : -1;
      if (c < 0) continue;
      cls[c].push_back(m);
      nmax[c] = std::max(nmax[c], n[m]);
    }
    for (int c = 0; c < kTridClasses; ++c) {
      std::stable_sort(cls[c].begin(), cls[c].end(), [&](int a, int b) { return n[a] > n[b]; });
      off[c] = (int)list.size();
      list.insert(list.end(), cls[c].begin(), cls[c].end());
    }
    off[kTridClasses] = (int)list.size();
  }
};

}  // namespace

// largest structure size (AOs) at which the GEMM tile shapes are measured
constexpr int kTileCalMax = 384;
// smallest modelled saving (fraction of the single-kernel time) for which a
// batch's GEMMs are split over both tile shapes
constexpr double kTileSplitGain = 0.05;

// ====================================================================== calculator
struct tb_calculator {
  HostParams hp;
  DevParams dp{};
  SpeciesParam* d_sp = nullptr;
  ShellParam* d_sh = nullptr;
  double* d_hscale = nullptr;
  double* d_d4c6 = nullptr;  // D4 reference C6 table (DevParams::d4_c6ref)
  int maxsh = 1;
  int lmask = 0;  // bit l set when shells of angular momentum l exist
  std::mutex mu;
  Arena arena;
  // eigensolver cost models for the automatic per-size choice (see choose_lib_above)
  struct EigModel {
    bool ready = false;
    double a = 0, b = 0;  // in-house latency of one structure: a N^2 + b N^3 seconds
    double c = 0, d = 0;  // one cuSOLVER call: c + d N^3 seconds
    double t_in[2] = {0, 0}, t_lib[2] = {0, 0};  // the measured points (256/512 and 256/1024 AOs)
  } eig;
  // small structures: the one-warp Jacobi variant against the one-CTA
  // eigensolver, measured once per calculator (batched throughput per size)
  struct SmallModel {
    bool ready = false;
    int jacobi_max = 0;              // chosen: Jacobi for N <= jacobi_max
    std::vector<int> n;              // measured sizes
    std::vector<double> t_cta, t_warp;  // seconds per structure in a full batch
  } small;
  int jacobi_override = -1;  // -1: measured choice; 0: never; 1..32: fixed bound
  // FP64 GEMM tile shape per structure size: k_gemm32 (32 x 32 tiles) where it
  // measured faster than k_gemm (64 x 64) on the SCF iteration's four GEMMs.
  // Sizes are measured in steps of 16 AOs: the tile grids and the K slabs of
  // both kernels are the same for every N in (n - 16, n], so the measurement
  // at n stands for that whole interval; above the largest, 64 x 64 tiles.
  struct TileModel {
    bool ready = false;
    std::vector<int> n;              // measured sizes (AOs)
    std::vector<double> t64, t32;    // seconds per structure in a full batch
    std::vector<char> use32;         // chosen per measured size
  } tile;
  int tile_override = -1;  // -1: measured choice; 0: 64 x 64 always; N > 0: 32 x 32 up to N AOs
  // index of the measured size that stands for n AOs (-1: above the table)
  int tile_index(int n) const {
    if (!tile.ready) return -1;
    for (size_t i = 0; i < tile.n.size(); ++i)
      if (n <= tile.n[i]) return (int)i;
    return -1;
  }
  int smem_tridiag = 0;  // FP64 structures of at least this many AOs reduced by k_trid_smem (0: none)
  std::mutex tune_mu;
  // pinned staging buffer for the batch metadata upload, reused across batches
  std::mutex stage_mu;
  char* stage = nullptr;
  size_t stage_bytes = 0;
  // pinned int slots for the batches' per-iteration active counts: pinning and
  // unpinning host memory are operating-system calls whose cost varies with
  // the host's load, so a batch takes a slot instead of allocating its own
  static constexpr int kPinSlots = 1024;
  std::mutex pin_mu;
  int* pin = nullptr;
  std::vector<int> pin_free;
  int* take_pin_slot() {
    std::lock_guard<std::mutex> lk(pin_mu);
    if (!pin) {
      if (cudaMallocHost(&pin, kPinSlots * sizeof(int)) != cudaSuccess) { pin = nullptr; return nullptr; }
      for (int i = kPinSlots - 1; i >= 0; --i) pin_free.push_back(i);
    }
    if (pin_free.empty()) return nullptr;
    const int i = pin_free.back();
    pin_free.pop_back();
    return pin + i;
  }
  bool give_pin_slot(int* p) {  // false: not from the pool
    std::lock_guard<std::mutex> lk(pin_mu);
    if (!pin || p < pin || p >= pin + kPinSlots) return false;
    pin_free.push_back((int)(p - pin));
    return true;
  }
  ~tb_calculator() {
    if (stage) cudaFreeHost(stage);
    if (pin) cudaFreeHost(pin);
    if (d_sp) cudaFree(d_sp);
    if (d_sh) cudaFree(d_sh);
    if (d_hscale) cudaFree(d_hscale);
    if (d_d4c6) cudaFree(d_d4c6);
  }
};

// ====================================================================== batch
struct tb_batch {
  tb_calculator* calc = nullptr;
  tb_options opt{};
  int nmol = 0, nat_tot = 0, nsh_tot = 0, nao_tot = 0, nmax = 0, natmax = 0, nshmax = 0;
  long long n2_tot = 0, pair_cap = 0, mix_tot = 0;
  Arena own;
  Arena* arena = nullptr;
  std::vector<int> h_aoff, h_soff, h_ooff, h_mixoff;
  std::vector<long long> h_moff, h_poff, h_s2off, h_a2off;
  std::vector<int4> tiles64, tiles32, tiles128;  // tiles32: upper 32x32 tiles (t <= u), Fock build
  // FP64 GEMM tiles by the tile autotuner's choice per structure: 64 x 64
  // (k_gemm) and 32 x 32 (k_gemm32), largest structures first in each
  std::vector<int4> gemm64, gemm32;
  std::vector<int2> chunks32;
  std::vector<double> h_xyz;
  // device views
  DevBatch db{};
  MolState ms{};
  double *cn, *mrad, *erep, *se, *n0sh;
  int *cnt, *npair, *pair_i, *pair_j;
  SpLists sp_w{};      // work space of the integral setup (in X..P, see the layout)
  size_t sp_off[4]{};  // its parts' offsets from X
  long long* inl;
  double *S, *H0, *D, *Q, *X, *W, *F, *Z, *P;
  double *gtab, *atab;  // Coulomb pair tables of the fixed geometry (k_pair_tables)
  // D4 dispersion of the fixed geometry (setup; only with a D4 parameter block):
  // per atom cn, W, dW (kD4MaxRef), energy share, dE/dCN, gradient; per structure e_disp
  double *d4cn = nullptr, *d4w = nullptr, *d4dw = nullptr, *d4e = nullptr, *d4dcn = nullptr, *d4g = nullptr,
         *e_disp = nullptr;
  double *w, *focc, *vsh, *vat, *vdp, *vqp, *colred, *qsh_out, *qat_out, *dpat_out, *qpat_out;
  int *perm, *kdim;
  double *q_in, *dq, *dqlast, *qlast, *df, *u, *amat, *omega;
  double* charge;
  int* uhf;
  // caller's starting moments (tb_wavefunction.guess): host copy in the q_in
  // layout, per-structure flags, and their device buffers
  std::vector<double> h_guess;
  std::vector<int> h_guess_flag;
  bool any_guess = false;
  double* d_guess = nullptr;
  int* d_guess_flag = nullptr;
  // gradient read-out: its own workspace (allocated on first use), the
  // gradient [nat_tot][3] and sigma [nmol][9] of the structures computed
  Arena grad_ws;
  double *d_grad = nullptr, *d_sigma = nullptr;
  std::vector<int> h_grad_done;
  // nspin = 2 read-out: per-channel occupations (3 x nao_tot) and structure flags
  double* d_fspin = nullptr;
  int* d_wflag = nullptr;
  int* d_jlist = nullptr;  // structures on the one-warp Jacobi eigensolver
  int njac = 0;
  TridPlan trid;            // structures tridiagonalised by k_trid_smem, per class
  int* d_tlist = nullptr;
  int4 *d_tiles64, *d_tiles32, *d_tiles128;
  int4 *d_gemm64 = nullptr, *d_gemm32 = nullptr;
  int ngemm64 = 0, ngemm32 = 0;
  int2* d_chunks32;
  int* h_nactive = nullptr;  // pinned
  // structures above the in-house size bound: cuSOLVER path (tb_large.cu)
  std::vector<int> big;
  int nmax_in = 0;           // largest N on the in-house eigensolver
  LargeSolver lib;
  void* lib_work = nullptr;
  size_t lib_bytes = 0;
  int* lib_info = nullptr;   // 2 per library structure
  std::vector<int> h_active, h_status, h_phase;
  std::vector<int> h_species;  // species index per atom of the batch
  // mixed-precision form (tb_options.precision = 1)
  bool mixed = false;
  float *Af = nullptr, *Zf = nullptr, *wf = nullptr;
  double *Vn = nullptr, *G = nullptr;
  int *act_lo = nullptr, *act_hi = nullptr;
  // stepping state (tb_batch_begin / tb_batch_step) and the captured iteration
  DevParams Pc{};
  int it = 0;
  cudaStream_t cap = nullptr;       // capture stream of the iteration graph
  cudaGraphExec_t gexec = nullptr;  // one SCF iteration (tb_options.use_graphs, serving)
  cudaGraphExec_t gloop = nullptr;  // the whole SCF loop as a conditional WHILE node (use_graphs)
  int* it_dev = nullptr;            // SCF iterations run by the loop graph
  int64_t launches_per_iter = 0;
  int64_t launches = 0;
  size_t bytes = 0;
  std::vector<double> h_nocc;  // closed-shell occupied orbitals per structure (work accounting)
  // kernel-class profile of the last run (tb_options.profile)
  struct KClass {
    std::string name;
    int64_t launches = 0;
    double ms = 0.0, work = 0.0;
    int unit = 0;
  };
  std::vector<KClass> kclass;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> pend;
  std::vector<cudaEvent_t> evpool;
  size_t evused = 0;
  ~tb_batch() {
    if (gexec) cudaGraphExecDestroy(gexec);
    if (gloop) cudaGraphExecDestroy(gloop);
    if (cap) cudaStreamDestroy(cap);
    if (h_nactive && !(calc && calc->give_pin_slot(h_nactive))) cudaFreeHost(h_nactive);
    for (cudaEvent_t e : evpool) cudaEventDestroy(e);
  }
};

namespace {

template <typename T>
T* at(char* base, size_t off) { return reinterpret_cast<T*>(base + off); }

tb_status calibrate_eigensolvers(tb_calculator* c);
tb_status calibrate_small(tb_calculator* c);
tb_status calibrate_tiles(tb_calculator* c);

// Automatic eigensolver choice for a batch (tb_options.solver = 0): the k
// largest structures go to cuSOLVER, the rest to the batched in-house solver,
// with k minimising the modelled time of one SCF iteration's eigensolve:
//   sum_{i<k} t_lib(N_i) + max(t_in(N_k), sum_{i>=k} t_in(N_i) / slots)
// (library calls run one after another; in-house structures run concurrently,
// one CTA each, up to `slots` at a time; t_in and t_lib are measured once per
// calculator).  Returns lib_above: structures with more AOs go to the library.
int choose_lib_above(tb_calculator* c, std::vector<int> sizes) {
  std::sort(sizes.begin(), sizes.end(), std::greater<int>());
  const int nmol = (int)sizes.size();
  int k0 = 0;
  while (k0 < nmol && sizes[k0] > kSyevMaxN) ++k0;
  if (k0 == nmol) return -1;
  if (sizes[k0] < 384) return kSyevMaxN;  // small structures: the batched solver always wins
  if (calibrate_eigensolvers(c) != TB_OK) return kSyevMaxN;
  const auto& M = c->eig;
  auto t_in = [&](double n) { return M.a * n * n + M.b * n * n * n; };
  auto t_lib = [&](double n) { return M.c + M.d * n * n * n; };
  auto slots = [&](int n) {
    const int per = (int)std::min<size_t>(3, (227 * 1024) / std::max<size_t>(syev_smem_bytes(n), 1));
    return 148.0 * std::max(per, 1);
  };
  std::vector<double> tail(nmol + 1, 0.0);
  for (int i = nmol - 1; i >= 0; --i) tail[i] = tail[i + 1] + t_in(sizes[i]);
  double lib_sum = 0.0, best = 1e300;
  int best_k = k0;
  for (int i = 0; i < k0; ++i) lib_sum += t_lib(sizes[i]);
  for (int k = k0; k <= nmol; ++k) {
    const double in_t = k == nmol ? 0.0 : std::max(t_in(sizes[k]), tail[k] / slots(sizes[k]));
    if (lib_sum + in_t < best) { best = lib_sum + in_t; best_k = k; }
    if (k < nmol) lib_sum += t_lib(sizes[k]);
  }
  if (best_k == nmol) return -1;
  return best_k == 0 ? kSyevMaxN : sizes[best_k];
}

// Build index maps, lay out the workspace, allocate, upload.
tb_status batch_build(tb_calculator* calc, const tb_structure* mols, int nmol, const tb_options* opt,
                      tb_batch* b, Arena* arena) {
  NvtxRange nv("tb.batch_build");
  const HostParams& P = calc->hp;
  b->calc = calc;
  b->opt = *opt;
  b->nmol = nmol;
  if (nmol <= 0) return fail(TB_BAD_INPUT, "nmol must be positive");
  if (opt->max_iter < 1 || opt->max_iter > 64) return fail(TB_BAD_INPUT, "max_iter must be in 1..64");
  if (opt->precision != 0 && opt->precision != 1) return fail(TB_BAD_INPUT, "precision must be 0 or 1");
  b->mixed = opt->precision == 1;
  b->h_aoff.assign(nmol + 1, 0); b->h_soff.assign(nmol + 1, 0); b->h_ooff.assign(nmol + 1, 0);
  b->h_mixoff.assign(nmol + 1, 0); b->h_moff.assign(nmol + 1, 0); b->h_poff.assign(nmol + 1, 0);
  b->h_s2off.assign(nmol + 1, 0); b->h_a2off.assign(nmol + 1, 0);
  std::vector<int> id, at_mol, sh_type, sh_at, sh_iao, at_ish, ao_at, ao_sh;
  b->h_xyz.clear();
  b->h_nocc.clear();
  // validation and sizes per structure, in order (the first bad structure is
  // the one reported), then offsets, then the index maps filled in parallel
  // over structures, each at its own offsets
  std::vector<int> nsh_m(nmol), nao_m(nmol);
  for (int m = 0; m < nmol; ++m) {
    const tb_structure& s = mols[m];
    if (s.nat <= 0 || !s.id || !s.xyz) return fail(TB_BAD_INPUT, "structure " + std::to_string(m) + ": empty or null");
    int sh = 0, ao = 0;
    for (int a = 0; a < s.nat; ++a) {
      const int z = s.id[a];
      if (z < 0 || z >= (int)P.sp.size()) return fail(TB_BAD_INPUT, "structure " + std::to_string(m) + ": bad species");
      for (int k = 0; k < 3; ++k)
        if (!std::isfinite(s.xyz[3 * a + k]))
          return fail(TB_BAD_INPUT, "structure " + std::to_string(m) + ": non-finite coordinate");
      const SpeciesParam& sp = P.sp[z];
      sh += sp.nsh;
      for (int k = 0; k < sp.nsh; ++k) ao += msao(P.sh[sp.sh0 + k].ang);
    }
    nsh_m[m] = sh;
    nao_m[m] = ao;
  }
  std::vector<long long> t64o(nmol + 1, 0), t128o(nmol + 1, 0), t32o(nmol + 1, 0), c32o(nmol + 1, 0);
  for (int m = 0; m < nmol; ++m) {
    const int nat = mols[m].nat, nsh = nsh_m[m], nao = nao_m[m];
    b->h_aoff[m + 1] = b->h_aoff[m] + nat;
    b->h_soff[m + 1] = b->h_soff[m] + nsh;
    b->h_ooff[m + 1] = b->h_ooff[m] + nao;
    b->h_mixoff[m + 1] = b->h_mixoff[m] + nsh + 9 * nat;
    b->h_moff[m + 1] = b->h_moff[m] + (long long)nao * nao;
    b->h_poff[m + 1] = b->h_poff[m] + (long long)nat * (nat - 1) / 2;
    b->h_s2off[m + 1] = b->h_s2off[m] + (long long)nsh * nsh;
    b->h_a2off[m + 1] = b->h_a2off[m] + (long long)nat * nat;
    b->nmax = std::max(b->nmax, nao);
    b->natmax = std::max(b->natmax, nat);
    b->nshmax = std::max(b->nshmax, nsh);
    const long long a64 = (nao + 63) / 64, a128 = (nao + kTcTile - 1) / kTcTile, a32 = (nao + 31) / 32;
    t64o[m + 1] = t64o[m] + a64 * a64;
    t128o[m + 1] = t128o[m] + a128 * a128;
    t32o[m + 1] = t32o[m] + a32 * (a32 + 1) / 2;
    c32o[m + 1] = c32o[m] + a32;
  }
  {
    const long long na = b->h_aoff[nmol], ns = b->h_soff[nmol], no = b->h_ooff[nmol];
    id.resize(na); at_mol.resize(na); at_ish.resize(na); b->h_xyz.resize(3 * na);
    sh_type.resize(ns); sh_at.resize(ns); sh_iao.resize(ns); ao_at.resize(no); ao_sh.resize(no);
    b->h_nocc.resize(nmol);
    b->tiles64.resize(t64o[nmol]); b->tiles128.resize(t128o[nmol]); b->tiles32.resize(t32o[nmol]);
    b->chunks32.resize(c32o[nmol]);
  }
  auto fill = [&](int m) {
    const tb_structure& s = mols[m];
    const int a0 = b->h_aoff[m], s0 = b->h_soff[m], o0 = b->h_ooff[m];
    int nsh = 0, nao = 0;
    double nref = -s.charge;
    for (int a = 0; a < s.nat; ++a) {
      const int z = s.id[a];
      id[a0 + a] = z;
      at_mol[a0 + a] = m;
      at_ish[a0 + a] = nsh;
      for (int k = 0; k < 3; ++k) b->h_xyz[3 * (long long)(a0 + a) + k] = s.xyz[3 * a + k];
      const SpeciesParam& sp = P.sp[z];
      for (int k = 0; k < sp.nsh; ++k) {
        const ShellParam& sh = P.sh[sp.sh0 + k];
        sh_type[s0 + nsh] = sp.sh0 + k;
        sh_at[s0 + nsh] = a;
        sh_iao[s0 + nsh] = nao;
        for (int x = 0; x < msao(sh.ang); ++x) { ao_at[o0 + nao + x] = a; ao_sh[o0 + nao + x] = nsh; }
        nao += msao(sh.ang);
        nsh += 1;
        nref += sh.refocc;
      }
    }
    b->h_nocc[m] = std::ceil(0.5 * nref);
    long long i64 = t64o[m], i128 = t128o[m], i32 = t32o[m], ic = c32o[m];
    for (int t = 0; t < (nao + 63) / 64; ++t)
      for (int u = 0; u < (nao + 63) / 64; ++u) b->tiles64[i64++] = make_int4(m, t, u, 0);
    for (int t = 0; t < (nao + kTcTile - 1) / kTcTile; ++t)
      for (int u = 0; u < (nao + kTcTile - 1) / kTcTile; ++u) b->tiles128[i128++] = make_int4(m, t, u, 0);
    for (int t = 0; t < (nao + 31) / 32; ++t) {
      b->chunks32[ic++] = make_int2(m, t);
      for (int u = t; u < (nao + 31) / 32; ++u) b->tiles32[i32++] = make_int4(m, t, u, 0);
    }
  };
  {
    const long long na = b->h_aoff[nmol];
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    const int nth = (int)std::min<long long>(std::min(hw, 8), std::max<long long>(1, na / 8192));
    if (nth <= 1) {
      for (int m = 0; m < nmol; ++m) fill(m);
    } else {  // contiguous ranges of about na / nth atoms
      std::vector<std::thread> pool;
      int lo = 0;
      try {
        for (int t = 0; t < nth && lo < nmol; ++t) {
          const long long target = na * (t + 1) / nth;
          int hi = lo;
          while (hi < nmol && (t == nth - 1 || b->h_aoff[hi] < target)) ++hi;
          if (hi == lo) hi = lo + 1;
          pool.emplace_back([&fill, lo, hi]() { for (int m = lo; m < hi; ++m) fill(m); });
          lo = hi;
        }
      } catch (...) {  // no thread: the ranges not handed out are filled here
      }
      for (int m = lo; m < nmol; ++m) fill(m);
      for (auto& th : pool) th.join();
    }
  }
  // solver choice: 0 auto (in-house up to kSyevMaxN AOs, library above), 1 in-house only, 2 library only
  int lib_above = 0;
  if (opt->solver == 0) {
    std::vector<int> sizes(nmol);
    for (int m = 0; m < nmol; ++m) sizes[m] = b->h_ooff[m + 1] - b->h_ooff[m];
    lib_above = choose_lib_above(calc, sizes);
  } else if (opt->solver == 2) {
    lib_above = -1;
  }
  else if (opt->solver != 1) return fail(TB_BAD_INPUT, "solver must be 0, 1 or 2");
  if (opt->solver == 1 && b->nmax > kSyevMaxN)
    return fail(TB_CAPACITY_EXCEEDED, "structure with " + std::to_string(b->nmax) +
                " AOs exceeds the in-house eigensolver limit (" + std::to_string(kSyevMaxN) + " AOs)");
  b->big.clear();
  b->nmax_in = 0;
  int nbig_max = 0;
  for (int m = 0; m < nmol; ++m) {
    const int n = b->h_ooff[m + 1] - b->h_ooff[m];
    if (lib_above != 0 && n > lib_above) {
      b->big.push_back(m);
      nbig_max = std::max(nbig_max, n);
    } else {
      b->nmax_in = std::max(b->nmax_in, n);
    }
  }
  // small structures: the one-warp Jacobi variant up to the measured (or set) bound
  int jacobi_max = 0;
  std::vector<int> jlist;
  {
    int nmin = 1 << 30;
    for (int m = 0; m < nmol; ++m) nmin = std::min(nmin, b->h_ooff[m + 1] - b->h_ooff[m]);
    if (calc->jacobi_override >= 0) {
      jacobi_max = std::min(calc->jacobi_override, kJacobiMaxN);
    } else if (nmin <= kJacobiMaxN) {
      const tb_status ts = calibrate_small(calc);
      if (ts != TB_OK) return ts;
      jacobi_max = calc->small.jacobi_max;
    }
    for (int m = 0; m < nmol; ++m) {
      const int n = b->h_ooff[m + 1] - b->h_ooff[m];
      if (n <= jacobi_max && !(lib_above != 0 && n > lib_above)) jlist.push_back(m);
    }
  }
  {
    std::vector<int> sizes(nmol);
    std::vector<char> in_house(nmol);
    for (int m = 0; m < nmol; ++m) {
      sizes[m] = b->h_ooff[m + 1] - b->h_ooff[m];
      in_house[m] = !(lib_above != 0 && sizes[m] > lib_above);
    }
    b->trid.build(sizes, in_house, calc->smem_tridiag);
  }
  // GEMM tile shape per structure (the measured choice unless overridden)
  {
    bool small = false;
    for (int m = 0; m < nmol && !small; ++m) small = b->h_ooff[m + 1] - b->h_ooff[m] <= kTileCalMax;
    if (calc->tile_override < 0 && small) {
      const tb_status ts = calibrate_tiles(calc);
      if (ts != TB_OK) return ts;
    }
    // Measured mode: each structure the faster shape of its size.  A batch
    // that would then need both kernels pays a second launch per product (its
    // own ramp and tail; on the 1024-cluster batch a modelled 1.3% saving
    // measured as a 5% loss), so it is split only when the modelled saving --
    // the measured per-structure times summed over the batch -- is at least
    // kTileSplitGain of the better single shape; otherwise the batch takes
    // that single shape (32 x 32 only when no structure is above the table).
    std::vector<char> t32(nmol, 0);
    if (calc->tile_override >= 0) {
      for (int m = 0; m < nmol; ++m) t32[m] = b->h_ooff[m + 1] - b->h_ooff[m] <= calc->tile_override;
    } else if (calc->tile.ready) {
      double s64 = 0, s32 = 0, smin = 0;
      int n32 = 0, n64 = 0, nbig = 0;
      for (int m = 0; m < nmol; ++m) {
        const int i = calc->tile_index(b->h_ooff[m + 1] - b->h_ooff[m]);
        if (i < 0) { ++nbig; continue; }
        const double a = calc->tile.t64[i], c = calc->tile.t32[i];
        s64 += a; s32 += c; smin += std::min(a, c);
        t32[m] = calc->tile.use32[i];
        (t32[m] ? n32 : n64) += 1;
      }
      if (n32 > 0 && (n64 > 0 || nbig > 0)) {  // the per-structure choice needs both kernels
        const bool all32 = nbig == 0 && s32 < s64;
        const double single = all32 ? s32 : s64;
        if (single - smin < kTileSplitGain * single)
          for (int m = 0; m < nmol; ++m)
            t32[m] = all32 && calc->tile_index(b->h_ooff[m + 1] - b->h_ooff[m]) >= 0;
      }
    }
    std::vector<int> ord(nmol);
    for (int m = 0; m < nmol; ++m) ord[m] = m;
    std::stable_sort(ord.begin(), ord.end(), [&](int x, int y) {
      return b->h_ooff[x + 1] - b->h_ooff[x] > b->h_ooff[y + 1] - b->h_ooff[y];
    });
    b->gemm64.clear();
    b->gemm32.clear();
    for (int m : ord) {
      const int n = b->h_ooff[m + 1] - b->h_ooff[m];
      const int nt = t32[m] ? (n + 31) / 32 : (n + 63) / 64;
      std::vector<int4>& v = t32[m] ? b->gemm32 : b->gemm64;
      for (int t = 0; t < nt; ++t)
        for (int u = 0; u < nt; ++u) v.push_back(make_int4(m, t, u, 0));
    }
    b->ngemm64 = (int)b->gemm64.size();
    b->ngemm32 = (int)b->gemm32.size();
  }
  b->lib_bytes = 0;
  if (!b->big.empty()) {
    const std::string e = b->lib.workspace(nbig_max, &b->lib_bytes);
    if (!e.empty()) return fail(TB_CUDA_ERROR, "library eigensolver: " + e);
  }
  b->nat_tot = b->h_aoff[nmol];
  b->nsh_tot = b->h_soff[nmol];
  b->nao_tot = b->h_ooff[nmol];
  b->n2_tot = b->h_moff[nmol];
  b->pair_cap = std::max<long long>(1, b->h_poff[nmol]);
  b->mix_tot = b->h_mixoff[nmol];
  const int mem = opt->max_iter;

  // ---- layout
  Layout L;
  const size_t D8 = sizeof(double), I4 = sizeof(int);
  const long long NA = b->nat_tot, NS = b->nsh_tot, NO = b->nao_tot, N2 = b->n2_tot, NM = nmol, MX = b->mix_tot;
  size_t o_meta_aoff = L.add((NM + 1) * I4), o_meta_soff = L.add((NM + 1) * I4), o_meta_ooff = L.add((NM + 1) * I4),
         o_meta_mixoff = L.add((NM + 1) * I4), o_meta_moff = L.add((NM + 1) * 8), o_meta_poff = L.add((NM + 1) * 8),
         o_meta_s2off = L.add((NM + 1) * 8), o_meta_a2off = L.add((NM + 1) * 8),
         o_xyz = L.add(3 * NA * D8), o_id = L.add(NA * I4), o_atmol = L.add(NA * I4), o_shtype = L.add(NS * I4),
         o_shat = L.add(NS * I4), o_shiao = L.add(NS * I4), o_atish = L.add(NA * I4), o_aoat = L.add(NO * I4),
         o_aosh = L.add(NO * I4), o_t64 = L.add(b->tiles64.size() * sizeof(int4)),
         o_t128 = L.add(b->tiles128.size() * sizeof(int4)),
         o_t32 = L.add(b->tiles32.size() * sizeof(int4)), o_c32 = L.add(b->chunks32.size() * sizeof(int2)),
         o_g64 = L.add(b->gemm64.size() * sizeof(int4)), o_g32 = L.add(b->gemm32.size() * sizeof(int4)),
         o_charge = L.add(NM * D8), o_uhf = L.add(NM * I4), o_order = L.add(NM * I4),
         o_jlist = L.add(NM * I4), o_tlist = L.add(NM * I4);
  const size_t meta_end = L.total;
  size_t o_gtab = L.add((size_t)b->h_s2off[nmol] * D8), o_atab = L.add((size_t)b->h_a2off[nmol] * 3 * D8);
  size_t o_cn = L.add(NA * D8), o_mrad = L.add(NA * D8), o_erep = L.add(NA * D8), o_se = L.add(NS * D8),
         o_n0sh = L.add(NS * D8), o_cnt = L.add(NA * I4), o_inl = L.add(NA * 8), o_npair = L.add(NM * I4),
         o_pi = L.add(b->pair_cap * I4), o_pj = L.add(b->pair_cap * I4), o_spc = L.add(32 * I4);
  size_t o_S = L.add(N2 * D8), o_H0 = L.add(N2 * D8), o_D = L.add(3 * N2 * D8), o_Q = L.add(6 * N2 * D8);
  size_t o_X = L.add(N2 * D8), o_W = L.add(N2 * D8), o_F = L.add(N2 * D8), o_Z = L.add(N2 * D8),
         o_P = L.add(N2 * D8);
  // Work space of the integral setup (SpLists: block records, class list,
  // item index, pair table) in X..P, which the setup fills only after the
  // integrals; extended here when the batch needs more.  Bounds: every atom
  // pair i > j of a structure within the cutoff, sum over pairs of
  // nsh_i nsh_j items and 10 nao_i nao_j + nsh_i nsh_j record doubles.
  {
    long long items = 0, rec = 0;
    for (int m = 0; m < nmol; ++m) {
      long long sh = 0, sh2 = 0, ao = 0, ao2 = 0;
      for (int a = b->h_aoff[m]; a < b->h_aoff[m + 1]; ++a) {
        const SpeciesParam& spa = P.sp[id[a]];
        long long na = 0;
        for (int k = 0; k < spa.nsh; ++k) na += msao(P.sh[spa.sh0 + k].ang);
        sh += spa.nsh; sh2 += (long long)spa.nsh * spa.nsh; ao += na; ao2 += na * na;
      }
      const long long it = (sh * sh - sh2) / 2;
      items += it;
      rec += 10 * ((ao * ao - ao2) / 2) + it;
    }
    const long long idx = b->pair_cap * (long long)calc->maxsh * calc->maxsh;
    if (items >= (1LL << 31) || b->pair_cap >= (1LL << 31) || nmol >= (1 << 23))
      return fail(TB_CAPACITY_EXCEEDED, "batch too large for the integral work space (" + std::to_string(items) +
                                            " shell pairs, " + std::to_string(nmol) + " structures)");
    auto up = [](size_t x) { return (x + 255) & ~size_t(255); };
    b->sp_w.items = items;
    b->sp_w.rec_len = rec;
    b->sp_w.tab_len = b->h_a2off[nmol];
    b->sp_off[0] = 0;                                            // records
    b->sp_off[1] = up((size_t)rec * D8);                         // class list
    b->sp_off[2] = b->sp_off[1] + up((size_t)items * sizeof(int2));  // item index
    b->sp_off[3] = b->sp_off[2] + up((size_t)idx * I4);          // pair table
    const size_t need = b->sp_off[3] + (size_t)b->sp_w.tab_len * I4, end = L.add(0);
    if (end - o_X < need) L.add(need - (end - o_X));
  }
  size_t o_w = L.add(NO * D8), o_focc = L.add(NO * D8), o_perm = L.add(NO * I4), o_kdim = L.add(NM * I4),
         o_vsh = L.add(NS * D8), o_vat = L.add(NA * D8), o_vdp = L.add(3 * NA * D8), o_vqp = L.add(6 * NA * D8),
         o_col = L.add(12 * NO * D8), o_qsho = L.add(NS * D8), o_qato = L.add(NA * D8), o_dpo = L.add(3 * NA * D8),
         o_qpo = L.add(6 * NA * D8);
  size_t o_qin = L.add(MX * D8), o_dq = L.add(MX * D8), o_dql = L.add(MX * D8), o_ql = L.add(MX * D8),
         o_df = L.add((size_t)mem * MX * D8), o_u = L.add((size_t)mem * MX * D8),
         o_amat = L.add((size_t)mem * mem * NM * D8), o_om = L.add((size_t)mem * NM * D8);
  size_t o_ms_erep = L.add(NM * D8), o_ms_nel = L.add(2 * NM * D8), o_ms_iscf = L.add(NM * I4),
         o_ms_mix = L.add(NM * I4), o_ms_eelec = L.add(NM * D8), o_ms_active = L.add(NM * I4),
         o_ms_status = L.add(NM * I4), o_ms_ets = L.add(NM * D8), o_ms_eband = L.add(NM * D8),
         o_ms_ees2 = L.add(NM * D8), o_ms_eaes2 = L.add(NM * D8), o_ms_ees3 = L.add(NM * D8),
         o_ms_err = L.add(NM * D8), o_ms_fw = L.add(NM * I4), o_ms_dip = L.add(3 * NM * D8),
         o_ms_nact = L.add(I4), o_itdev = L.add(I4);
  size_t o_guess = L.add(MX * D8), o_gflag = L.add(NM * I4), o_fspin = L.add(3 * NO * D8),
         o_wflag = L.add(NM * I4);
  size_t o_d4cn = L.add(NA * D8), o_d4w = L.add(kD4MaxRef * NA * D8), o_d4dw = L.add(kD4MaxRef * NA * D8),
         o_d4e = L.add(NA * D8), o_d4dcn = L.add(NA * D8), o_d4g = L.add(3 * NA * D8), o_edisp = L.add(NM * D8);
  size_t o_lwork = L.add(std::max<size_t>(b->lib_bytes, 16)), o_linfo = L.add((2 * b->big.size() + 2) * I4);
  // mixed-precision form: FP32 eigensolver input/output, refinement buffers, phase state
  const long long MXN2 = b->mixed ? N2 : 0, MXNO = b->mixed ? NO : 0, MXNM = b->mixed ? NM : 0;
  size_t o_Af = L.add(MXN2 * 4), o_Zf = L.add(MXN2 * 4), o_wf = L.add(MXNO * 4), o_Vn = L.add(MXN2 * D8),
         o_G = L.add(MXN2 * D8), o_lo = L.add(MXNM * I4), o_hi = L.add(MXNM * I4), o_phase = L.add(MXNM * I4),
         o_n64 = L.add(MXNM * I4);
  b->bytes = L.total;
  b->arena = arena;
  {
    cudaError_t e = arena->reserve(L.total);
    if (e != cudaSuccess)
      return fail(TB_CUDA_ERROR, "workspace of " + std::to_string(L.total >> 20) + " MiB: " + cudaGetErrorString(e));
  }
  char* base = arena->base;
  // ---- metadata upload (one host blob in the calculator's pinned staging
  // buffer, one copy; the padding between fields is never read)
  std::lock_guard<std::mutex> stage_lk(calc->stage_mu);
  if (calc->stage_bytes < meta_end) {
    if (calc->stage) cudaFreeHost(calc->stage);
    calc->stage = nullptr;
    calc->stage_bytes = 0;
    TB_CUDA(cudaMallocHost(&calc->stage, meta_end + (meta_end >> 2)));
    calc->stage_bytes = meta_end + (meta_end >> 2);
  }
  char* blob = calc->stage;
  auto put = [&](size_t off, const void* src, size_t n) { if (n) std::memcpy(blob + off, src, n); };
  put(o_meta_aoff, b->h_aoff.data(), (NM + 1) * I4);
  put(o_meta_soff, b->h_soff.data(), (NM + 1) * I4);
  put(o_meta_ooff, b->h_ooff.data(), (NM + 1) * I4);
  put(o_meta_mixoff, b->h_mixoff.data(), (NM + 1) * I4);
  put(o_meta_moff, b->h_moff.data(), (NM + 1) * 8);
  put(o_meta_poff, b->h_poff.data(), (NM + 1) * 8);
  put(o_meta_s2off, b->h_s2off.data(), (NM + 1) * 8);
  put(o_meta_a2off, b->h_a2off.data(), (NM + 1) * 8);
  put(o_xyz, b->h_xyz.data(), 3 * NA * D8);
  put(o_id, id.data(), NA * I4);
  b->h_species.swap(id);
  put(o_atmol, at_mol.data(), NA * I4);
  put(o_shtype, sh_type.data(), NS * I4);
  put(o_shat, sh_at.data(), NS * I4);
  put(o_shiao, sh_iao.data(), NS * I4);
  put(o_atish, at_ish.data(), NA * I4);
  put(o_aoat, ao_at.data(), NO * I4);
  put(o_aosh, ao_sh.data(), NO * I4);
  // GEMM tiles of the largest structures first: their tiles carry the longest
  // K ranges, so the grid-stride waves end on short tiles (LPT order)
  std::stable_sort(b->tiles64.begin(), b->tiles64.end(), [&](const int4& x, const int4& y) {
    return b->h_ooff[x.x + 1] - b->h_ooff[x.x] > b->h_ooff[y.x + 1] - b->h_ooff[y.x];
  });
  put(o_t64, b->tiles64.data(), b->tiles64.size() * sizeof(int4));
  put(o_t128, b->tiles128.data(), b->tiles128.size() * sizeof(int4));
  put(o_t32, b->tiles32.data(), b->tiles32.size() * sizeof(int4));
  put(o_c32, b->chunks32.data(), b->chunks32.size() * sizeof(int2));
  put(o_g64, b->gemm64.data(), b->gemm64.size() * sizeof(int4));
  put(o_g32, b->gemm32.data(), b->gemm32.size() * sizeof(int4));
  std::vector<double> ch(nmol);
  std::vector<int> uh(nmol);
  for (int m = 0; m < nmol; ++m) { ch[m] = mols[m].charge; uh[m] = mols[m].uhf; }
  put(o_charge, ch.data(), NM * D8);
  put(o_uhf, uh.data(), NM * I4);
  // largest structures first: long eigensolves start early, small ones fill in (LPT)
  std::vector<int> order(nmol);
  for (int m = 0; m < nmol; ++m) order[m] = m;
  std::stable_sort(order.begin(), order.end(), [&](int a, int c) {
    return b->h_ooff[a + 1] - b->h_ooff[a] > b->h_ooff[c + 1] - b->h_ooff[c];
  });
  put(o_order, order.data(), NM * I4);
  if (!jlist.empty()) put(o_jlist, jlist.data(), jlist.size() * I4);
  if (!b->trid.list.empty()) put(o_tlist, b->trid.list.data(), b->trid.list.size() * I4);
  TB_CUDA(cudaMemcpy(base, blob, meta_end, cudaMemcpyHostToDevice));

  DevBatch& d = b->db;
  d.nmol = nmol; d.nat_tot = (int)NA; d.nsh_tot = (int)NS; d.nao_tot = (int)NO;
  d.aoff = at<int>(base, o_meta_aoff); d.soff = at<int>(base, o_meta_soff); d.ooff = at<int>(base, o_meta_ooff);
  d.mixoff = at<int>(base, o_meta_mixoff); d.moff = at<long long>(base, o_meta_moff);
  d.poff = at<long long>(base, o_meta_poff);
  d.s2off = at<long long>(base, o_meta_s2off); d.a2off = at<long long>(base, o_meta_a2off);
  b->gtab = at<double>(base, o_gtab); b->atab = at<double>(base, o_atab); d.xyz = at<double>(base, o_xyz); d.id = at<int>(base, o_id);
  d.at_mol = at<int>(base, o_atmol); d.sh_type = at<int>(base, o_shtype); d.sh_at = at<int>(base, o_shat);
  d.sh_iao = at<int>(base, o_shiao); d.at_ish = at<int>(base, o_atish); d.ao_at = at<int>(base, o_aoat);
  d.ao_sh = at<int>(base, o_aosh);
  d.order = at<int>(base, o_order);
  d.lib_above = lib_above;
  d.jacobi_max = jacobi_max;
  d.trid_min = b->trid.trid_min;
  d.trid_max = b->trid.trid_max;
  b->d_jlist = at<int>(base, o_jlist);
  b->d_tlist = at<int>(base, o_tlist);
  b->njac = (int)jlist.size();
  b->lib_work = base + o_lwork;
  b->lib_info = at<int>(base, o_linfo);
  if (b->mixed) {
    b->Af = at<float>(base, o_Af); b->Zf = at<float>(base, o_Zf); b->wf = at<float>(base, o_wf);
    b->Vn = at<double>(base, o_Vn); b->G = at<double>(base, o_G);
    b->act_lo = at<int>(base, o_lo); b->act_hi = at<int>(base, o_hi);
  }
  b->d_tiles64 = at<int4>(base, o_t64); b->d_tiles128 = at<int4>(base, o_t128); b->d_tiles32 = at<int4>(base, o_t32); b->d_chunks32 = at<int2>(base, o_c32);
  b->d_gemm64 = at<int4>(base, o_g64);
  b->d_gemm32 = at<int4>(base, o_g32);
  b->charge = at<double>(base, o_charge); b->uhf = at<int>(base, o_uhf);
  b->d_guess = at<double>(base, o_guess); b->d_guess_flag = at<int>(base, o_gflag);
  b->d_fspin = at<double>(base, o_fspin); b->d_wflag = at<int>(base, o_wflag);
  b->d4cn = at<double>(base, o_d4cn); b->d4w = at<double>(base, o_d4w); b->d4dw = at<double>(base, o_d4dw);
  b->d4e = at<double>(base, o_d4e); b->d4dcn = at<double>(base, o_d4dcn); b->d4g = at<double>(base, o_d4g);
  b->e_disp = at<double>(base, o_edisp);
  b->h_guess.clear();
  b->h_guess_flag.clear();
  b->any_guess = false;
  b->cn = at<double>(base, o_cn); b->mrad = at<double>(base, o_mrad); b->erep = at<double>(base, o_erep);
  b->se = at<double>(base, o_se); b->n0sh = at<double>(base, o_n0sh); b->cnt = at<int>(base, o_cnt);
  b->inl = at<long long>(base, o_inl); b->npair = at<int>(base, o_npair); b->pair_i = at<int>(base, o_pi);
  b->sp_w.cls = at<int>(base, o_spc);
  b->sp_w.rec = at<double>(base, o_X + b->sp_off[0]);
  b->sp_w.list = at<int2>(base, o_X + b->sp_off[1]);
  b->sp_w.idx = at<int>(base, o_X + b->sp_off[2]);
  b->sp_w.tab = at<int>(base, o_X + b->sp_off[3]);
  b->pair_j = at<int>(base, o_pj);
  b->S = at<double>(base, o_S); b->H0 = at<double>(base, o_H0); b->D = at<double>(base, o_D);
  b->Q = at<double>(base, o_Q); b->X = at<double>(base, o_X); b->W = at<double>(base, o_W);
  b->F = at<double>(base, o_F); b->Z = at<double>(base, o_Z); b->P = at<double>(base, o_P);
  b->w = at<double>(base, o_w); b->focc = at<double>(base, o_focc); b->perm = at<int>(base, o_perm);
  b->kdim = at<int>(base, o_kdim); b->vsh = at<double>(base, o_vsh); b->vat = at<double>(base, o_vat);
  b->vdp = at<double>(base, o_vdp); b->vqp = at<double>(base, o_vqp); b->colred = at<double>(base, o_col);
  b->qsh_out = at<double>(base, o_qsho); b->qat_out = at<double>(base, o_qato);
  b->dpat_out = at<double>(base, o_dpo); b->qpat_out = at<double>(base, o_qpo);
  b->q_in = at<double>(base, o_qin); b->dq = at<double>(base, o_dq); b->dqlast = at<double>(base, o_dql);
  b->qlast = at<double>(base, o_ql); b->df = at<double>(base, o_df); b->u = at<double>(base, o_u);
  b->amat = at<double>(base, o_amat); b->omega = at<double>(base, o_om);
  MolState& s = b->ms;
  s.e_rep = at<double>(base, o_ms_erep); s.nel = at<double>(base, o_ms_nel); s.iscf = at<int>(base, o_ms_iscf);
  s.mix_iter = at<int>(base, o_ms_mix); s.eelec = at<double>(base, o_ms_eelec);
  s.active = at<int>(base, o_ms_active); s.status = at<int>(base, o_ms_status);
  s.e_ts = at<double>(base, o_ms_ets); s.e_band = at<double>(base, o_ms_eband);
  s.e_es2 = at<double>(base, o_ms_ees2); s.e_aes2 = at<double>(base, o_ms_eaes2);
  s.e_es3 = at<double>(base, o_ms_ees3); s.scf_error = at<double>(base, o_ms_err);
  s.fermi_warn = at<int>(base, o_ms_fw); s.dipole = at<double>(base, o_ms_dip); s.n_active = at<int>(base, o_ms_nact);
  b->it_dev = at<int>(base, o_itdev);
  s.phase = b->mixed ? at<int>(base, o_phase) : nullptr;
  s.n64 = b->mixed ? at<int>(base, o_n64) : nullptr;
  if (!b->h_nactive) b->h_nactive = calc->take_pin_slot();
  if (!b->h_nactive) TB_CUDA(cudaMallocHost(&b->h_nactive, sizeof(int)));  // pool exhausted
  return TB_OK;
}

inline int nblk(long long n, int t) { return (int)((n + t - 1) / t); }

// ---- kernel-class profiling (CUDA events on the run's stream)
cudaEvent_t prof_event(tb_batch* b) {
  if (b->evused == b->evpool.size()) {
    cudaEvent_t e;
    cudaEventCreate(&e);
    b->evpool.push_back(e);
  }
  return b->evpool[b->evused++];
}
void prof_start(tb_batch* b, cudaStream_t st, cudaEvent_t* e0) {
  if (!b->opt.profile) return;
  *e0 = prof_event(b);
  cudaEventRecord(*e0, st);
}
void prof_stop(tb_batch* b, cudaStream_t st, const char* name, cudaEvent_t e0, double work, int unit) {
  if (!b->opt.profile) return;
  cudaEvent_t e1 = prof_event(b);
  cudaEventRecord(e1, st);
  int idx = -1;
  for (size_t i = 0; i < b->kclass.size(); ++i)
    if (b->kclass[i].name == name) idx = (int)i;
  if (idx < 0) {
    b->kclass.push_back({});
    idx = (int)b->kclass.size() - 1;
    b->kclass[idx].name = name;
    b->kclass[idx].unit = unit;
  }
  b->kclass[idx].launches += 1;
  b->kclass[idx].work += work;
  b->pend.push_back({idx, {e0, e1}});
}
tb_status prof_collect(tb_batch* b, cudaStream_t st) {
  if (!b->opt.profile) return TB_OK;
  TB_CUDA(cudaStreamSynchronize(st));
  for (auto& p : b->pend) {
    float ms = 0.f;
    TB_CUDA(cudaEventElapsedTime(&ms, p.second.first, p.second.second));
    b->kclass[p.first].ms += ms;
  }
  b->pend.clear();
  return TB_OK;
}

// launch + error check + profile record of one kernel class
#define TB_K(name, work, unit, ...)            \
  do {                                         \
    cudaEvent_t e0_ = nullptr;                 \
    prof_start(b, st, &e0_);                   \
    __VA_ARGS__;                               \
    TB_LAUNCH_CHECK();                         \
    prof_stop(b, st, name, e0_, work, unit);   \
  } while (0)

#define TB_LAUNCH_CHECK()                                                                  \
  do {                                                                                     \
    cudaError_t e_ = cudaGetLastError();                                                   \
    if (e_ != cudaSuccess) return fail(TB_CUDA_ERROR, std::string("launch: ") + cudaGetErrorString(e_)); \
    ++b->launches;                                                                         \
  } while (0)

// k_trid_smem for the structures of the batch's plan (one launch per class;
// timed with k_syev in the "syev" class), before k_syev
tb_status launch_trid_plan(tb_batch* b, const int* active, cudaStream_t st) {
  const TridPlan& tp = b->trid;
  for (int c = 0; c < kTridClasses; ++c) {
    const int cnt = tp.off[c + 1] - tp.off[c];
    if (cnt == 0) continue;
    cudaEvent_t e0 = nullptr;
    prof_start(b, st, &e0);
    const cudaError_t e = launch_trid(b->db, b->F, b->W, b->ms.status, active, b->d_tlist + tp.off[c], cnt,
                                      kTridClusterSizes[c], tp.nmax[c], st);
    if (e != cudaSuccess) return fail(TB_CUDA_ERROR, std::string("k_trid_smem: ") + cudaGetErrorString(e));
    ++b->launches;
    prof_stop(b, st, "syev", e0, 0.0, 1);
  }
  return TB_OK;
}

// One batched FP64 GEMM (k_gemm's operands) over the batch's two GEMM tile
// lists: k_gemm on the structures given 64 x 64 tiles, k_gemm32 on those given
// 32 x 32 (the same bits either way).  One CTA per tile: the block scheduler
// hands the tiles, largest structures first, to SMs as they free up, which
// balances tiles of very different K better than a fixed grid stride.  With
// a profile name both launches are timed in that class and the algorithmic
// work is booked once.
tb_status launch_gemm(tb_batch* b, cudaStream_t st, const char* prof, double work, const double* A, int ta,
                      const double* Bm, int tb_, const int* perm, const double* ks, const int* kdim, double* C,
                      double alpha, double beta, const int* active, int shape) {
  bool booked = false;
  for (int v = 0; v < 2; ++v) {
    const int nt = v ? b->ngemm32 : b->ngemm64;
    if (nt == 0) continue;
    cudaEvent_t e0 = nullptr;
    if (prof) prof_start(b, st, &e0);
    if (v == 0)
      k_gemm<<<nt, kGemmThreads, 0, st>>>(b->db, b->d_gemm64, nt, A, ta, Bm, tb_, perm, ks, kdim, C, alpha, beta,
                                          active, shape);
    else
      k_gemm32<<<nt, kGemmThreads, 0, st>>>(b->db, b->d_gemm32, nt, A, ta, Bm, tb_, perm, ks, kdim, C, alpha, beta,
                                            active, shape);
    TB_LAUNCH_CHECK();
    if (prof) prof_stop(b, st, prof, e0, booked ? 0.0 : work, 1);
    booked = true;
  }
  return TB_OK;
}
#define TB_GEMM(work, ...)                                                  \
  do {                                                                      \
    const tb_status gs_ = launch_gemm(b, st, "gemm", work, __VA_ARGS__);   \
    if (gs_ != TB_OK) return gs_;                                           \
  } while (0)

// The mixed phase hands over to FP64 once |dE| and the charge error are below
// this multiple of the final thresholds, but never below the floors: the FP32
// contractions leave iteration-to-iteration noise of about 1e-6 in charges.
constexpr double kMixedSwitchScale = 10.0, kMixedSwitchFloorE = 1e-5, kMixedSwitchFloorQ = 2e-4;

// Eigen-decomposition and density of one SCF iteration in the mixed-precision
// form (tb_mixed.cu).  Every matrix is stored in FP64.  Structures in the
// mixed phase: F', C and P as TF32x3 tensor-core GEMMs (k_gemm_tc, tcgen05),
// eigenpairs from the FP32 eigensolver and one FP64 Ogita-Aishima refinement
// step.  Structures in the FP64 phase (the final iterations) run the plain
// form's FP64 iteration: FP64 GEMMs and the FP64 eigensolver, so the
// converged result carries no FP32 error.  Leaves w, focc, kdim and P as the
// plain form does.
tb_status mixed_core(tb_batch* b, cudaStream_t st, double n3_lo, double n3_hi, double n2occ_lo, double n2occ_hi,
                     int gemm_grid, size_t fermi_smem) {
  const DevBatch& B = b->db;
  MolState& S = b->ms;
  const int nmol = b->nmol, nt = (int)b->tiles64.size();
  const int4* T = b->d_tiles64;
  const size_t smem32 = syev_smem_bytes(std::max(b->nmax_in, 1), sizeof(float));
  const size_t eig_smem = syev_smem_bytes(std::max(b->nmax_in, 1));
  int *lo = b->act_lo, *hi = b->act_hi;
  const int nt128 = (int)b->tiles128.size(), tc_grid = std::min(nt128, 148);
  const int4* T128 = b->d_tiles128;
  const size_t tc_smem = gemm_tc_smem_bytes();
  TB_K("masks", 0, 0, k_phase_masks<<<nblk(nmol, 256), 256, 0, st>>>(nmol, S.active, S.phase, lo, hi));
  // F' = X^T F X into F (T = F X in W), each phase in its precision
  TB_K("gemm_tc", 2.0 * n3_lo, 1,
       k_gemm_tc<<<tc_grid, kTcThreads, tc_smem, st>>>(B, T128, nt128, b->F, 0, b->X, 0, nullptr, nullptr, nullptr, b->W, 1.0, 0.0, lo, S.status));
  TB_GEMM(2.0 * n3_hi, b->F, 0, b->X, 0, nullptr, nullptr, nullptr, b->W, 1.0, 0.0, hi, kGemmKUpToJ);
  TB_K("gemm_tc", 2.0 * n3_lo, 1,
       k_gemm_tc<<<tc_grid, kTcThreads, tc_smem, st>>>(B, T128, nt128, b->X, 1, b->W, 0, nullptr, nullptr, nullptr, b->F, 1.0, 0.0, lo, S.status));
  TB_GEMM(2.0 * n3_hi, b->X, 1, b->W, 0, nullptr, nullptr, nullptr, b->F, 1.0, 0.0, hi, kGemmKUpToI | kGemmSym);
  // mixed phase: FP32 eigensolve
  TB_K("convert", 0, 0, k_to_f32<<<gemm_grid, 256, 0, st>>>(B, T, nt, b->F, b->Af, lo));
  TB_K("syev_f32", 4.0 * n3_lo, 1,
       k_syev_f32<<<nmol, kEigThreads, smem32, st>>>(B, b->Af, b->Zf, b->w, b->perm, S.status, lo));
  // FP64 phase: the FP64 eigensolver (eigenvectors as rows of Z, W as its scratch)
  {
    const tb_status ts = launch_trid_plan(b, hi, st);
    if (ts != TB_OK) return ts;
  }
  TB_K("syev", 4.0 * n3_hi, 1,
       k_syev<<<nmol, kEigThreads, eig_smem, st>>>(B, b->F, b->Z, b->W, b->w, b->perm, S.status, hi));
  if (b->njac > 0)
    TB_K("syev_jacobi", 0, 0,
         k_syev_jacobi<<<nblk(b->njac, kJacobiWarps), kJacobiWarps * 32, jacobi_smem_bytes(), st>>>(
             B, b->F, b->Z, b->w, b->perm, S.status, hi, b->d_jlist, b->njac));
  for (size_t k = 0; k < b->big.size(); ++k) {
    const int m = b->big[k], n = b->h_ooff[m + 1] - b->h_ooff[m];
    if (!b->h_active[m] || b->h_status[m] != kStOk) continue;
    const long long mo = b->h_moff[m], vo = b->h_ooff[m];
    cudaEvent_t e0 = nullptr;
    prof_start(b, st, &e0);
    std::string e;
    if (b->h_phase[m] == 0)
      e = b->lib.syev32(st, b->Af + mo, b->Zf + mo, b->wf + vo, b->w + vo, b->perm + vo, n, b->lib_work,
                        b->lib_bytes, b->lib_info + 2 * k, S.status + m);
    else
      e = b->lib.syev(st, b->F + mo, b->Z + mo, b->w + vo, b->perm + vo, n, b->lib_work, b->lib_bytes,
                      b->lib_info + 2 * k, S.status + m);
    if (!e.empty()) return fail(TB_CUDA_ERROR, "library eigensolver: " + e);
    ++b->launches;
    prof_stop(b, st, b->h_phase[m] == 0 ? "syev_lib_f32" : "syev_lib", e0, 4.0 * n * n * n, 1);
  }
  // mixed phase: one FP64 refinement step (GEMMs included) of the FP32
  // eigenvectors, gathered into FP64 columns in ascending order (Z -> Vn)
  const size_t oa_smem = oa_smem_bytes(b->nmax);
  TB_K("refine", 0, 0, k_gather_vectors<<<gemm_grid, 256, 0, st>>>(B, T, nt, b->Zf, b->perm, b->Z, lo));
  {
    double* V = b->Z;
    double* Vo = b->Vn;
    const double wk = 2.0 * n3_lo;
    TB_GEMM(wk,  // G = V^T V
            V, 1, V, 0, nullptr, nullptr, nullptr, b->G, 1.0, 0.0, lo, 0);
    TB_GEMM(wk,  // W = F' V
            b->F, 0, V, 0, nullptr, nullptr, nullptr, b->W, 1.0, 0.0, lo, 0);
    TB_GEMM(wk,  // Sm = V^T W (in P)
            V, 1, b->W, 0, nullptr, nullptr, nullptr, b->P, 1.0, 0.0, lo, 0);
    TB_K("refine", 0, 0, k_oa_step<<<nmol, 256, oa_smem, st>>>(B, b->G, b->P, V, b->w, lo, nullptr));
    TB_CUDA(cudaMemcpyAsync(Vo, V, (size_t)b->n2_tot * sizeof(double), cudaMemcpyDeviceToDevice, st));
    TB_GEMM(wk,  // Vo = V + V E
            V, 0, b->G, 0, nullptr, nullptr, nullptr, Vo, 1.0, 1.0, lo, 0);
  }
  TB_K("fermi", 0, 0, k_fermi<<<nmol, 128, fermi_smem, st>>>(B, b->w, b->opt.kt, b->focc, b->kdim, S));
  // C = X V into W (mixed phase: V after the refinement step, in Vn; FP64
  // phase: the eigenvector rows of Z in ascending order through perm)
  TB_K("gemm_tc", 2.0 * n3_lo, 1,
       k_gemm_tc<<<tc_grid, kTcThreads, tc_smem, st>>>(B, T128, nt128, b->X, 0, b->Vn, 0, nullptr, nullptr, nullptr, b->W, 1.0, 0.0, lo, S.status));
  TB_GEMM(2.0 * n3_hi, b->X, 0, b->Z, 1, b->perm, nullptr, nullptr, b->W, 1.0, 0.0, hi, kGemmKFromI);
  // P = C diag(f) C^T
  TB_K("gemm_tc", 2.0 * n2occ_lo, 1,
       k_gemm_tc<<<tc_grid, kTcThreads, tc_smem, st>>>(B, T128, nt128, b->W, 0, b->W, 1, nullptr, b->focc, b->kdim, b->P, 1.0, 0.0, lo, S.status));
  TB_GEMM(2.0 * n2occ_hi, b->W, 0, b->W, 1, nullptr, b->focc, b->kdim, b->P, 1.0, 0.0, hi, kGemmSym);
  return TB_OK;
}

// Dynamic shared memory of the one-CTA-per-structure kernels grows with N.
// The opt-in limit is a per-kernel attribute shared by every batch of the
// process (batches of different sizes can be resident at once), so it is
// raised once to the device maximum rather than set per batch.
tb_status raise_smem_limits() {
  int dev = 0, optin = 0;
  TB_CUDA(cudaGetDevice(&dev));
  TB_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  const void* ks[] = {(const void*)k_syev, (const void*)k_syev_f32, (const void*)k_fermi, (const void*)k_oa_step,
                      (const void*)k_gemm_tc, (const void*)k_fock, (const void*)k_syev_jacobi};
  for (const void* k : ks) {
    cudaFuncAttributes a;
    TB_CUDA(cudaFuncGetAttributes(&a, k));
    TB_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, optin - (int)a.sharedSizeBytes));
  }
  TB_CUDA(trid_raise_limits());
  return TB_OK;
}

// Measures the two eigensolvers once per calculator: the in-house k_syev on
// one structure (latency, at 256 and 512 AOs, fitted by a N^2 + b N^3) and one
// cuSOLVER syevd call (at 256 and 1024 AOs, fitted by c + d N^3), on
// deterministic random symmetric matrices.
tb_status calibrate_eigensolvers(tb_calculator* c) {
  std::lock_guard<std::mutex> lk(c->tune_mu);
  if (c->eig.ready) return TB_OK;
  {
    const tb_status ss = raise_smem_limits();
    if (ss != TB_OK) return ss;
  }
  const int NL = 1024;
  Arena ar;
  const size_t nn = (size_t)NL * NL;
  LargeSolver ls;
  size_t wbytes = 0;
  const std::string we = ls.workspace(NL, &wbytes);
  if (!we.empty()) return fail(TB_CUDA_ERROR, "eigensolver calibration: " + we);
  Layout L;
  const size_t oA = L.add(nn * 8), oZ = L.add(nn * 8), oW = L.add(nn * 8), ow = L.add(NL * 8), op = L.add(NL * 4), os = L.add(16),
               oo = L.add(16), om = L.add(16), owk = L.add(std::max<size_t>(wbytes, 16)), oi = L.add(16),
               ol = L.add(16);
  TB_CUDA(ar.reserve(L.total));
  char* base = ar.base;
  std::vector<double> h(nn);
  uint64_t x = 0x9e3779b97f4a7c15ull;
  auto rnd = [&]() {  // xorshift64*, uniform in (-1, 1)
    x ^= x >> 12; x ^= x << 25; x ^= x >> 27;
    return (double)((x * 0x2545f4914f6cdd1dull) >> 11) * (2.0 / 9007199254740992.0) - 1.0;
  };
  cudaEvent_t e0, e1;
  TB_CUDA(cudaEventCreate(&e0));
  TB_CUDA(cudaEventCreate(&e1));
  auto upload = [&](int n) -> tb_status {
    for (int i = 0; i < n; ++i)
      for (int j = 0; j <= i; ++j) h[(size_t)i * n + j] = h[(size_t)j * n + i] = rnd() / std::sqrt((double)n);
    TB_CUDA(cudaMemcpy(base + oA, h.data(), (size_t)n * n * 8, cudaMemcpyHostToDevice));
    const int oo_h[2] = {0, n};
    const long long om_h[2] = {0, (long long)n * n};
    TB_CUDA(cudaMemcpy(base + oo, oo_h, 8, cudaMemcpyHostToDevice));
    TB_CUDA(cudaMemcpy(base + om, om_h, 16, cudaMemcpyHostToDevice));
    TB_CUDA(cudaMemset(base + os, 0, 16));
    return TB_OK;
  };
  auto inhouse = [&](int n, double* sec) -> tb_status {
    DevBatch B{};
    B.nmol = 1;
    B.ooff = at<int>(base, oo);
    B.moff = at<long long>(base, om);
    TridPlan tp;  // the eigensolver as a batch runs it
    tp.build({n}, {1}, c->smem_tridiag);
    B.trid_min = tp.trid_min;
    B.trid_max = tp.trid_max;
    TB_CUDA(cudaMemset(base + ol, 0, 16));
    float ms = 0.f;
    for (int rep = 0; rep < 2; ++rep) {
      const tb_status us = upload(n);
      if (us != TB_OK) return us;
      TB_CUDA(cudaEventRecord(e0));
      for (int cl = 0; cl < kTridClasses; ++cl)
        if (tp.off[cl + 1] > tp.off[cl])
          TB_CUDA(launch_trid(B, at<double>(base, oA), at<double>(base, oW), at<int>(base, os), nullptr,
                              at<int>(base, ol), 1, kTridClusterSizes[cl], n, 0));
      k_syev<<<1, kEigThreads, syev_smem_bytes(n)>>>(B, at<double>(base, oA), at<double>(base, oZ),
                                                     at<double>(base, oW), at<double>(base, ow), at<int>(base, op),
                                                     at<int>(base, os), nullptr);
      TB_CUDA(cudaEventRecord(e1));
      TB_CUDA(cudaEventSynchronize(e1));
      TB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    }
    *sec = ms * 1e-3;
    return TB_OK;
  };
  auto library = [&](int n, double* sec) -> tb_status {
    float ms = 0.f;
    for (int rep = 0; rep < 2; ++rep) {
      const tb_status us = upload(n);
      if (us != TB_OK) return us;
      TB_CUDA(cudaEventRecord(e0));
      const std::string e = ls.syev(0, at<double>(base, oA), at<double>(base, oZ), at<double>(base, ow),
                                    at<int>(base, op), n, base + owk, wbytes, at<int>(base, oi), at<int>(base, os));
      if (!e.empty()) return fail(TB_CUDA_ERROR, "eigensolver calibration: " + e);
      TB_CUDA(cudaEventRecord(e1));
      TB_CUDA(cudaEventSynchronize(e1));
      TB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    }
    *sec = ms * 1e-3;
    return TB_OK;
  };
  double t1 = 0, t2 = 0, l1 = 0, l2 = 0;
  tb_status st = inhouse(256, &t1);
  if (st == TB_OK) st = inhouse(512, &t2);
  if (st == TB_OK) st = library(256, &l1);
  if (st == TB_OK) st = library(NL, &l2);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st != TB_OK) return st;
  // t = a n^2 + b n^3 through (256, t1), (512, t2); t = c + d n^3 through (256, l1), (1024, l2)
  const double n1 = 256, n2 = 512, m1 = 256, m2 = NL;
  const double det = n1 * n1 * n2 * n2 * n2 - n2 * n2 * n1 * n1 * n1;
  c->eig.a = std::max(0.0, (t1 * n2 * n2 * n2 - t2 * n1 * n1 * n1) / det);
  c->eig.b = std::max(0.0, (n1 * n1 * t2 - n2 * n2 * t1) / det);
  c->eig.d = std::max(0.0, (l2 - l1) / (m2 * m2 * m2 - m1 * m1 * m1));
  c->eig.c = std::max(0.0, l1 - c->eig.d * m1 * m1 * m1);
  c->eig.t_in[0] = t1; c->eig.t_in[1] = t2;
  c->eig.t_lib[0] = l1; c->eig.t_lib[1] = l2;
  c->eig.ready = true;
  return TB_OK;
}

// Measures, once per calculator, the batched throughput of the one-CTA
// eigensolver (k_syev, implicit QL below 64 AOs) and the one-warp Jacobi
// variant (k_syev_jacobi) at N = 8, 12, ..., 32: 592 deterministic random
// symmetric matrices per size (four per SM), the same inputs for both, the
// faster of two timed launches each.  The warp variant is chosen up to the
// largest N below which it is faster at every measured size.
tb_status calibrate_small(tb_calculator* c) {
  std::lock_guard<std::mutex> lk(c->tune_mu);
  if (c->small.ready) return TB_OK;
  {
    const tb_status ss = raise_smem_limits();
    if (ss != TB_OK) return ss;
  }
  const int cnt = 592, NM = kJacobiMaxN;
  const size_t nn = (size_t)cnt * NM * NM;
  Arena ar;
  Layout L;
  const size_t oA0 = L.add(nn * 8), oA = L.add(nn * 8), oZ = L.add(nn * 8), oW = L.add(nn * 8),
               ow = L.add((size_t)cnt * NM * 8), op = L.add((size_t)cnt * NM * 4), os = L.add(cnt * 4),
               oo = L.add((cnt + 1) * 4), om = L.add((cnt + 1) * 8), ol = L.add(cnt * 4);
  TB_CUDA(ar.reserve(L.total));
  char* base = ar.base;
  std::vector<double> h(nn);
  std::vector<int> oo_h(cnt + 1), list(cnt);
  std::vector<long long> om_h(cnt + 1);
  uint64_t x = 0x2545f4914f6cdd1dull;
  auto rnd = [&]() {  // xorshift64*, uniform in (-1, 1)
    x ^= x >> 12; x ^= x << 25; x ^= x >> 27;
    return (double)((x * 0x2545f4914f6cdd1dull) >> 11) * (2.0 / 9007199254740992.0) - 1.0;
  };
  for (int i = 0; i < cnt; ++i) list[i] = i;
  TB_CUDA(cudaMemcpy(base + ol, list.data(), cnt * 4, cudaMemcpyHostToDevice));
  cudaEvent_t e0, e1;
  TB_CUDA(cudaEventCreate(&e0));
  TB_CUDA(cudaEventCreate(&e1));
  tb_status st = TB_OK;
  std::vector<int> sizes = {8, 12, 16, 20, 24, 28, 32};
  std::vector<double> tc(sizes.size()), tw(sizes.size());
  for (size_t si = 0; si < sizes.size() && st == TB_OK; ++si) {
    const int n = sizes[si];
    for (int k = 0; k < cnt; ++k) {
      oo_h[k] = k * n;
      om_h[k] = (long long)k * n * n;
      double* M = h.data() + (size_t)k * n * n;
      for (int i = 0; i < n; ++i)
        for (int j = 0; j <= i; ++j) M[(size_t)i * n + j] = M[(size_t)j * n + i] = rnd();
    }
    oo_h[cnt] = cnt * n;
    om_h[cnt] = (long long)cnt * n * n;
    const size_t bytes = (size_t)cnt * n * n * 8;
    if (cudaMemcpy(base + oA0, h.data(), bytes, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(base + oo, oo_h.data(), (cnt + 1) * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(base + om, om_h.data(), (cnt + 1) * 8, cudaMemcpyHostToDevice) != cudaSuccess) {
      st = fail(TB_CUDA_ERROR, "small eigensolver calibration: upload");
      break;
    }
    DevBatch Bk{};
    Bk.nmol = cnt;
    Bk.ooff = at<int>(base, oo);
    Bk.moff = at<long long>(base, om);
    float best[2] = {1e30f, 1e30f};
    for (int variant = 0; variant < 2; ++variant)
      for (int rep = 0; rep < 2; ++rep) {
        cudaMemcpy(base + oA, base + oA0, bytes, cudaMemcpyDeviceToDevice);
        cudaMemset(base + os, 0, cnt * 4);
        cudaEventRecord(e0);
        if (variant == 0)
          k_syev<<<cnt, kEigThreads, syev_smem_bytes(n)>>>(Bk, at<double>(base, oA), at<double>(base, oZ),
                                                           at<double>(base, oW), at<double>(base, ow),
                                                           at<int>(base, op), at<int>(base, os), nullptr);
        else
          k_syev_jacobi<<<nblk(cnt, kJacobiWarps), kJacobiWarps * 32, jacobi_smem_bytes()>>>(
              Bk, at<double>(base, oA), at<double>(base, oZ), at<double>(base, ow), at<int>(base, op),
              at<int>(base, os), nullptr, at<int>(base, ol), cnt);
        cudaEventRecord(e1);
        float ms = 0.f;
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess ||
            cudaGetLastError() != cudaSuccess) {
          st = fail(TB_CUDA_ERROR, "small eigensolver calibration: launch");
          break;
        }
        best[variant] = std::min(best[variant], ms);
      }
    tc[si] = best[0] * 1e-3 / cnt;
    tw[si] = best[1] * 1e-3 / cnt;
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st != TB_OK) return st;
  int jmax = 0;
  for (size_t si = 0; si < sizes.size() && tw[si] < tc[si]; ++si) jmax = sizes[si];
  c->small.n = sizes;
  c->small.t_cta = tc;
  c->small.t_warp = tw;
  c->small.jacobi_max = jmax;
  c->small.ready = true;
  return TB_OK;
}

// Measures, once per calculator, the batched FP64 GEMM on both tile shapes
// (k_gemm, 64 x 64; k_gemm32, 32 x 32) at N = 16, 32, ..., kTileCalMax: the
// SCF iteration's four GEMM forms (F X with X upper triangular, X^T W into a
// symmetric result, X Z through a permutation, W diag(f) W^T over the occupied
// columns), each on floor(E / N^2) structures of N AOs (E = two waves of
// 64 x 64 tiles on 148 SMs), the same inputs for both shapes, the faster of
// two timed repetitions after an untimed one.  32 x 32 tiles are chosen at
// the sizes where they were faster; both shapes give the same bits.
tb_status calibrate_tiles(tb_calculator* c) {
  std::lock_guard<std::mutex> lk(c->tune_mu);
  if (c->tile.ready) return TB_OK;
  const size_t E = 2ull * 148 * 8 * 64 * 64;  // matrix elements per size
  const int cmax = (int)(E / (16 * 16));      // structures at the smallest size
  Arena ar;
  Layout L;
  const size_t oA = L.add(E * 8), oB = L.add(E * 8), oC = L.add(E * 8), oK = L.add(E / 16 * 8),
               oP = L.add(E / 16 * 4), oD = L.add((size_t)cmax * 4), oo = L.add((size_t)(cmax + 1) * 4),
               om = L.add((size_t)(cmax + 1) * 8), oT = L.add((E / 256 + 1) * sizeof(int4));
  TB_CUDA(ar.reserve(L.total));
  char* base = ar.base;
  {
    std::vector<double> h(E);
    uint64_t x = 0x9e3779b97f4a7c15ull;
    for (size_t i = 0; i < E; ++i) {  // xorshift64*, uniform in (-1, 1)
      x ^= x >> 12; x ^= x << 25; x ^= x >> 27;
      h[i] = (double)((x * 0x2545f4914f6cdd1dull) >> 11) * (2.0 / 9007199254740992.0) - 1.0;
    }
    TB_CUDA(cudaMemcpy(base + oA, h.data(), E * 8, cudaMemcpyHostToDevice));
    TB_CUDA(cudaMemcpy(base + oB, h.data(), E * 8, cudaMemcpyHostToDevice));
    h.assign(E / 16, 0.5);
    TB_CUDA(cudaMemcpy(base + oK, h.data(), E / 16 * 8, cudaMemcpyHostToDevice));
  }
  const double* A = at<double>(base, oA);
  const double* Bm = at<double>(base, oB);
  double* C = at<double>(base, oC);
  const double* ks = at<double>(base, oK);
  const int* perm = at<int>(base, oP);
  const int* kdim = at<int>(base, oD);
  int4* dT = at<int4>(base, oT);
  cudaEvent_t e0, e1;
  TB_CUDA(cudaEventCreate(&e0));
  TB_CUDA(cudaEventCreate(&e1));
  tb_status st = TB_OK;
  std::vector<int> sizes;
  for (int n = 16; n <= kTileCalMax; n += 16) sizes.push_back(n);
  std::vector<double> t64(sizes.size()), t32(sizes.size());
  std::vector<int> oo_h, pm_h, kd_h;
  std::vector<long long> om_h;
  std::vector<int4> tl;
  for (size_t si = 0; si < sizes.size() && st == TB_OK; ++si) {
    const int n = sizes[si], cnt = (int)std::max<size_t>(1, E / ((size_t)n * n));
    oo_h.resize(cnt + 1);
    om_h.resize(cnt + 1);
    pm_h.resize((size_t)cnt * n);
    kd_h.assign(cnt, n / 2);
    for (int k = 0; k <= cnt; ++k) {
      oo_h[k] = k * n;
      om_h[k] = (long long)k * n * n;
    }
    for (int k = 0; k < cnt; ++k)
      for (int j = 0; j < n; ++j) pm_h[(size_t)k * n + j] = j;
    if (cudaMemcpy(base + oo, oo_h.data(), (cnt + 1) * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(base + om, om_h.data(), (cnt + 1) * 8, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(base + oP, pm_h.data(), (size_t)cnt * n * 4, cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemcpy(base + oD, kd_h.data(), (size_t)cnt * 4, cudaMemcpyHostToDevice) != cudaSuccess) {
      st = fail(TB_CUDA_ERROR, "GEMM tile calibration: upload");
      break;
    }
    DevBatch Bk{};
    Bk.nmol = cnt;
    Bk.ooff = at<int>(base, oo);
    Bk.moff = at<long long>(base, om);
    for (int v = 0; v < 2 && st == TB_OK; ++v) {
      const int tile = v ? 32 : 64, nt1 = (n + tile - 1) / tile;
      tl.clear();
      for (int m = 0; m < cnt; ++m)
        for (int t = 0; t < nt1; ++t)
          for (int u = 0; u < nt1; ++u) tl.push_back(make_int4(m, t, u, 0));
      const int nt = (int)tl.size(), grid = nt;  // one CTA per tile, as launch_gemm
      if (cudaMemcpy(dT, tl.data(), tl.size() * sizeof(int4), cudaMemcpyHostToDevice) != cudaSuccess) {
        st = fail(TB_CUDA_ERROR, "GEMM tile calibration: upload");
        break;
      }
      auto launch = [&](const double* a, int ta, const double* bb, int tb_, const int* pm, const double* kv,
                        const int* kd, int shape) {
        if (v == 0)
          k_gemm<<<grid, kGemmThreads>>>(Bk, dT, nt, a, ta, bb, tb_, pm, kv, kd, C, 1.0, 0.0, nullptr, shape);
        else
          k_gemm32<<<grid, kGemmThreads>>>(Bk, dT, nt, a, ta, bb, tb_, pm, kv, kd, C, 1.0, 0.0, nullptr, shape);
      };
      float best = 1e30f;
      for (int rep = 0; rep < 3; ++rep) {
        cudaEventRecord(e0);
        launch(A, 0, Bm, 0, nullptr, nullptr, nullptr, kGemmKUpToJ);
        launch(A, 1, Bm, 0, nullptr, nullptr, nullptr, kGemmKUpToI | kGemmSym);
        launch(A, 0, Bm, 1, perm, nullptr, nullptr, kGemmKFromI);
        launch(A, 0, A, 1, nullptr, ks, kdim, kGemmSym);
        cudaEventRecord(e1);
        float ms = 0.f;
        if (cudaEventSynchronize(e1) != cudaSuccess || cudaEventElapsedTime(&ms, e0, e1) != cudaSuccess ||
            cudaGetLastError() != cudaSuccess) {
          st = fail(TB_CUDA_ERROR, "GEMM tile calibration: launch");
          break;
        }
        if (rep > 0) best = std::min(best, ms);
      }
      (v ? t32 : t64)[si] = best * 1e-3 / cnt;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (st != TB_OK) return st;
  c->tile.n = sizes;
  c->tile.t64 = t64;
  c->tile.t32 = t32;
  c->tile.use32.resize(sizes.size());
  for (size_t si = 0; si < sizes.size(); ++si) c->tile.use32[si] = t32[si] < t64[si];
  c->tile.ready = true;
  return TB_OK;
}

// Host copy of active/status, read where a run synchronises anyway, so that
// converged or failed library structures are not diagonalised again.
tb_status read_flags(tb_batch* b, cudaStream_t st) {
  if (b->big.empty()) return TB_OK;
  const int nmol = b->nmol;
  b->h_active.resize(nmol);
  b->h_status.resize(nmol);
  TB_CUDA(cudaMemcpyAsync(b->h_active.data(), b->ms.active, nmol * sizeof(int), cudaMemcpyDeviceToHost, st));
  TB_CUDA(cudaMemcpyAsync(b->h_status.data(), b->ms.status, nmol * sizeof(int), cudaMemcpyDeviceToHost, st));
  b->h_phase.assign(nmol, 0);
  if (b->mixed)
    TB_CUDA(cudaMemcpyAsync(b->h_phase.data(), b->ms.phase, nmol * sizeof(int), cudaMemcpyDeviceToHost, st));
  TB_CUDA(cudaStreamSynchronize(st));
  return TB_OK;
}

// Setup of a run: status reset, per-structure setup kernels (CN, neighbour
// list, integrals, S = L L^T and X = L^-T) and the SCF start (k_scf_init).
tb_status batch_setup(tb_batch* b, cudaStream_t st) {
  NvtxRange nv("tb.setup");
  tb_calculator* c = b->calc;
  const DevBatch& B = b->db;
  MolState& S = b->ms;
  const int nmol = b->nmol;
  b->launches = 0;
  b->kclass.clear();
  b->pend.clear();
  b->evused = 0;
  b->Pc = c->dp;
  DevParams& Pc = b->Pc;
  Pc.intcut = integral_cutoff(b->opt.accuracy);
  Pc.cutoff = std::min(std::sqrt(2.0 * Pc.intcut / c->hp.min_alpha), 40.0);  // get_cutoff, src/basis/type.cu:43-64
  b->it = 0;
  TB_CUDA(cudaMemsetAsync(S.status, 0, nmol * sizeof(int), st));
  TB_CUDA(cudaMemsetAsync(S.fermi_warn, 0, nmol * sizeof(int), st));
  TB_CUDA(cudaMemsetAsync(S.n_active, 0, sizeof(int), st));
  TB_CUDA(cudaMemsetAsync(b->kdim, 0, nmol * sizeof(int), st));  // no occupied orbitals before k_fermi
  // ---- setup (once per structure)
  TB_K("atoms", 0, 0, k_atoms<<<nblk(B.nat_tot, 128), 128, 0, st>>>(Pc, B, b->cn, b->mrad, b->erep, b->se));
  // D4 dispersion of the fixed geometry (dispersion_get_engrad, src/xtb.cu:274-277)
  if (Pc.d4) {
    cudaEvent_t e0 = nullptr;
    prof_start(b, st, &e0);
    TB_CUDA(launch_dispersion(Pc, B, nmol, b->d4cn, b->d4w, b->d4dw, b->d4e, b->d4dcn, b->d4g, b->e_disp, st));
    b->launches += 5;
    prof_stop(b, st, "dispersion", e0, 0, 0);
  } else {
    TB_CUDA(cudaMemsetAsync(b->e_disp, 0, nmol * sizeof(double), st));
  }
  {
    const long long mx = std::max((long long)b->nshmax * b->nshmax, (long long)b->natmax * b->natmax);
    TB_K("pair_tables", 0, 0,
         k_pair_tables<<<dim3(nmol, (unsigned)std::min<long long>(nblk(mx, 256), 64)), 256, 0, st>>>(
             Pc, B, b->mrad, b->gtab, b->atab));
  }
  TB_K("adjacency", 0, 0,
       k_adj_count<<<nblk((long long)B.nat_tot * 32, 256), 256, 0, st>>>(B, Pc.cutoff, b->cnt);
       TB_LAUNCH_CHECK();
       k_adj_scan<<<nmol, 256, 0, st>>>(B, b->cnt, b->inl, b->npair);
       TB_LAUNCH_CHECK();
       k_adj_fill<<<nblk((long long)B.nat_tot * 32, 256), 256, 0, st>>>(B, Pc.cutoff, b->inl, b->pair_i, b->pair_j));
  // S, H0, D, Q: every element is written by the integral setup (zeros included)
  {
    MatOut out{b->S, b->H0, b->D, b->Q};
    const int maxsp = c->maxsh * c->maxsh;
    cudaEvent_t e0 = nullptr;
    prof_start(b, st, &e0);
    TB_CUDA(launch_integrals(Pc, B, b->npair, b->pair_i, b->pair_j, b->se, out, maxsp, b->pair_cap, c->lmask,
                             b->sp_w, st, &b->launches));
    prof_stop(b, st, "integrals", e0, 0, 0);
  }
  TB_K("cholesky", 0, 0, k_cholesky<<<nmol, 256, 0, st>>>(B, b->S, b->W, S.status, nullptr));
  TB_K("trinv", 0, 0, k_trinv<<<nmol, 256, 0, st>>>(B, b->W, b->X, S.status));
  for (size_t k = 0; k < b->big.size(); ++k) {
    const int m = b->big[k], n = b->h_ooff[m + 1] - b->h_ooff[m];
    const long long mo = b->h_moff[m];
    cudaEvent_t e0 = nullptr;
    prof_start(b, st, &e0);
    const std::string e = b->lib.factor(st, b->S + mo, b->X + mo, n, b->lib_work, b->lib_bytes, b->lib_info + 2 * k,
                                        S.status + m);
    if (!e.empty()) return fail(TB_CUDA_ERROR, "library Cholesky: " + e);
    ++b->launches;
    prof_stop(b, st, "factor_lib", e0, 0, 0);
  }
  TB_K("scf_init", 0, 0, k_scf_init<<<nmol, 256, 0, st>>>(Pc, B, b->charge, b->uhf, b->erep, b->n0sh, b->q_in, S));
  if (b->any_guess) {
    TB_CUDA(cudaMemcpyAsync(b->d_guess, b->h_guess.data(), b->h_guess.size() * sizeof(double),
                            cudaMemcpyHostToDevice, st));
    TB_CUDA(cudaMemcpyAsync(b->d_guess_flag, b->h_guess_flag.data(), nmol * sizeof(int), cudaMemcpyHostToDevice,
                            st));
    TB_K("scf_init", 0, 0, k_apply_guess<<<nmol, 256, 0, st>>>(B, b->d_guess, b->d_guess_flag, b->q_in));
  }
  {
    const tb_status ss = raise_smem_limits();
    if (ss != TB_OK) return ss;
  }
  return read_flags(b, st);
}

// One SCF iteration (next_scf, src/scf/iterators.cu:317-424) for every
// active structure: launches only, no host synchronisation, so that the same
// sequence can be captured once as a CUDA graph.
tb_status iterate_body(tb_batch* b, cudaStream_t st) {
  NvtxRange nv("tb.scf_iteration");
  const DevBatch& B = b->db;
  MolState& S = b->ms;
  const DevParams& Pc = b->Pc;
  const int nmol = b->nmol;
  const double econv = 1.0e-6 * b->opt.accuracy, pconv = 2.0e-5 * b->opt.accuracy;
  const int ntile64 = (int)b->tiles64.size(), ntile32 = (int)b->tiles32.size(), nchunk = (int)b->chunks32.size();
  const int gemm_grid = std::min(ntile64, 148 * 8);
  const size_t fermi_smem = (size_t)b->nmax * sizeof(double);
  const dim3 pot_grid(nmol, nblk(std::max(b->natmax, b->nshmax), kPotTargets));
  std::vector<int> act, phase;
  // algorithmic work of this iteration over the active structures (profile mode only)
  double n3 = 0, n2 = 0, n2occ = 0, n3_lo = 0, n3_hi = 0, n2occ_lo = 0, n2occ_hi = 0;
  if (b->opt.profile) {
    act.resize(nmol);
    phase.assign(nmol, 1);
    TB_CUDA(cudaMemcpyAsync(act.data(), S.active, nmol * sizeof(int), cudaMemcpyDeviceToHost, st));
    if (b->mixed)
      TB_CUDA(cudaMemcpyAsync(phase.data(), S.phase, nmol * sizeof(int), cudaMemcpyDeviceToHost, st));
    TB_CUDA(cudaStreamSynchronize(st));
    for (int m = 0; m < nmol; ++m) {
      if (!act[m]) continue;
      const double n = b->h_ooff[m + 1] - b->h_ooff[m];
      const double occ = n * n * std::min(n, b->h_nocc[m]);
      n3 += n * n * n;
      n2 += n * n;
      n2occ += occ;
      (phase[m] ? n3_hi : n3_lo) += n * n * n;
      (phase[m] ? n2occ_hi : n2occ_lo) += occ;
    }
  }
  // (k_mix_next leaves structures in their first iteration alone)
  TB_K("mix_next", 0, 0,
         k_mix_next<<<nmol, 256, 0, st>>>(B, b->q_in, b->dq, b->dqlast, b->qlast, b->df, b->u, b->amat,
                                          b->omega, b->opt.max_iter, b->opt.mixer_damping, S));
  TB_K("potential", 0, 0,
       k_potential<<<pot_grid, 32 * kPotTargets, 0, st>>>(Pc, B, b->q_in, b->mrad, b->vsh, b->vat, b->vdp, b->vqp, S.active,
                                             b->gtab, b->atab));
  // Fock build: reads S, H0, D(3), Q(6), writes F -> 12 N^2 doubles
  TB_K("fock", 96.0 * n2, 2,
       k_fock<<<ntile32, 256, fock_smem_bytes(), st>>>(B, b->d_tiles32, ntile32, b->S, b->H0, b->D, b->Q, b->vsh, b->vat, b->vdp,
                                       b->vqp, b->F, S.active));
  if (!b->mixed) {
    // F' = X^T F X  (T = F X in W, then F' into F): 2 x 2N^3
    TB_GEMM(2.0 * n3, b->F, 0, b->X, 0, nullptr, nullptr, nullptr, b->W, 1.0, 0.0, S.active, kGemmKUpToJ);
    TB_GEMM(2.0 * n3, b->X, 1, b->W, 0, nullptr, nullptr, nullptr, b->F, 1.0, 0.0, S.active, kGemmKUpToI | kGemmSym);
    // symmetric eigensolve with vectors: canonical 4 N^3 (k_trid_smem + k_syev)
    {
      const tb_status ts = launch_trid_plan(b, S.active, st);
      if (ts != TB_OK) return ts;
    }
    TB_K("syev", 4.0 * n3, 1,
         k_syev<<<nmol, kEigThreads, syev_smem_bytes(std::max(b->nmax_in, 1)), st>>>(
             B, b->F, b->Z, b->W, b->w, b->perm, S.status, S.active));
    if (b->njac > 0)
      TB_K("syev_jacobi", 0, 0,
           k_syev_jacobi<<<nblk(b->njac, kJacobiWarps), kJacobiWarps * 32, jacobi_smem_bytes(), st>>>(
               B, b->F, b->Z, b->w, b->perm, S.status, S.active, b->d_jlist, b->njac));
    for (size_t k = 0; k < b->big.size(); ++k) {
      const int m = b->big[k], n = b->h_ooff[m + 1] - b->h_ooff[m];
      if (!b->h_active[m] || b->h_status[m] != kStOk) continue;
      const long long mo = b->h_moff[m], vo = b->h_ooff[m];
      cudaEvent_t e0 = nullptr;
      prof_start(b, st, &e0);
      const std::string e = b->lib.syev(st, b->F + mo, b->Z + mo, b->w + vo, b->perm + vo, n, b->lib_work,
                                        b->lib_bytes, b->lib_info + 2 * k, S.status + m);
      if (!e.empty()) return fail(TB_CUDA_ERROR, "library eigensolver: " + e);
      ++b->launches;
      prof_stop(b, st, "syev_lib", e0, 4.0 * n * n * n, 1);
    }
    TB_K("fermi", 0, 0, k_fermi<<<nmol, 128, fermi_smem, st>>>(B, b->w, b->opt.kt, b->focc, b->kdim, S));
    // C = X Z (eigenvectors in ascending order through perm): 2N^3; P = C diag(f) C^T: 2 N^2 n_occ
    TB_GEMM(2.0 * n3, b->X, 0, b->Z, 1, b->perm, nullptr, nullptr, b->W, 1.0, 0.0, S.active, kGemmKFromI);
    TB_GEMM(2.0 * n2occ, b->W, 0, b->W, 1, nullptr, b->focc, b->kdim, b->P, 1.0, 0.0, S.active, kGemmSym);
  } else {
    const tb_status ms = mixed_core(b, st, n3_lo, n3_hi, n2occ_lo, n2occ_hi, gemm_grid, fermi_smem);
    if (ms != TB_OK) return ms;
  }
  // Mulliken + band energy: reads P, S, H0, D(3), Q(6) -> 11 N^2 doubles
  TB_K("mulliken", 88.0 * n2, 2,
       k_mulliken_cols<<<nchunk, 256, 0, st>>>(B, b->d_chunks32, nchunk, b->P, b->S, b->H0, b->D, b->Q, b->colred,
                                               S.active));
  TB_K("finalize", 0, 0,
       k_finalize<<<nmol, 256, 0, st>>>(Pc, B, b->colred, b->n0sh, b->mrad, b->q_in, b->dq, b->qsh_out, b->qat_out,
                                        b->dpat_out, b->qpat_out, econv, pconv, b->opt.max_iter, S,
                                        std::max(kMixedSwitchScale * econv, kMixedSwitchFloorE),
                                        std::max(kMixedSwitchScale * pconv, kMixedSwitchFloorQ), b->gtab, b->atab));
  return TB_OK;
}


// One iteration plus the host read of the active count; *n_active = structures
// still iterating.  With tb_options.use_graphs (and no structure on the
// library path, whose calls depend on host-side flags) the launches of
// iterate_body are captured once per batch and replayed.
tb_status launch_iteration(tb_batch* b, cudaStream_t st) {
  const bool graphs = b->opt.use_graphs && !b->opt.profile && b->big.empty();
  if (graphs) {
    if (!b->gexec) {
      if (!b->cap) TB_CUDA(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking));
      const int64_t l0 = b->launches;
      TB_CUDA(cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal));
      const tb_status bs = iterate_body(b, b->cap);
      cudaGraph_t g = nullptr;
      const cudaError_t ce = cudaStreamEndCapture(b->cap, &g);
      if (bs != TB_OK) {
        if (g) cudaGraphDestroy(g);
        return bs;
      }
      TB_CUDA(ce);
      const cudaError_t ie = cudaGraphInstantiate(&b->gexec, g, 0);
      cudaGraphDestroy(g);
      TB_CUDA(ie);
      b->launches_per_iter = b->launches - l0;
      b->launches = l0;
    }
    TB_CUDA(cudaGraphLaunch(b->gexec, st));
    b->launches += b->launches_per_iter;
  } else {
    const tb_status bs = iterate_body(b, st);
    if (bs != TB_OK) return bs;
  }
  ++b->it;
  TB_CUDA(cudaMemcpyAsync(b->h_nactive, b->ms.n_active, sizeof(int), cudaMemcpyDeviceToHost, st));
  return TB_OK;
}

// Waits for the iteration launched on st and reads the active count.
tb_status finish_iteration(tb_batch* b, cudaStream_t st, int* n_active) {
  TB_CUDA(cudaStreamSynchronize(st));
  *n_active = *b->h_nactive;
  if (*n_active > 0) return read_flags(b, st);
  return TB_OK;
}

tb_status batch_iterate(tb_batch* b, cudaStream_t st, int* n_active) {
  const tb_status s = launch_iteration(b, st);
  if (s != TB_OK) return s;
  return finish_iteration(b, st, n_active);
}

// The whole SCF loop as one graph launch: a conditional WHILE node whose body
// is one captured iteration (iterate_body) followed by k_loop_control, which
// counts the iteration on the device and sets the loop condition to "some
// structure still iterating and fewer than max_iter iterations", the same
// test the host loop of batch_run makes after each iteration.  No host
// synchronisation inside the loop; one read of the iteration count after it.
tb_status run_loop_graph(tb_batch* b, cudaStream_t st) {
  NvtxRange nv("tb.scf_loop_graph");
  if (!b->gloop) {
    if (!b->cap) TB_CUDA(cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking));
    cudaGraph_t g = nullptr;
    TB_CUDA(cudaGraphCreate(&g, 0));
    auto fail_graph = [&](cudaError_t e) {
      cudaGraphDestroy(g);
      return fail(TB_CUDA_ERROR, std::string("SCF loop graph: ") + cudaGetErrorString(e));
    };
    cudaGraphConditionalHandle h;
    cudaError_t e = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault);
    if (e != cudaSuccess) return fail_graph(e);
    cudaGraphNodeParams cp{};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node;
    e = cudaGraphAddNode(&node, g, nullptr, 0, &cp);
    if (e != cudaSuccess) return fail_graph(e);
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    e = cudaStreamBeginCaptureToGraph(b->cap, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return fail_graph(e);
    const int64_t l0 = b->launches;
    tb_status bs = iterate_body(b, b->cap);
    if (bs == TB_OK) {
      k_loop_control<<<1, 1, 0, b->cap>>>(h, b->ms.n_active, b->it_dev, b->opt.max_iter);
      e = cudaGetLastError();
      if (e == cudaSuccess) ++b->launches;
    }
    cudaGraph_t captured = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(b->cap, &captured);
    if (bs != TB_OK) { cudaGraphDestroy(g); return bs; }
    if (e != cudaSuccess) return fail_graph(e);
    if (ce != cudaSuccess) return fail_graph(ce);
    e = cudaGraphInstantiate(&b->gloop, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) { b->gloop = nullptr; return fail(TB_CUDA_ERROR, std::string("SCF loop graph: ") + cudaGetErrorString(e)); }
    b->launches_per_iter = b->launches - l0;
    b->launches = l0;
  }
  TB_CUDA(cudaMemsetAsync(b->it_dev, 0, sizeof(int), st));
  TB_CUDA(cudaGraphLaunch(b->gloop, st));
  TB_CUDA(cudaMemcpyAsync(b->h_nactive, b->it_dev, sizeof(int), cudaMemcpyDeviceToHost, st));
  TB_CUDA(cudaStreamSynchronize(st));
  b->it = *b->h_nactive;
  b->launches += b->launches_per_iter * b->it;
  return TB_OK;
}

tb_status batch_run(tb_batch* b, cudaStream_t st) {
  tb_status s = batch_setup(b, st);
  if (s != TB_OK) return s;
  if (b->opt.use_graphs && !b->opt.profile && b->big.empty()) return run_loop_graph(b, st);
  for (int it = 0; it < b->opt.max_iter; ++it) {
    int na = 0;
    s = batch_iterate(b, st, &na);
    if (s != TB_OK) return s;
    if (na <= 0) break;
  }
  return prof_collect(b, st);
}

tb_status batch_results(tb_batch* b, tb_result* out, cudaStream_t st) {
  NvtxRange nv("tb.results");
  const int nmol = b->nmol;
  const int NA = b->nat_tot, NS = b->nsh_tot;
  // the device results land in the calculator's pinned staging buffer (one
  // copy each at full link speed; pageable destinations would be copied
  // through driver bounce buffers), then go to the caller's records
  const size_t nd = 12 * (size_t)nmol + 10 * (size_t)NA + (size_t)NS, bytes = 8 * nd + 12 * (size_t)nmol;
  std::lock_guard<std::mutex> stage_lk(b->calc->stage_mu);
  if (b->calc->stage_bytes < bytes) {
    if (b->calc->stage) cudaFreeHost(b->calc->stage);
    b->calc->stage = nullptr;
    b->calc->stage_bytes = 0;
    TB_CUDA(cudaMallocHost(&b->calc->stage, bytes + (bytes >> 2)));
    b->calc->stage_bytes = bytes + (bytes >> 2);
  }
  double* hd = reinterpret_cast<double*>(b->calc->stage);
  double *erep = hd, *eelec = erep + nmol, *eband = eelec + nmol, *ets = eband + nmol, *e2 = ets + nmol,
         *ea = e2 + nmol, *e3 = ea + nmol, *err = e3 + nmol, *edisp = err + nmol, *dip = edisp + nmol,
         *qat = dip + 3 * nmol,
         *qsh = qat + NA, *dp = qsh + NS, *qp = dp + 3 * NA;
  int* hi = reinterpret_cast<int*>(hd + nd);
  int *iscf = hi, *status = iscf + nmol, *fw = status + nmol;
  const MolState& S = b->ms;
  auto cp = [&](void* dst, const void* src, size_t n) {
    return cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, st);
  };
  TB_CUDA(cp(erep, S.e_rep, nmol * 8)); TB_CUDA(cp(eelec, S.eelec, nmol * 8));
  TB_CUDA(cp(eband, S.e_band, nmol * 8)); TB_CUDA(cp(ets, S.e_ts, nmol * 8));
  TB_CUDA(cp(e2, S.e_es2, nmol * 8)); TB_CUDA(cp(ea, S.e_aes2, nmol * 8));
  TB_CUDA(cp(e3, S.e_es3, nmol * 8)); TB_CUDA(cp(err, S.scf_error, nmol * 8));
  TB_CUDA(cp(edisp, b->e_disp, nmol * 8));
  TB_CUDA(cp(dip, S.dipole, 3 * nmol * 8)); TB_CUDA(cp(iscf, S.iscf, nmol * 4));
  TB_CUDA(cp(status, S.status, nmol * 4)); TB_CUDA(cp(fw, S.fermi_warn, nmol * 4));
  TB_CUDA(cp(qat, b->qat_out, NA * 8)); TB_CUDA(cp(qsh, b->qsh_out, NS * 8));
  TB_CUDA(cp(dp, b->dpat_out, 3 * NA * 8)); TB_CUDA(cp(qp, b->qpat_out, 6 * NA * 8));
  TB_CUDA(cudaStreamSynchronize(st));
  tb_status first = TB_OK;
  for (int m = 0; m < nmol; ++m) {
    tb_result& r = out[m];
    r.e_rep = erep[m]; r.e_elec = eelec[m]; r.e_disp = edisp[m]; r.energy = eelec[m] + erep[m] + edisp[m];
    r.e_band = eband[m]; r.e_ts = ets[m]; r.e_es2 = e2[m]; r.e_aes2 = ea[m]; r.e_es3 = e3[m];
    r.scf_error = err[m]; r.iterations = iscf[m];
    for (int k = 0; k < 3; ++k) r.dipole[k] = dip[3 * m + k];
    int stt = status[m];
    if (stt == kStOk && fw[m]) stt = kStFermiNotConverged;
    r.status = stt;
    r.nsh = b->h_soff[m + 1] - b->h_soff[m];
    r.nao = b->h_ooff[m + 1] - b->h_ooff[m];
    const int a0 = b->h_aoff[m], na = b->h_aoff[m + 1] - a0, s0 = b->h_soff[m];
    if (r.qat) std::memcpy(r.qat, qat + a0, na * 8);
    if (r.qsh) std::memcpy(r.qsh, qsh + s0, r.nsh * 8);
    if (r.dpat) std::memcpy(r.dpat, dp + 3 * a0, 3 * na * 8);
    if (r.qpat) std::memcpy(r.qpat, qp + 6 * a0, 6 * na * 8);
    if (stt != kStOk && first == TB_OK) first = (tb_status)stt;
  }
  if (first != TB_OK) g_err = "at least one structure did not finish with TB_OK (see tb_result.status)";
  return first;
}

// Starting moments of the next run from the caller's wavefunctions: records
// with guess = 1 provide qsh, dpat and qpat, written into the mixer layout
// [qsh, dpat, qpat] of their structure (k_apply_guess copies them over the
// default guess after k_scf_init).
tb_status batch_set_guess(tb_batch* b, const tb_wavefunction* wfn) {
  const int nmol = b->nmol;
  b->h_guess.assign((size_t)b->mix_tot, 0.0);
  b->h_guess_flag.assign(nmol, 0);
  b->any_guess = false;
  if (!wfn) return TB_OK;
  for (int m = 0; m < nmol; ++m) {
    const tb_wavefunction& w = wfn[m];
    if (!w.guess) continue;
    if (!w.qsh || !w.dpat || !w.qpat)
      return fail(TB_BAD_INPUT, "wavefunction " + std::to_string(m) + ": guess = 1 needs qsh, dpat and qpat");
    const int nat = b->h_aoff[m + 1] - b->h_aoff[m], nsh = b->h_soff[m + 1] - b->h_soff[m];
    double* g = b->h_guess.data() + b->h_mixoff[m];
    for (int i = 0; i < nsh; ++i) g[i] = w.qsh[i];
    for (int i = 0; i < 3 * nat; ++i) g[nsh + i] = w.dpat[i];
    for (int i = 0; i < 6 * nat; ++i) g[nsh + 3 * nat + i] = w.qpat[i];
    for (int i = 0; i < nsh + 9 * nat; ++i)
      if (!std::isfinite(g[i])) return fail(TB_BAD_INPUT, "wavefunction " + std::to_string(m) + ": non-finite guess");
    b->h_guess_flag[m] = 1;
    b->any_guess = true;
  }
  return TB_OK;
}

// wavefunction_type of every structure after a run (tb_wavefunction): the
// scalars, the per-structure vectors gathered in one copy per field, and the
// density and coefficient matrices copied straight into the caller's arrays.
// W holds C = X Z of the structure's last iteration (the density GEMM reads
// it; nothing later overwrites it), P its density, w and focc its orbital
// energies (ascending) and occupations.
// Analytic nuclear gradient and virial of the structures with flag[m] set,
// after a run (the gradient/sigma outputs of xtb_singlepoint,
// src/xtb.cu:195-196): the potentials of the final moments (k_potential on
// [qsh, dpat, qpat] into the potential buffers, free after a run), the
// energy-weighted density W = C diag(f e) C^T (into F, free after a run), the
// shell-pair terms (k_grad_pairs_t, one item per neighbour shell pair, summed
// per atom pair by k_grad_pair_reduce), dE/dCN per atom (k_grad_cn), every
// atom's pair sum (k_grad_atoms) and sigma.  The workspace is the batch's own
// (allocated on first use, reused by later calls).
tb_status batch_gradient(tb_batch* b, const std::vector<int>& flag, cudaStream_t st) {
  NvtxRange nv("tb.gradient");
  tb_calculator* c = b->calc;
  const DevBatch& B = b->db;
  const int nmol = b->nmol;
  const long long NA = b->nat_tot, NO = b->nao_tot, NM = nmol, MX = b->mix_tot;
  const int maxsp = c->maxsh * c->maxsh;
  const long long items = b->pair_cap * maxsp;
  Layout L;
  const size_t o_item = L.add((size_t)items * 3 * 8), o_ese = L.add((size_t)b->h_s2off[nmol] * 8),
               o_G = L.add((size_t)b->h_a2off[nmol] * 3 * 8), o_cn = L.add(NA * 8), o_fe = L.add(NO * 8),
               o_qv = L.add(MX * 8), o_grad = L.add(3 * NA * 8), o_sig = L.add(9 * NM * 8), o_flag = L.add(NM * 4);
  {
    const cudaError_t e = b->grad_ws.reserve(L.total);
    if (e != cudaSuccess)
      return fail(TB_CUDA_ERROR, "gradient workspace of " + std::to_string(L.total >> 20) + " MiB: " +
                                     cudaGetErrorString(e));
  }
  char* base = b->grad_ws.base;
  double *item = at<double>(base, o_item), *ese = at<double>(base, o_ese), *G = at<double>(base, o_G),
         *dcn = at<double>(base, o_cn), *fe = at<double>(base, o_fe), *qv = at<double>(base, o_qv);
  int* dflag = at<int>(base, o_flag);
  b->d_grad = at<double>(base, o_grad);
  b->d_sigma = at<double>(base, o_sig);
  TB_CUDA(cudaMemcpyAsync(dflag, flag.data(), nmol * sizeof(int), cudaMemcpyHostToDevice, st));
  TB_CUDA(cudaMemsetAsync(item, 0, (size_t)items * 3 * 8, st));
  TB_CUDA(cudaMemsetAsync(ese, 0, (size_t)b->h_s2off[nmol] * 8, st));
  TB_CUDA(cudaMemsetAsync(G, 0, (size_t)b->h_a2off[nmol] * 3 * 8, st));
  k_grad_prep<<<nmol, 256, 0, st>>>(B, dflag, b->focc, b->w, b->qsh_out, b->dpat_out, b->qpat_out, fe, qv);
  TB_LAUNCH_CHECK();
  const dim3 pot_grid(nmol, nblk(std::max(b->natmax, b->nshmax), kPotTargets));
  k_potential<<<pot_grid, 32 * kPotTargets, 0, st>>>(b->Pc, B, qv, b->mrad, b->vsh, b->vat, b->vdp, b->vqp, dflag, b->gtab,
                                        b->atab);
  TB_LAUNCH_CHECK();
  {
    const tb_status gs = launch_gemm(b, st, nullptr, 0.0, b->W, 0, b->W, 1, nullptr, fe, b->kdim, b->F, 1.0, 0.0,
                                     dflag, kGemmSym);
    if (gs != TB_OK) return gs;
  }
  TB_CUDA(launch_grad_pairs(b->Pc, B, b->npair, b->pair_i, b->pair_j, b->se, b->P, b->F, b->vsh, b->vat, b->vdp,
                            b->vqp, dflag, maxsp, items, c->lmask, item, ese, st));
  ++b->launches;
  k_grad_pair_reduce<<<(int)std::min<long long>(nblk(b->pair_cap, 256), 148 * 16), 256, 0, st>>>(
      B, b->npair, b->pair_i, b->pair_j, dflag, maxsp, b->pair_cap, item, G);
  TB_LAUNCH_CHECK();
  const dim3 at_grid(nmol, nblk(b->natmax, 128));
  k_grad_cn<<<at_grid, 128, 0, st>>>(b->Pc, B, dflag, b->P, ese, b->cn, b->mrad, b->qat_out, b->dpat_out,
                                     b->qpat_out, dcn);
  TB_LAUNCH_CHECK();
  k_grad_atoms<<<at_grid, 128, 0, st>>>(b->Pc, B, dflag, G, dcn, b->mrad, b->qsh_out, b->qat_out, b->dpat_out,
                                        b->qpat_out, b->d_grad);
  TB_LAUNCH_CHECK();
  if (b->Pc.d4) {  // the dispersion gradient of the setup
    k_d4_add_grad<<<nblk(B.nat_tot, 128), 128, 0, st>>>(B, dflag, b->d4g, b->d_grad);
    TB_LAUNCH_CHECK();
  }
  k_grad_sigma<<<nmol, 128, 0, st>>>(B, dflag, b->d_grad, b->d_sigma);
  TB_LAUNCH_CHECK();
  b->h_grad_done = flag;
  return TB_OK;
}

// Gradient and sigma of the last batch_gradient into host buffers: packed
// [nat_tot][3] and [nmol][9] (either may be NULL), or per structure into the
// results whose gradient pointer is set.
tb_status gradient_copy(tb_batch* b, double* grad, double* sigma, tb_result* out, cudaStream_t st) {
  const int nmol = b->nmol;
  std::vector<double> g(3 * (size_t)b->nat_tot), sg(9 * (size_t)nmol);
  TB_CUDA(cudaMemcpyAsync(g.data(), b->d_grad, g.size() * 8, cudaMemcpyDeviceToHost, st));
  TB_CUDA(cudaMemcpyAsync(sg.data(), b->d_sigma, sg.size() * 8, cudaMemcpyDeviceToHost, st));
  TB_CUDA(cudaStreamSynchronize(st));
  if (grad) std::memcpy(grad, g.data(), g.size() * 8);
  if (sigma) std::memcpy(sigma, sg.data(), sg.size() * 8);
  if (out)
    for (int m = 0; m < nmol; ++m) {
      if (!out[m].gradient || !b->h_grad_done[m]) continue;
      const int a0 = b->h_aoff[m], na = b->h_aoff[m + 1] - a0;
      std::memcpy(out[m].gradient, g.data() + 3 * (size_t)a0, 3 * (size_t)na * 8);
      std::memcpy(out[m].sigma, sg.data() + 9 * (size_t)m, 9 * 8);
    }
  return TB_OK;
}

// Records with nspin = 2 get tblite's open-shell representation: both spin
// channels share the orbital energies and coefficients (GFN2 has no
// spin-dependent potential); per channel the Fermi filling of its electrons
// (k_spin_occupations), the densities P_alpha = C f_a C^T and P_beta = C f_b
// C^T (into X and F, free after a run: the next run's setup rewrites them),
// and the moments as (total, up - down), the latter from the Mulliken sums of
// P_alpha - P_beta = C (f_a - f_b) C^T (into Z; k_spin_moments, into the
// potential buffers, also free after a run).
tb_status spin_readout(tb_batch* b, const std::vector<int>& flag, cudaStream_t st) {
  const DevBatch& B = b->db;
  const int nmol = b->nmol, nchunk = (int)b->chunks32.size();
  const long long NO = b->nao_tot;
  TB_CUDA(cudaMemcpyAsync(b->d_wflag, flag.data(), nmol * sizeof(int), cudaMemcpyHostToDevice, st));
  k_spin_occupations<<<nmol, 128, (size_t)b->nmax * sizeof(double), st>>>(B, b->w, b->opt.kt, b->ms.nel, b->d_wflag,
                                                                          b->d_fspin);
  TB_LAUNCH_CHECK();
  double* out[3] = {b->X, b->F, b->Z};  // P_alpha, P_beta, P_alpha - P_beta
  for (int c = 0; c < 3; ++c) {
    const tb_status gs = launch_gemm(b, st, nullptr, 0.0, b->W, 0, b->W, 1, nullptr, b->d_fspin + c * NO, b->kdim,
                                     out[c], 1.0, 0.0, b->d_wflag, kGemmSym);
    if (gs != TB_OK) return gs;
  }
  k_mulliken_cols<<<nchunk, 256, 0, st>>>(B, b->d_chunks32, nchunk, b->Z, b->S, b->H0, b->D, b->Q, b->colred,
                                          b->d_wflag);
  TB_LAUNCH_CHECK();
  k_spin_moments<<<nmol, 256, 0, st>>>(b->Pc, B, b->colred, b->d_wflag, b->vsh, b->vat, b->vdp, b->vqp);
  TB_LAUNCH_CHECK();
  return TB_OK;
}

tb_status batch_wavefunction(tb_batch* b, tb_wavefunction* wfn, cudaStream_t st) {
  NvtxRange nv("tb.wavefunction");
  const int nmol = b->nmol;
  const int NA = b->nat_tot, NS = b->nsh_tot, NO = b->nao_tot;
  std::vector<int> spin2(nmol, 0);
  bool any2 = false;
  for (int m = 0; m < nmol; ++m) {
    if (wfn[m].nspin != 0 && wfn[m].nspin != 1 && wfn[m].nspin != 2)
      return fail(TB_BAD_INPUT, "wavefunction " + std::to_string(m) + ": nspin must be 1 or 2");
    spin2[m] = wfn[m].nspin == 2;
    any2 |= spin2[m] != 0;
  }
  std::vector<double> fsp, msh, mat, mdp, mqp;
  if (any2) {
    const tb_status ss = spin_readout(b, spin2, st);
    if (ss != TB_OK) return ss;
    fsp.resize(3 * (size_t)NO); msh.resize(NS); mat.resize(NA); mdp.resize(3 * (size_t)NA); mqp.resize(6 * (size_t)NA);
    TB_CUDA(cudaMemcpyAsync(fsp.data(), b->d_fspin, 2 * (size_t)NO * 8, cudaMemcpyDeviceToHost, st));
    TB_CUDA(cudaMemcpyAsync(msh.data(), b->vsh, NS * 8, cudaMemcpyDeviceToHost, st));
    TB_CUDA(cudaMemcpyAsync(mat.data(), b->vat, NA * 8, cudaMemcpyDeviceToHost, st));
    TB_CUDA(cudaMemcpyAsync(mdp.data(), b->vdp, 3 * (size_t)NA * 8, cudaMemcpyDeviceToHost, st));
    TB_CUDA(cudaMemcpyAsync(mqp.data(), b->vqp, 6 * (size_t)NA * 8, cudaMemcpyDeviceToHost, st));
  }
  std::vector<double> emo(NO), focc(NO), n0sh(NS), nel(2 * (size_t)nmol), qat(NA), qsh(NS), dp(3 * (size_t)NA),
      qp(6 * (size_t)NA);
  auto cp = [&](void* dst, const void* src, size_t n) { return cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, st); };
  TB_CUDA(cp(emo.data(), b->w, NO * 8));
  TB_CUDA(cp(focc.data(), b->focc, NO * 8));
  TB_CUDA(cp(n0sh.data(), b->n0sh, NS * 8));
  TB_CUDA(cp(nel.data(), b->ms.nel, 2 * (size_t)nmol * 8));
  TB_CUDA(cp(qat.data(), b->qat_out, NA * 8));
  TB_CUDA(cp(qsh.data(), b->qsh_out, NS * 8));
  TB_CUDA(cp(dp.data(), b->dpat_out, 3 * (size_t)NA * 8));
  TB_CUDA(cp(qp.data(), b->qpat_out, 6 * (size_t)NA * 8));
  for (int m = 0; m < nmol; ++m) {
    tb_wavefunction& w = wfn[m];
    const long long mo = b->h_moff[m], nn = b->h_moff[m + 1] - mo;
    if (spin2[m]) {  // [2][nao][nao]: alpha, beta
      if (w.density) {
        TB_CUDA(cp(w.density, b->X + mo, nn * 8));
        TB_CUDA(cp(w.density + nn, b->F + mo, nn * 8));
      }
      if (w.coeff) {
        TB_CUDA(cp(w.coeff, b->W + mo, nn * 8));
        TB_CUDA(cp(w.coeff + nn, b->W + mo, nn * 8));
      }
    } else {
      if (w.density) TB_CUDA(cp(w.density, b->P + mo, nn * 8));
      if (w.coeff) TB_CUDA(cp(w.coeff, b->W + mo, nn * 8));
    }
  }
  TB_CUDA(cudaStreamSynchronize(st));
  const HostParams& P = b->calc->hp;
  for (int m = 0; m < nmol; ++m) {
    tb_wavefunction& w = wfn[m];
    const int a0 = b->h_aoff[m], s0 = b->h_soff[m], o0 = b->h_ooff[m];
    w.nspin = spin2[m] ? 2 : 1;
    w.nat = b->h_aoff[m + 1] - a0;
    w.nsh = b->h_soff[m + 1] - s0;
    w.nao = b->h_ooff[m + 1] - o0;
    w.kt = b->opt.kt;
    w.nel[0] = nel[2 * m];
    w.nel[1] = nel[2 * m + 1];
    w.nocc = w.nel[0] + w.nel[1];
    w.nuhf = w.nel[0] - w.nel[1];
    for (int s = 0; s < 2; ++s) w.homo[s] = (int32_t)std::floor(w.nel[s]);
    if (w.emo) std::memcpy(w.emo, emo.data() + o0, w.nao * 8);
    if (w.emo && spin2[m]) std::memcpy(w.emo + w.nao, emo.data() + o0, w.nao * 8);
    if (w.focc && !spin2[m]) std::memcpy(w.focc, focc.data() + o0, w.nao * 8);
    if (w.focc && spin2[m]) {
      std::memcpy(w.focc, fsp.data() + o0, w.nao * 8);
      std::memcpy(w.focc + w.nao, fsp.data() + NO + o0, w.nao * 8);
    }
    if (w.n0sh) std::memcpy(w.n0sh, n0sh.data() + s0, w.nsh * 8);
    if (w.n0at) {  // the shells of an atom are consecutive
      int s = s0;
      for (int a = 0; a < w.nat; ++a) {
        const int nsh_a = P.sp[b->h_species[a0 + a]].nsh;
        double t = 0.0;
        for (int k = 0; k < nsh_a; ++k) t += n0sh[s++];
        w.n0at[a] = t;
      }
    }
    if (w.qat) std::memcpy(w.qat, qat.data() + a0, w.nat * 8);
    if (w.qsh) std::memcpy(w.qsh, qsh.data() + s0, w.nsh * 8);
    if (w.dpat) std::memcpy(w.dpat, dp.data() + 3 * (size_t)a0, 3 * (size_t)w.nat * 8);
    if (w.qpat) std::memcpy(w.qpat, qp.data() + 6 * (size_t)a0, 6 * (size_t)w.nat * 8);
    if (spin2[m]) {  // channel 1: up - down
      if (w.qat) std::memcpy(w.qat + w.nat, mat.data() + a0, w.nat * 8);
      if (w.qsh) std::memcpy(w.qsh + w.nsh, msh.data() + s0, w.nsh * 8);
      if (w.dpat) std::memcpy(w.dpat + 3 * w.nat, mdp.data() + 3 * (size_t)a0, 3 * (size_t)w.nat * 8);
      if (w.qpat) std::memcpy(w.qpat + 6 * w.nat, mqp.data() + 6 * (size_t)a0, 6 * (size_t)w.nat * 8);
    }
  }
  return TB_OK;
}

}  // namespace

// error text for the allocation-free entry point (tb_noalloc.cu)
const char* tb_noalloc_set_error(const char* msg) {
  g_err = msg;
  return g_err.c_str();
}

// ====================================================================== C ABI
extern "C" {

const char* tb_last_error(void) { return g_err.c_str(); }

void tb_default_options(tb_options* o) {
  std::memset(o, 0, sizeof(*o));
  o->accuracy = 1.0;
  o->kt = 300.0 * 3.166811563455546e-6;
  o->max_iter = 32;
  o->mixer_damping = 0.4;
  o->verbosity = 0;
  o->use_graphs = 0;
  o->solver = 0;
}

tb_status tb_calculator_create(const char* param_file, tb_calculator** out) {
  if (!param_file || !out) return fail(TB_BAD_INPUT, "null argument");
  *out = nullptr;
  auto* c = new tb_calculator();
  std::string err;
  if (!parse_params(param_file, c->hp, err)) { delete c; return fail(TB_PARAM_ERROR, err); }
  const HostParams& P = c->hp;
  const int nt = (int)P.sh.size();
  std::vector<double> hs((size_t)nt * nt);
  for (int i = 0; i < nt; ++i)
    for (int j = 0; j < nt; ++j) hs[(size_t)i * nt + j] = hscale_of(P, i, j);
  for (auto& s : P.sp) c->maxsh = std::max(c->maxsh, s.nsh);
  for (auto& s : P.sh) c->lmask |= 1 << s.ang;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) { delete c; return fail(TB_CUDA_ERROR, std::string("no CUDA device: ") + cudaGetErrorString(e)); }
  if (cudaMalloc(&c->d_sp, P.sp.size() * sizeof(SpeciesParam)) != cudaSuccess ||
      cudaMalloc(&c->d_sh, P.sh.size() * sizeof(ShellParam)) != cudaSuccess ||
      cudaMalloc(&c->d_hscale, hs.size() * sizeof(double)) != cudaSuccess) {
    delete c;
    return fail(TB_CUDA_ERROR, "cannot allocate parameter tables");
  }
  cudaMemcpy(c->d_sp, P.sp.data(), P.sp.size() * sizeof(SpeciesParam), cudaMemcpyHostToDevice);
  cudaMemcpy(c->d_sh, P.sh.data(), P.sh.size() * sizeof(ShellParam), cudaMemcpyHostToDevice);
  e = cudaMemcpy(c->d_hscale, hs.data(), hs.size() * sizeof(double), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) { delete c; return fail(TB_CUDA_ERROR, cudaGetErrorString(e)); }
  DevParams& d = c->dp;
  d.sp = c->d_sp; d.sh = c->d_sh; d.hscale = c->d_hscale;
  d.nsp = (int)P.sp.size(); d.nshtype = nt;
  d.gexp = P.glob("gexp", 2.0); d.kdmp3 = P.glob("kdmp3"); d.kdmp5 = P.glob("kdmp5");
  d.mp_shift = P.glob("mp_shift"); d.mp_kexp = P.glob("mp_kexp"); d.mp_rmax = P.glob("mp_rmax");
  d.rep_kexp = P.glob("rep_kexp"); d.rep_kexp_light = P.glob("rep_kexp_light"); d.rep_rexp = P.glob("rep_rexp");
  d.cn_cutoff = P.glob("cn_cutoff", 25.0); d.rep_cutoff = P.glob("rep_cutoff", 25.0);
  d.intcut = integral_cutoff(1.0);
  d.cutoff = std::min(std::sqrt(2.0 * d.intcut / P.min_alpha), 40.0);
  d.d4 = 0;
  d.d4_c6ref = nullptr;
  if (!P.d4_freq.empty()) {
    // reference C6 of every pair of reference systems, Casimir-Polder on the
    // file's grid: C6 = 3/pi sum_k wts_k alpha_Ai(i w_k) alpha_Bj(i w_k)
    const int ns = (int)P.sp.size(), R = kD4MaxRef;
    std::vector<double> c6((size_t)ns * ns * R * R, 0.0);
    for (int a = 0; a < ns; ++a)
      for (int b = 0; b < ns; ++b)
        for (int i = 0; i < P.sp[a].d4_nref; ++i)
          for (int j = 0; j < P.sp[b].d4_nref; ++j) {
            double x = 0.0;
            for (size_t k = 0; k < P.d4_freq.size(); ++k) x += P.d4_wts[k] * P.d4_alpha[a][i][k] * P.d4_alpha[b][j][k];
            c6[(((size_t)a * ns + b) * R + i) * R + j] = 3.0 / M_PI * x;
          }
    if (cudaMalloc(&c->d_d4c6, c6.size() * sizeof(double)) != cudaSuccess ||
        cudaMemcpy(c->d_d4c6, c6.data(), c6.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
      delete c;
      return fail(TB_CUDA_ERROR, "cannot allocate the D4 reference table");
    }
    d.d4 = 1;
    d.d4_c6ref = c->d_d4c6;
    d.d4_s6 = P.glob("d4_s6"); d.d4_s8 = P.glob("d4_s8"); d.d4_a1 = P.glob("d4_a1"); d.d4_a2 = P.glob("d4_a2");
    d.d4_s9 = P.glob("d4_s9"); d.d4_alp = P.glob("d4_alp"); d.d4_wf = P.glob("d4_wf"); d.d4_k0 = P.glob("d4_k0");
    d.d4_k1 = P.glob("d4_k1"); d.d4_k4 = P.glob("d4_k4"); d.d4_k5 = P.glob("d4_k5"); d.d4_k6 = P.glob("d4_k6");
    d.d4_cn_cut = P.glob("d4_cn_cut"); d.d4_atm_cut = P.glob("d4_atm_cut"); d.d4_pair_cut = P.glob("d4_pair_cut");
  }
  *out = c;
  return TB_OK;
}

void tb_calculator_destroy(tb_calculator* c) { delete c; }

int32_t tb_bounds_check_build(void) {
#ifdef TB_BOUNDS_CHECK
  return 1;
#else
  return 0;
#endif
}

tb_status tb_bounds_violations(int64_t* count, int32_t* site, int64_t* index, int64_t* lo, int64_t* hi,
                               int32_t reset) {
  OobRecord r[3];
  cudaError_t e = oob_setup(&r[0], reset != 0);
  if (e == cudaSuccess) e = oob_scf(&r[1], reset != 0);
  if (e == cudaSuccess) e = oob_linalg(&r[2], reset != 0);
  if (e != cudaSuccess) return fail(TB_CUDA_ERROR, cudaGetErrorString(e));
  int64_t total = 0;
  const OobRecord* first = nullptr;
  for (const OobRecord& x : r) {
    total += (int64_t)x.count;
    if (x.count && !first) first = &x;
  }
  if (count) *count = total;
  if (site) *site = first ? first->site : 0;
  if (index) *index = first ? first->index : 0;
  if (lo) *lo = first ? first->lo : 0;
  if (hi) *hi = first ? first->hi : 0;
  return TB_OK;
}

tb_status tb_calculator_set_small_solver(tb_calculator* c, int32_t jacobi_max) {
  if (!c) return fail(TB_BAD_INPUT, "null calculator");
  if (jacobi_max < -1 || jacobi_max > kJacobiMaxN)
    return fail(TB_BAD_INPUT, "jacobi_max must be -1 (measured), 0 (never) or 1.." + std::to_string(kJacobiMaxN));
  c->jacobi_override = jacobi_max;
  return TB_OK;
}

// Structure file input (the structure I/O beside periodic images in the
// reference's plan, src/xtb.cu:342-346 and src/adjlist.cu:28-29): the XYZ
// format -- a count line, a comment line, then "symbol x y z" per atom in
// Angstrom -- into atomic numbers and Bohr.
tb_status tb_read_xyz(const char* path, int32_t cap, int32_t* nat, int32_t* z, double* xyz, char* comment,
                      int32_t comment_len) {
  static const char* kSym[] = {"H",  "He", "Li", "Be", "B",  "C",  "N",  "O",  "F",  "Ne", "Na", "Mg", "Al", "Si", "P",
                               "S",  "Cl", "Ar", "K",  "Ca", "Sc", "Ti", "V",  "Cr", "Mn", "Fe", "Co", "Ni", "Cu", "Zn",
                               "Ga", "Ge", "As", "Se", "Br", "Kr", "Rb", "Sr", "Y",  "Zr", "Nb", "Mo", "Tc", "Ru", "Rh",
                               "Pd", "Ag", "Cd", "In", "Sn", "Sb", "Te", "I",  "Xe", "Cs", "Ba", "La", "Ce", "Pr", "Nd",
                               "Pm", "Sm", "Eu", "Gd", "Tb", "Dy", "Ho", "Er", "Tm", "Yb", "Lu", "Hf", "Ta", "W",  "Re",
                               "Os", "Ir", "Pt", "Au", "Hg", "Tl", "Pb", "Bi", "Po", "At", "Rn"};
  if (!path || !nat) return fail(TB_BAD_INPUT, "null argument");
  std::ifstream f(path);
  if (!f) return fail(TB_BAD_INPUT, std::string("cannot open ") + path);
  std::string line;
  long long n = -1;
  if (!std::getline(f, line) || !(std::istringstream(line) >> n) || n <= 0)
    return fail(TB_BAD_INPUT, "xyz: bad atom count line");
  *nat = (int32_t)n;
  std::getline(f, line);
  if (comment && comment_len > 0) std::snprintf(comment, (size_t)comment_len, "%s", line.c_str());
  if (n > cap || !z || !xyz) return n > cap ? fail(TB_CAPACITY_EXCEEDED, "xyz: more atoms than cap") : TB_OK;
  const double bohr = 1.0 / 0.529177210903;
  for (long long a = 0; a < n; ++a) {
    if (!std::getline(f, line)) return fail(TB_BAD_INPUT, "xyz: fewer atom lines than the count");
    std::istringstream is(line);
    std::string sym;
    double x, y, w;
    if (!(is >> sym >> x >> y >> w)) return fail(TB_BAD_INPUT, "xyz: bad atom line " + std::to_string(a + 1));
    int zz = 0;
    if (std::isdigit((unsigned char)sym[0])) {
      zz = std::atoi(sym.c_str());
    } else {
      std::string s2 = sym;
      s2[0] = (char)std::toupper((unsigned char)s2[0]);
      for (size_t i = 1; i < s2.size(); ++i) s2[i] = (char)std::tolower((unsigned char)s2[i]);
      for (int k = 0; k < (int)(sizeof(kSym) / sizeof(kSym[0])); ++k)
        if (s2 == kSym[k]) { zz = k + 1; break; }
    }
    if (zz <= 0) return fail(TB_BAD_INPUT, "xyz: unknown element " + sym);
    z[a] = zz;
    xyz[3 * a] = x * bohr;
    xyz[3 * a + 1] = y * bohr;
    xyz[3 * a + 2] = w * bohr;
  }
  return TB_OK;
}

int32_t tb_calculator_species(const tb_calculator* c, int32_t z) {
  if (!c) return -1;
  for (size_t i = 0; i < c->hp.sp.size(); ++i)
    if (c->hp.sp[i].z == z) return (int32_t)i;
  return -1;
}

tb_status tb_calculator_set_smem_tridiag(tb_calculator* c, int32_t min_n) {
  if (!c) return fail(TB_BAD_INPUT, "null calculator");
  if (min_n < 0) return fail(TB_BAD_INPUT, "min_n must be 0 (never) or a size in AOs");
  c->smem_tridiag = min_n;
  return TB_OK;
}

tb_status tb_calculator_set_gemm_tiles(tb_calculator* c, int32_t max_n32) {
  if (!c) return fail(TB_BAD_INPUT, "null calculator");
  if (max_n32 < -1) return fail(TB_BAD_INPUT, "max_n32 must be -1 (measured), 0 (64 x 64 always) or a size in AOs");
  c->tile_override = max_n32;
  return TB_OK;
}

int32_t tb_calculator_tuning(const tb_calculator* c, char* buf, int32_t len) {
  if (!c) return 0;
  std::ostringstream o;
  o.precision(6);
  o << "{\"small\": {\"measured\": " << (c->small.ready ? "true" : "false") << ", \"override\": "
    << c->jacobi_override << ", \"jacobi_max\": " << c->small.jacobi_max << ", \"sizes\": [";
  for (size_t i = 0; i < c->small.n.size(); ++i) {
    o << (i ? ", " : "") << "{\"n\": " << c->small.n[i] << ", \"s_per_structure_cta\": " << c->small.t_cta[i]
      << ", \"s_per_structure_warp_jacobi\": " << c->small.t_warp[i] << "}";
  }
  o << "]}, \"large\": {\"measured\": " << (c->eig.ready ? "true" : "false")
    << ", \"inhouse_s\": {\"256\": " << c->eig.t_in[0] << ", \"512\": " << c->eig.t_in[1] << "}"
    << ", \"cusolver_s\": {\"256\": " << c->eig.t_lib[0] << ", \"1024\": " << c->eig.t_lib[1] << "}"
    << ", \"model\": {\"inhouse\": \"" << c->eig.a << " N^2 + " << c->eig.b << " N^3\", \"cusolver\": \""
    << c->eig.c << " + " << c->eig.d << " N^3\"}, \"inhouse_limit\": " << kSyevMaxN << "}"
    << ", \"smem_tridiag\": {\"min_n\": " << c->smem_tridiag << ", \"classes\": [";
  for (int k = 0; k < kTridClasses; ++k)
    o << (k ? ", " : "") << "{\"cluster\": " << kTridClusterSizes[k] << ", \"max_n\": " << kTridClassMax[k]
      << ", \"smem_bytes\": " << trid_smem_bytes(kTridClassMax[k], kTridClusterSizes[k]) << "}";
  o << "], \"smallest\": " << kTridMin << "}";
  o << ", \"gemm_tiles\": {\"measured\": " << (c->tile.ready ? "true" : "false") << ", \"override\": "
    << c->tile_override << ", \"split_gain\": " << kTileSplitGain << ", \"sizes\": [";
  for (size_t i = 0; i < c->tile.n.size(); ++i)
    o << (i ? ", " : "") << "{\"n\": " << c->tile.n[i] << ", \"s_per_structure_64\": " << c->tile.t64[i]
      << ", \"s_per_structure_32\": " << c->tile.t32[i] << ", \"tile\": " << (c->tile.use32[i] ? 32 : 64) << "}";
  o << "]}}";
  const std::string t = o.str();
  if (buf && len > 0) std::snprintf(buf, (size_t)len, "%s", t.c_str());
  return (int32_t)t.size();
}
int32_t tb_calculator_nspecies(const tb_calculator* c) { return c ? (int32_t)c->hp.sp.size() : 0; }

double tb_get_cutoff(const tb_calculator* c, double accuracy) {
  return std::min(std::sqrt(2.0 * integral_cutoff(accuracy) / c->hp.min_alpha), 40.0);
}

tb_status tb_basis_size(const tb_calculator* c, const tb_structure* mol, int32_t* nsh, int32_t* nao) {
  if (!c || !mol || !nsh || !nao || !mol->id) return fail(TB_BAD_INPUT, "null argument");
  int s = 0, o = 0;
  for (int a = 0; a < mol->nat; ++a) {
    const int z = mol->id[a];
    if (z < 0 || z >= (int)c->hp.sp.size()) return fail(TB_BAD_INPUT, "bad species");
    const SpeciesParam& sp = c->hp.sp[z];
    for (int k = 0; k < sp.nsh; ++k) o += msao(c->hp.sh[sp.sh0 + k].ang);
    s += sp.nsh;
  }
  *nsh = s; *nao = o;
  return TB_OK;
}

tb_status tb_batch_create(tb_calculator* calc, const tb_structure* mols, int32_t nmol, const tb_options* opt,
                          tb_batch** out) {
  if (!calc || !mols || !out) return fail(TB_BAD_INPUT, "null argument");
  tb_options o;
  if (opt) o = *opt; else tb_default_options(&o);
  auto* b = new tb_batch();
  tb_status st = batch_build(calc, mols, nmol, &o, b, &b->own);
  if (st != TB_OK) { delete b; return st; }
  *out = b;
  return TB_OK;
}

tb_status tb_batch_run(tb_batch* b, void* stream) {
  if (!b) return fail(TB_BAD_INPUT, "null batch");
  return batch_run(b, (cudaStream_t)stream);
}

tb_status tb_batch_results(tb_batch* b, tb_result* out, void* stream) {
  if (!b || !out) return fail(TB_BAD_INPUT, "null argument");
  return batch_results(b, out, (cudaStream_t)stream);
}

tb_status tb_batch_set_guess(tb_batch* b, const tb_wavefunction* wfn) {
  if (!b) return fail(TB_BAD_INPUT, "null batch");
  return batch_set_guess(b, wfn);
}

tb_status tb_batch_gradient(tb_batch* b, double* grad, double* sigma, void* stream) {
  if (!b) return fail(TB_BAD_INPUT, "null batch");
  const std::vector<int> flag(b->nmol, 1);
  tb_status st = batch_gradient(b, flag, (cudaStream_t)stream);
  if (st != TB_OK) return st;
  return gradient_copy(b, grad, sigma, nullptr, (cudaStream_t)stream);
}

tb_status tb_batch_wavefunction(tb_batch* b, tb_wavefunction* wfn, void* stream) {
  if (!b || !wfn) return fail(TB_BAD_INPUT, "null argument");
  return batch_wavefunction(b, wfn, (cudaStream_t)stream);
}

int64_t tb_batch_launches(const tb_batch* b) { return b ? b->launches : 0; }

int32_t tb_batch_profile(const tb_batch* b, int32_t max, char* names, int64_t* launches, double* ms, double* work,
                         int32_t* units) {
  if (!b) return 0;
  const int n = std::min<int>(max, (int)b->kclass.size());
  for (int i = 0; i < n; ++i) {
    const auto& k = b->kclass[i];
    if (names) std::snprintf(names + 32 * i, 32, "%s", k.name.c_str());
    if (launches) launches[i] = k.launches;
    if (ms) ms[i] = k.ms;
    if (work) work[i] = k.work;
    if (units) units[i] = k.unit;
  }
  return n;
}
void tb_batch_destroy(tb_batch* b) { delete b; }

tb_status tb_singlepoint_batch(tb_calculator* calc, const tb_structure* mols, int32_t nmol, const tb_options* opt,
                               tb_wavefunction* wfn_inout, tb_result* out, void* stream) {
  if (!calc || !mols || !out) return fail(TB_BAD_INPUT, "null argument");
  tb_options o;
  if (opt) o = *opt; else tb_default_options(&o);
  std::lock_guard<std::mutex> lk(calc->mu);
  tb_batch b;
  tb_status st = batch_build(calc, mols, nmol, &o, &b, &calc->arena);
  if (st != TB_OK) return st;
  if (wfn_inout) {
    st = batch_set_guess(&b, wfn_inout);
    if (st != TB_OK) return st;
  }
  st = batch_run(&b, (cudaStream_t)stream);
  if (st != TB_OK) return st;
  std::vector<int> gflag(nmol, 0);
  bool any_grad = false;
  for (int m = 0; m < nmol; ++m) any_grad |= (gflag[m] = out[m].gradient != nullptr) != 0;
  if (any_grad) {
    st = batch_gradient(&b, gflag, (cudaStream_t)stream);
    if (st != TB_OK) return st;
  }
  const tb_status rs = batch_results(&b, out, (cudaStream_t)stream);
  if (rs == TB_CUDA_ERROR) return rs;
  if (any_grad) {
    st = gradient_copy(&b, nullptr, nullptr, out, (cudaStream_t)stream);
    if (st != TB_OK) return st;
  }
  if (wfn_inout) {  // also for structures that failed: their records hold their last state
    st = batch_wavefunction(&b, wfn_inout, (cudaStream_t)stream);
    if (st != TB_OK) return st;
  }
  return rs;
}

}  // extern "C"

// ====================================================================== stage entry points
// Each runs the same device kernels as the singlepoint on one structure (or
// a list of matrices) and copies the stage's outputs back to host buffers.
namespace {

struct OneBatch {
  tb_batch b;
  tb_status st = TB_OK;
  OneBatch(tb_calculator* c, const tb_structure* mol) {
    tb_options o;
    tb_default_options(&o);
    st = batch_build(c, mol, 1, &o, &b, &b.own);
  }
};

DevParams params_for(const tb_calculator* c, double accuracy) {
  DevParams P = c->dp;
  P.intcut = integral_cutoff(accuracy);
  P.cutoff = std::min(std::sqrt(2.0 * P.intcut / c->hp.min_alpha), 40.0);
  return P;
}

tb_status d2h(void* dst, const void* src, size_t bytes) {
  TB_CUDA(cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToHost));
  return TB_OK;
}

tb_status run_setup_to_integrals(tb_batch* b, bool with_integrals) {
  const DevParams P = params_for(b->calc, 1.0);
  const DevBatch& B = b->db;
  k_atoms<<<nblk(B.nat_tot, 128), 128>>>(P, B, b->cn, b->mrad, b->erep, b->se);
  TB_LAUNCH_CHECK();
  if (!with_integrals) return TB_OK;
  k_adj_count<<<nblk((long long)B.nat_tot * 32, 256), 256>>>(B, P.cutoff, b->cnt);
  TB_LAUNCH_CHECK();
  k_adj_scan<<<b->nmol, 256>>>(B, b->cnt, b->inl, b->npair);
  TB_LAUNCH_CHECK();
  k_adj_fill<<<nblk((long long)B.nat_tot * 32, 256), 256>>>(B, P.cutoff, b->inl, b->pair_i, b->pair_j);
  TB_LAUNCH_CHECK();
  MatOut out{b->S, b->H0, b->D, b->Q};
  const int maxsp = b->calc->maxsh * b->calc->maxsh;
  TB_CUDA(launch_integrals(P, B, b->npair, b->pair_i, b->pair_j, b->se, out, maxsp, b->pair_cap, b->calc->lmask,
                           b->sp_w, 0, &b->launches));
  TB_CUDA(cudaDeviceSynchronize());
  return TB_OK;
}

}  // namespace

extern "C" {

tb_status tb_adjacency_list(const tb_calculator* calc, const tb_structure* mol, double cutoff, int32_t* inl,
                            int32_t* nnl, int32_t* nlat, int32_t cap, int32_t* npair) {
  if (!calc || !mol || !inl || !nnl || !npair) return fail(TB_BAD_INPUT, "null argument");
  OneBatch ob(const_cast<tb_calculator*>(calc), mol);
  if (ob.st != TB_OK) return ob.st;
  tb_batch* b = &ob.b;
  const DevBatch& B = b->db;
  k_adj_count<<<nblk((long long)B.nat_tot * 32, 256), 256>>>(B, cutoff, b->cnt);
  TB_LAUNCH_CHECK();
  k_adj_scan<<<1, 256>>>(B, b->cnt, b->inl, b->npair);
  TB_LAUNCH_CHECK();
  k_adj_fill<<<nblk((long long)B.nat_tot * 32, 256), 256>>>(B, cutoff, b->inl, b->pair_i, b->pair_j);
  TB_LAUNCH_CHECK();
  const int nat = mol->nat;
  std::vector<long long> l(nat);
  int np = 0;
  if (d2h(l.data(), b->inl, nat * sizeof(long long)) || d2h(nnl, b->cnt, nat * sizeof(int)) ||
      d2h(&np, b->npair, sizeof(int)))
    return TB_CUDA_ERROR;
  for (int a = 0; a < nat; ++a) inl[a] = (int32_t)l[a];
  *npair = np;
  if (np > cap) return fail(TB_CAPACITY_EXCEEDED, "nlat capacity too small");
  if (np > 0 && nlat && d2h(nlat, b->pair_j, np * sizeof(int))) return TB_CUDA_ERROR;
  return TB_OK;
}

tb_status tb_atomic_properties(const tb_calculator* calc, const tb_structure* mol, double* cn, double* mrad,
                               double* se) {
  if (!calc || !mol) return fail(TB_BAD_INPUT, "null argument");
  OneBatch ob(const_cast<tb_calculator*>(calc), mol);
  if (ob.st != TB_OK) return ob.st;
  tb_batch* b = &ob.b;
  tb_status st = run_setup_to_integrals(b, false);
  if (st != TB_OK) return st;
  if (cn && d2h(cn, b->cn, mol->nat * 8)) return TB_CUDA_ERROR;
  if (mrad && d2h(mrad, b->mrad, mol->nat * 8)) return TB_CUDA_ERROR;
  if (se && d2h(se, b->se, b->nsh_tot * 8)) return TB_CUDA_ERROR;
  return TB_OK;
}

tb_status tb_repulsion(const tb_calculator* calc, const tb_structure* mol, double* erep) {
  if (!calc || !mol || !erep) return fail(TB_BAD_INPUT, "null argument");
  OneBatch ob(const_cast<tb_calculator*>(calc), mol);
  if (ob.st != TB_OK) return ob.st;
  tb_status st = run_setup_to_integrals(&ob.b, false);
  if (st != TB_OK) return st;
  return d2h(erep, ob.b.erep, mol->nat * 8);
}

tb_status tb_dispersion(const tb_calculator* calc, const tb_structure* mol, double* edisp, double* gradient,
                        double* sigma) {
  if (!calc || !mol || !edisp) return fail(TB_BAD_INPUT, "null argument");
  OneBatch ob(const_cast<tb_calculator*>(calc), mol);
  if (ob.st != TB_OK) return ob.st;
  const int nat = mol->nat;
  std::vector<double> g(3 * (size_t)nat, 0.0);
  if (calc->dp.d4) {
    tb_batch& b = ob.b;
    TB_CUDA(launch_dispersion(calc->dp, b.db, 1, b.d4cn, b.d4w, b.d4dw, b.d4e, b.d4dcn, b.d4g, b.e_disp, 0));
    TB_CUDA(cudaDeviceSynchronize());
    const tb_status st = d2h(edisp, b.d4e, nat * 8);
    if (st != TB_OK) return st;
    const tb_status sg = d2h(g.data(), b.d4g, g.size() * 8);
    if (sg != TB_OK) return sg;
  } else {
    for (int a = 0; a < nat; ++a) edisp[a] = 0.0;
  }
  if (gradient) std::memcpy(gradient, g.data(), g.size() * 8);
  if (sigma)
    for (int a = 0; a < 3; ++a)
      for (int c = 0; c < 3; ++c) {
        double s = 0.0;
        for (int i = 0; i < nat; ++i) s += g[3 * i + a] * mol->xyz[3 * i + c];
        sigma[3 * a + c] = s;
      }
  return TB_OK;
}

tb_status tb_get_hamiltonian(const tb_calculator* calc, const tb_structure* mol, double* S, double* H0, double* D,
                             double* Q) {
  if (!calc || !mol) return fail(TB_BAD_INPUT, "null argument");
  OneBatch ob(const_cast<tb_calculator*>(calc), mol);
  if (ob.st != TB_OK) return ob.st;
  tb_batch* b = &ob.b;
  tb_status st = run_setup_to_integrals(b, true);
  if (st != TB_OK) return st;
  const size_t nn = (size_t)b->n2_tot * 8;
  if (S && d2h(S, b->S, nn)) return TB_CUDA_ERROR;
  if (H0 && d2h(H0, b->H0, nn)) return TB_CUDA_ERROR;
  if (D && d2h(D, b->D, 3 * nn)) return TB_CUDA_ERROR;
  if (Q && d2h(Q, b->Q, 6 * nn)) return TB_CUDA_ERROR;
  return TB_OK;
}

tb_status tb_coulomb_potential(const tb_calculator* calc, const tb_structure* mol, const double* qsh,
                               const double* dpat, const double* qpat, double* vsh, double* vat, double* vdp,
                               double* vqp) {
  if (!calc || !mol || !qsh || !dpat || !qpat) return fail(TB_BAD_INPUT, "null argument");
  OneBatch ob(const_cast<tb_calculator*>(calc), mol);
  if (ob.st != TB_OK) return ob.st;
  tb_batch* b = &ob.b;
  tb_status st = run_setup_to_integrals(b, false);
  if (st != TB_OK) return st;
  const int nat = mol->nat, nsh = b->nsh_tot;
  TB_CUDA(cudaMemcpy(b->q_in, qsh, nsh * 8, cudaMemcpyHostToDevice));
  TB_CUDA(cudaMemcpy(b->q_in + nsh, dpat, 3 * nat * 8, cudaMemcpyHostToDevice));
  TB_CUDA(cudaMemcpy(b->q_in + nsh + 3 * nat, qpat, 6 * nat * 8, cudaMemcpyHostToDevice));
  const int one = 1;
  TB_CUDA(cudaMemcpy(b->ms.active, &one, sizeof(int), cudaMemcpyHostToDevice));
  const DevParams P = params_for(calc, 1.0);
  k_potential<<<dim3(1, nblk(std::max(nat, nsh), kPotTargets)), 32 * kPotTargets>>>(
      P, b->db, b->q_in, b->mrad, b->vsh, b->vat, b->vdp, b->vqp, b->ms.active, nullptr, nullptr);
  TB_LAUNCH_CHECK();
  if (vsh && d2h(vsh, b->vsh, nsh * 8)) return TB_CUDA_ERROR;
  if (vat && d2h(vat, b->vat, nat * 8)) return TB_CUDA_ERROR;
  if (vdp && d2h(vdp, b->vdp, 3 * nat * 8)) return TB_CUDA_ERROR;
  if (vqp && d2h(vqp, b->vqp, 6 * nat * 8)) return TB_CUDA_ERROR;
  return TB_OK;
}

tb_status tb_add_pot_to_h1(const tb_calculator* calc, const tb_structure* mol, const double* S, const double* H0,
                           const double* D, const double* Q, const double* vsh, const double* vat, const double* vdp,
                           const double* vqp, double* F) {
  if (!calc || !mol || !S || !H0 || !D || !Q || !vsh || !vat || !vdp || !vqp || !F)
    return fail(TB_BAD_INPUT, "null argument");
  OneBatch ob(const_cast<tb_calculator*>(calc), mol);
  if (ob.st != TB_OK) return ob.st;
  tb_batch* b = &ob.b;
  const int nat = mol->nat, nsh = b->nsh_tot;
  const size_t nn = (size_t)b->n2_tot * 8;
  TB_CUDA(cudaMemcpy(b->S, S, nn, cudaMemcpyHostToDevice));
  TB_CUDA(cudaMemcpy(b->H0, H0, nn, cudaMemcpyHostToDevice));
  TB_CUDA(cudaMemcpy(b->D, D, 3 * nn, cudaMemcpyHostToDevice));
  TB_CUDA(cudaMemcpy(b->Q, Q, 6 * nn, cudaMemcpyHostToDevice));
  TB_CUDA(cudaMemcpy(b->vsh, vsh, nsh * 8, cudaMemcpyHostToDevice));
  TB_CUDA(cudaMemcpy(b->vat, vat, nat * 8, cudaMemcpyHostToDevice));
  TB_CUDA(cudaMemcpy(b->vdp, vdp, 3 * nat * 8, cudaMemcpyHostToDevice));
  TB_CUDA(cudaMemcpy(b->vqp, vqp, 6 * nat * 8, cudaMemcpyHostToDevice));
  const int one = 1;
  TB_CUDA(cudaMemcpy(b->ms.active, &one, sizeof(int), cudaMemcpyHostToDevice));
  {
    const tb_status ss = raise_smem_limits();
    if (ss != TB_OK) return ss;
  }
  const int nt = (int)b->tiles32.size();
  k_fock<<<nt, 256, fock_smem_bytes()>>>(b->db, b->d_tiles32, nt, b->S, b->H0, b->D, b->Q, b->vsh, b->vat, b->vdp, b->vqp, b->F,
                      b->ms.active);
  TB_LAUNCH_CHECK();
  return d2h(F, b->F, nn);
}

}  // extern "C"

// ---------------------------------------------------------------- matrix batches
namespace {

// Minimal batch of nmat square matrices (sizes n[i]) for the eigensolver and
// Fermi entry points: only the AO/matrix offsets are meaningful.
struct MatBatch {
  Arena arena;
  DevBatch db{};
  MolState ms{};
  std::vector<int4> tiles;
  int4* d_tiles = nullptr;
  double *S = nullptr, *X = nullptr, *W = nullptr, *F = nullptr, *Z = nullptr, *w = nullptr, *focc = nullptr;
  int *perm = nullptr, *kdim = nullptr;
  long long n2 = 0, no = 0;
  int nmax = 0, nmax_in = 0;
  int64_t launches = 0;
  // matrices above the in-house size bound go to the library path (tb_large.cu)
  std::vector<int> big;
  std::vector<long long> h_moff;
  std::vector<int> h_ooff;
  LargeSolver lib;
  void* lib_work = nullptr;
  size_t lib_bytes = 0;
  int* lib_info = nullptr;
  TridPlan trid;
  int* d_tlist = nullptr;
  tb_status build(int nmat, const int32_t* n, int smem_tridiag = kTridMin) {
    std::vector<int> ooff(nmat + 1, 0);
    std::vector<long long> moff(nmat + 1, 0);
    for (int m = 0; m < nmat; ++m) {
      if (n[m] <= 0) return fail(TB_BAD_INPUT, "matrix size must be positive");
      ooff[m + 1] = ooff[m] + n[m];
      moff[m + 1] = moff[m] + (long long)n[m] * n[m];
      nmax = std::max(nmax, (int)n[m]);
      for (int t = 0; t < (n[m] + 63) / 64; ++t)
        for (int u = 0; u < (n[m] + 63) / 64; ++u) tiles.push_back(make_int4(m, t, u, 0));
    }
    int nbig_max = 0;
    for (int m = 0; m < nmat; ++m) {
      if (n[m] > kSyevMaxN) { big.push_back(m); nbig_max = std::max(nbig_max, (int)n[m]); }
      else nmax_in = std::max(nmax_in, (int)n[m]);
    }
    if (!big.empty()) {
      const std::string e = lib.workspace(nbig_max, &lib_bytes);
      if (!e.empty()) return fail(TB_CUDA_ERROR, "library eigensolver: " + e);
    }
    {
      std::vector<int> sizes(n, n + nmat);
      std::vector<char> in_house(nmat);
      for (int m = 0; m < nmat; ++m) in_house[m] = n[m] <= kSyevMaxN;
      trid.build(sizes, in_house, smem_tridiag);
    }
    h_moff = moff;
    h_ooff = ooff;
    n2 = moff[nmat];
    no = ooff[nmat];
    Layout L;
    size_t o_ooff = L.add((nmat + 1) * 4), o_moff = L.add((nmat + 1) * 8), o_t = L.add(tiles.size() * sizeof(int4));
    size_t o_S = L.add(n2 * 8), o_X = L.add(n2 * 8), o_W = L.add(n2 * 8), o_F = L.add(n2 * 8), o_Z = L.add(n2 * 8);
    size_t o_w = L.add(no * 8), o_f = L.add(no * 8), o_p = L.add(no * 4), o_k = L.add(nmat * 4);
    size_t o_st = L.add(nmat * 4), o_act = L.add(nmat * 4), o_nel = L.add(2 * nmat * 8), o_ets = L.add(nmat * 8),
           o_fw = L.add(nmat * 4), o_ef = L.add(nmat * 8), o_na = L.add(4);
    size_t o_lw = L.add(std::max<size_t>(lib_bytes, 16)), o_li = L.add((2 * big.size() + 2) * 4),
           o_tl = L.add((nmat + 1) * 4);
    TB_CUDA(arena.reserve(L.total));
    char* base = arena.base;
    TB_CUDA(cudaMemset(base, 0, L.total));
    TB_CUDA(cudaMemcpy(base + o_ooff, ooff.data(), (nmat + 1) * 4, cudaMemcpyHostToDevice));
    TB_CUDA(cudaMemcpy(base + o_moff, moff.data(), (nmat + 1) * 8, cudaMemcpyHostToDevice));
    TB_CUDA(cudaMemcpy(base + o_t, tiles.data(), tiles.size() * sizeof(int4), cudaMemcpyHostToDevice));
    db.nmol = nmat;
    db.ooff = at<int>(base, o_ooff);
    db.moff = at<long long>(base, o_moff);
    db.lib_above = kSyevMaxN;
    db.trid_min = trid.trid_min;
    db.trid_max = trid.trid_max;
    d_tlist = at<int>(base, o_tl);
    if (!trid.list.empty())
      TB_CUDA(cudaMemcpy(d_tlist, trid.list.data(), trid.list.size() * 4, cudaMemcpyHostToDevice));
    lib_work = base + o_lw;
    lib_info = at<int>(base, o_li);
    d_tiles = at<int4>(base, o_t);
    S = at<double>(base, o_S); X = at<double>(base, o_X); W = at<double>(base, o_W); F = at<double>(base, o_F);
    Z = at<double>(base, o_Z); w = at<double>(base, o_w); focc = at<double>(base, o_f);
    perm = at<int>(base, o_p); kdim = at<int>(base, o_k);
    ms.status = at<int>(base, o_st); ms.active = at<int>(base, o_act); ms.nel = at<double>(base, o_nel);
    ms.e_ts = at<double>(base, o_ets); ms.fermi_warn = at<int>(base, o_fw); ms.e_fermi = at<double>(base, o_ef);
    ms.n_active = at<int>(base, o_na);
    std::vector<int> ones(nmat, 1);
    TB_CUDA(cudaMemcpy(ms.active, ones.data(), nmat * 4, cudaMemcpyHostToDevice));
    return TB_OK;
  }
};

}  // namespace

extern "C" {

tb_status tb_sygvd_batch(int32_t nmat, const int32_t* n, const double* H, const double* S, double* w, double* C) {
  if (nmat <= 0 || !n || !H || !S || !w || !C) return fail(TB_BAD_INPUT, "null argument or empty batch");
  MatBatch mb;
  tb_status st = mb.build(nmat, n);
  if (st != TB_OK) return st;
  TB_CUDA(cudaMemcpy(mb.S, S, mb.n2 * 8, cudaMemcpyHostToDevice));
  TB_CUDA(cudaMemcpy(mb.F, H, mb.n2 * 8, cudaMemcpyHostToDevice));
  const DevBatch& B = mb.db;
  const int nt = (int)mb.tiles.size(), grid = std::min(nt, 148 * 8);
  k_cholesky<<<nmat, 256>>>(B, mb.S, mb.W, mb.ms.status, nullptr);
  k_trinv<<<nmat, 256>>>(B, mb.W, mb.X, mb.ms.status);
  for (size_t k = 0; k < mb.big.size(); ++k) {
    const int m = mb.big[k];
    const long long mo = mb.h_moff[m];
    const std::string e = mb.lib.factor(0, mb.S + mo, mb.X + mo, n[m], mb.lib_work, mb.lib_bytes, mb.lib_info + 2 * k,
                                        mb.ms.status + m);
    if (!e.empty()) return fail(TB_CUDA_ERROR, "library Cholesky: " + e);
  }
  k_gemm<<<grid, kGemmThreads>>>(B, mb.d_tiles, nt, mb.F, 0, mb.X, 0, nullptr, nullptr, nullptr, mb.W, 1.0, 0.0, mb.ms.active,
                                 kGemmKUpToJ);
  k_gemm<<<grid, kGemmThreads>>>(B, mb.d_tiles, nt, mb.X, 1, mb.W, 0, nullptr, nullptr, nullptr, mb.F, 1.0, 0.0, mb.ms.active,
                                 kGemmKUpToI | kGemmSym);
  const size_t smem = syev_smem_bytes(std::max(mb.nmax_in, 1));
  {
    const tb_status ss = raise_smem_limits();
    if (ss != TB_OK) return ss;
  }
  for (int c = 0; c < kTridClasses; ++c) {
    const int cnt = mb.trid.off[c + 1] - mb.trid.off[c];
    if (cnt == 0) continue;
    TB_CUDA(launch_trid(B, mb.F, mb.W, mb.ms.status, mb.ms.active, mb.d_tlist + mb.trid.off[c], cnt,
                        kTridClusterSizes[c], mb.trid.nmax[c], 0));
  }
  k_syev<<<nmat, kEigThreads, smem>>>(B, mb.F, mb.Z, mb.W, mb.w, mb.perm, mb.ms.status, mb.ms.active);
  std::vector<int> fstat(nmat, 0);
  if (!mb.big.empty()) TB_CUDA(cudaMemcpy(fstat.data(), mb.ms.status, nmat * 4, cudaMemcpyDeviceToHost));
  for (size_t k = 0; k < mb.big.size(); ++k) {
    const int m = mb.big[k];
    if (fstat[m] != kStOk) continue;  // S not positive definite: reported below
    const long long mo = mb.h_moff[m], vo = mb.h_ooff[m];
    const std::string e = mb.lib.syev(0, mb.F + mo, mb.Z + mo, mb.w + vo, mb.perm + vo, n[m], mb.lib_work,
                                      mb.lib_bytes, mb.lib_info + 2 * k + 1, mb.ms.status + m);
    if (!e.empty()) return fail(TB_CUDA_ERROR, "library eigensolver: " + e);
  }
  k_gemm<<<grid, kGemmThreads>>>(B, mb.d_tiles, nt, mb.X, 0, mb.Z, 1, mb.perm, nullptr, nullptr, mb.W, 1.0, 0.0, mb.ms.active,
                                 kGemmKFromI);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(TB_CUDA_ERROR, cudaGetErrorString(e));
  TB_CUDA(cudaMemcpy(w, mb.w, mb.no * 8, cudaMemcpyDeviceToHost));
  TB_CUDA(cudaMemcpy(C, mb.W, mb.n2 * 8, cudaMemcpyDeviceToHost));
  std::vector<int> status(nmat);
  TB_CUDA(cudaMemcpy(status.data(), mb.ms.status, nmat * 4, cudaMemcpyDeviceToHost));
  for (int m = 0; m < nmat; ++m)
    if (status[m] != kStOk) return fail((tb_status)status[m], "matrix " + std::to_string(m) + " failed");
  return TB_OK;
}

tb_status tb_fermi_filling(int32_t n, double nel, double kt, const double* emo, double* occ, double* efermi,
                           double* ts) {
  if (n <= 0 || !emo || !occ || !efermi || !ts) return fail(TB_BAD_INPUT, "null argument");
  MatBatch mb;
  tb_status st = mb.build(1, &n);
  if (st != TB_OK) return st;
  const double nels[2] = {nel, 0.0};
  TB_CUDA(cudaMemcpy(mb.w, emo, n * 8, cudaMemcpyHostToDevice));
  TB_CUDA(cudaMemcpy(mb.ms.nel, nels, 16, cudaMemcpyHostToDevice));
  {
    const tb_status ss = raise_smem_limits();
    if (ss != TB_OK) return ss;
  }
  k_fermi<<<1, 128, (size_t)n * 8>>>(mb.db, mb.w, kt, mb.focc, mb.kdim, mb.ms);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return fail(TB_CUDA_ERROR, cudaGetErrorString(e));
  TB_CUDA(cudaMemcpy(occ, mb.focc, n * 8, cudaMemcpyDeviceToHost));
  TB_CUDA(cudaMemcpy(ts, mb.ms.e_ts, 8, cudaMemcpyDeviceToHost));
  TB_CUDA(cudaMemcpy(efermi, mb.ms.e_fermi, 8, cudaMemcpyDeviceToHost));
  int fw = 0;
  TB_CUDA(cudaMemcpy(&fw, mb.ms.fermi_warn, 4, cudaMemcpyDeviceToHost));
  return fw ? fail(TB_FERMI_NOT_CONVERGED, "Fermi level iteration cap reached") : TB_OK;
}

}  // extern "C"

// ====================================================================== serving
struct tb_server {
  struct Req {
    int64_t ticket = 0;
    int nat = 0, uhf = 0, nsh = 0, nao = 0;
    double charge = 0.0;
    std::vector<int32_t> id;
    std::vector<double> xyz;
    int64_t bytes = 0;  // workspace estimate
    std::chrono::steady_clock::time_point t_submit;
  };
  struct Live {
    tb_batch* b = nullptr;
    cudaStream_t st = nullptr;
    std::vector<Req> reqs;
    std::vector<char> done;
    int64_t bytes = 0;
    bool inflight = false;  // an SCF iteration of this micro-batch is queued on st
    std::unique_ptr<Arena> ar;  // its workspace (from the pool)
    int* h_act = nullptr;       // pinned: active flags, copied after each iteration on st
    int h_cap = 0;
  };
  struct Done {
    int64_t ticket = 0;
    tb_result r{};
    std::vector<double> qat, qsh, dpat, qpat;
  };
  tb_calculator* calc = nullptr;
  tb_options opt{};
  int64_t budget = 0, resident = 0, next_ticket = 0;
  int max_batch = 1;
  std::deque<Req> queue;
  std::vector<Live> live;
  std::deque<Done> done;
  // Workspaces and streams of retired micro-batches are kept for reuse:
  // cudaFree would synchronise the whole device and stall the other streams.
  std::vector<std::unique_ptr<Arena>> pool;
  int64_t pooled = 0;
  std::vector<cudaStream_t> streams;
  // pinned host buffers for the micro-batches' active flags, reused like the
  // streams (pinning host memory is an operating-system call)
  std::vector<std::pair<int*, int>> pinned;
  int64_t compactions = 0;  // micro-batches moved to their unfinished structures
  // arrivals are collected this long (or until max_batch are queued, or while
  // nothing is resident) so that micro-batches hold more than one request
  double window_s = 0.002;
  ~tb_server() {
    for (Live& L : live) {
      delete L.b;
      if (L.st) cudaStreamDestroy(L.st);
    }
    for (cudaStream_t st : streams) cudaStreamDestroy(st);
    for (Live& L : live)
      if (L.h_act) cudaFreeHost(L.h_act);
    for (auto& p : pinned) cudaFreeHost(p.first);
  }
};

namespace {

// Device workspace of one structure in a batch, following batch_build's
// layout: 16 N^2 doubles of matrices (S, H0, D, Q, X, W, F, Z, P), 3 more N^2
// in the mixed-precision form, the pair lists, the Broyden history and the
// library workspace above the in-house size bound; 4 KiB per array of slack.
int64_t workspace_estimate(const tb_options& o, int nat, int nsh, int nao) {
  const double n2 = (double)nao * nao;
  double b = 128.0 * n2 + (o.precision == 1 ? 24.0 * n2 : 0.0);
  b += 4.0 * nat * (nat - 1);  // pair_i, pair_j
  // integral work space beyond X..P: the records' hij, the class list, the
  // item index (at most 9 shell pairs per atom pair) and the pair table
  b += 8.0 * nsh * nsh + 22.0 * nat * nat;
  const double mx = nsh + 9.0 * nat;
  b += 8.0 * mx * (4 + 2.0 * o.max_iter) + 8.0 * o.max_iter * o.max_iter;
  b += 8.0 * (30.0 * nao + 30.0 * nat);  // per-AO / per-atom vectors
  if (o.solver != 1 && (o.solver == 2 || nao > kSyevMaxN)) b += 16.0 * n2 + 64.0 * nao;
  return (int64_t)b + 64 * 4096;
}

tb_status server_admit(tb_server* s) {
  NvtxRange nv("tb.server_admit");
  if (s->queue.empty()) return TB_OK;
  const double waited =
      std::chrono::duration<double>(std::chrono::steady_clock::now() - s->queue.front().t_submit).count();
  if ((int)s->queue.size() < s->max_batch && waited < s->window_s && !s->live.empty()) return TB_OK;
  std::vector<tb_server::Req> take;
  int64_t est = 0;
  while (!s->queue.empty() && (int)take.size() < s->max_batch) {
    const tb_server::Req& r = s->queue.front();
    if (s->resident + est + r.bytes > s->budget) break;
    est += r.bytes;
    take.push_back(std::move(s->queue.front()));
    s->queue.pop_front();
  }
  if (take.empty()) return TB_OK;
  // release pooled workspaces that would push the total held past the budget
  while (!s->pool.empty() && s->resident + s->pooled + est > s->budget) {
    s->pooled -= (int64_t)s->pool.back()->cap;
    s->pool.pop_back();  // Arena frees its buffer
  }
  // smallest pooled workspace that fits, else a new one
  std::unique_ptr<Arena> ar;
  {
    int best = -1;
    for (int i = 0; i < (int)s->pool.size(); ++i)
      if ((int64_t)s->pool[i]->cap >= est && (best < 0 || s->pool[i]->cap < s->pool[best]->cap)) best = i;
    if (best >= 0) {
      ar = std::move(s->pool[best]);
      s->pool.erase(s->pool.begin() + best);
      s->pooled -= (int64_t)ar->cap;
    } else {
      ar.reset(new Arena());
    }
  }
  std::vector<tb_structure> mols(take.size());
  for (size_t i = 0; i < take.size(); ++i)
    mols[i] = {take[i].nat, take[i].uhf, take[i].charge, take[i].id.data(), take[i].xyz.data()};
  tb_server::Live L;
  L.b = new tb_batch();
  L.ar = std::move(ar);
  tb_status st = batch_build(s->calc, mols.data(), (int)mols.size(), &s->opt, L.b, L.ar.get());
  if (st == TB_OK) {
    if (!s->streams.empty()) {
      L.st = s->streams.back();
      s->streams.pop_back();
    } else if (cudaStreamCreateWithFlags(&L.st, cudaStreamNonBlocking) != cudaSuccess) {
      st = fail(TB_CUDA_ERROR, "cannot create a stream for a micro-batch");
    }
  }
  if (st == TB_OK) st = batch_setup(L.b, L.st);
  if (st != TB_OK) {
    delete L.b;
    if (L.st) cudaStreamDestroy(L.st);
    for (auto r = take.rbegin(); r != take.rend(); ++r) s->queue.push_front(std::move(*r));  // back in order
    return st;
  }
  L.bytes = (int64_t)L.ar->cap;
  s->resident += L.bytes;
  L.reqs = std::move(take);
  L.done.assign(L.reqs.size(), 0);
  s->live.push_back(std::move(L));
  return TB_OK;
}

// Compaction (continuous batching): once at most half of a micro-batch is
// still iterating, its unfinished structures continue in a new, smaller
// micro-batch -- built from their requests, set up (integrals and
// factorisation recomputed, the same bits), and given their SCF state
// (k_compact_state) -- and the old workspace returns to the pool, where
// admission can use it at once.  A structure's iterations and results are
// unchanged by the move: the kernels treat every structure independently.
tb_status server_compact(tb_server* s, tb_server::Live& L) {
  const int nmol = L.b->nmol;
  std::vector<int> keep;
  for (int m = 0; m < nmol; ++m)
    if (L.h_act[m] && !L.done[m]) keep.push_back(m);
  if (keep.empty() || nmol < 4 || 2 * (int)keep.size() > nmol) return TB_OK;
  NvtxRange nv("tb.server_compact");
  const int nk = (int)keep.size();
  std::vector<tb_structure> mols(nk);
  std::vector<tb_server::Req> reqs;
  for (int k = 0; k < nk; ++k) {
    tb_server::Req& r = L.reqs[keep[k]];
    mols[k] = {r.nat, r.uhf, r.charge, r.id.data(), r.xyz.data()};
  }
  int64_t est = 0;
  for (int k = 0; k < nk; ++k) est += L.reqs[keep[k]].bytes;
  std::unique_ptr<Arena> ar;
  {
    int best = -1;
    for (int i = 0; i < (int)s->pool.size(); ++i)
      if ((int64_t)s->pool[i]->cap >= est && (best < 0 || s->pool[i]->cap < s->pool[best]->cap)) best = i;
    if (best >= 0) {
      ar = std::move(s->pool[best]);
      s->pool.erase(s->pool.begin() + best);
      s->pooled -= (int64_t)ar->cap;
    } else {
      ar.reset(new Arena());
    }
  }
  tb_batch* nb = new tb_batch();
  tb_status st = batch_build(s->calc, mols.data(), nk, &s->opt, nb, ar.get());
  if (st == TB_OK) st = batch_setup(nb, L.st);
  if (st == TB_OK) {
    tb_batch* ob = L.b;
    TB_CUDA(cudaMemcpyAsync(nb->d_wflag, keep.data(), nk * sizeof(int), cudaMemcpyHostToDevice, L.st));
    ScfState so{ob->q_in, ob->dq, ob->dqlast, ob->qlast, ob->df, ob->u, ob->amat, ob->omega, ob->ms};
    ScfState sn{nb->q_in, nb->dq, nb->dqlast, nb->qlast, nb->df, nb->u, nb->amat, nb->omega, nb->ms};
    k_compact_state<<<nk, 256, 0, L.st>>>(ob->db, nb->db, nb->d_wflag, so, sn, s->opt.max_iter);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) st = fail(TB_CUDA_ERROR, std::string("compaction: ") + cudaGetErrorString(e));
    if (st == TB_OK) TB_CUDA(cudaMemcpyAsync(nb->ms.n_active, &nk, sizeof(int), cudaMemcpyHostToDevice, L.st));
    if (st == TB_OK) TB_CUDA(cudaStreamSynchronize(L.st));  // the old workspace is read until here
    // the host copies of the flags (active, status, phase: the library path
    // chooses its solver by them) were read by batch_setup before the move
    if (st == TB_OK) st = read_flags(nb, L.st);
  }
  if (st != TB_OK) {
    delete nb;
    s->pooled += (int64_t)ar->cap;
    s->pool.push_back(std::move(ar));
    return st;
  }
  nb->it = L.b->it;
  for (int k = 0; k < nk; ++k) reqs.push_back(std::move(L.reqs[keep[k]]));
  delete L.b;
  s->resident -= L.bytes;
  s->pooled += (int64_t)L.ar->cap;
  s->pool.push_back(std::move(L.ar));
  L.b = nb;
  L.ar = std::move(ar);
  L.bytes = (int64_t)L.ar->cap;
  s->resident += L.bytes;
  L.reqs = std::move(reqs);
  L.done.assign(nk, 0);
  s->compactions += 1;
  return TB_OK;
}

// Results of the structures of L that finished since the last call.
// Next SCF iteration of a micro-batch on its stream, followed on the same
// stream by the copy of its active flags into the micro-batch's pinned buffer
// (taken from the server's pool on first use).
tb_status server_launch(tb_server* s, tb_server::Live& L) {
  const int nmol = L.b->nmol;
  if (!L.h_act) {
    for (size_t i = 0; i < s->pinned.size(); ++i)
      if (s->pinned[i].second >= nmol) {
        L.h_act = s->pinned[i].first;
        L.h_cap = s->pinned[i].second;
        s->pinned.erase(s->pinned.begin() + i);
        break;
      }
    if (!L.h_act) {
      const int cap = std::max(nmol, 64);
      TB_CUDA(cudaMallocHost(&L.h_act, cap * sizeof(int)));
      L.h_cap = cap;
    }
  }
  const tb_status st = launch_iteration(L.b, L.st);
  if (st != TB_OK) return st;
  TB_CUDA(cudaMemcpyAsync(L.h_act, L.b->ms.active, nmol * sizeof(int), cudaMemcpyDeviceToHost, L.st));
  return TB_OK;
}

tb_status server_collect(tb_server* s, tb_server::Live& L) {
  const int nmol = L.b->nmol;
  // the active flags were copied on L.st after the iteration (server_launch),
  // which has finished: no device round trip here
  const std::vector<int> act(L.h_act, L.h_act + nmol);
  bool any = false;
  for (int m = 0; m < nmol; ++m) any |= !act[m] && !L.done[m];
  if (!any) return TB_OK;
  std::vector<tb_result> res(nmol);
  std::vector<tb_server::Done> out(nmol);
  for (int m = 0; m < nmol; ++m) {
    const tb_server::Req& r = L.reqs[m];
    out[m].qat.resize(r.nat); out[m].qsh.resize(r.nsh); out[m].dpat.resize(3 * r.nat); out[m].qpat.resize(6 * r.nat);
    res[m] = tb_result{};
    res[m].qat = out[m].qat.data(); res[m].qsh = out[m].qsh.data();
    res[m].dpat = out[m].dpat.data(); res[m].qpat = out[m].qpat.data();
  }
  const std::string keep = g_err;
  const tb_status rs = batch_results(L.b, res.data(), L.st);
  if (rs == TB_CUDA_ERROR) return rs;
  g_err = keep;  // per-structure statuses travel in the results
  for (int m = 0; m < nmol; ++m) {
    if (act[m] || L.done[m]) continue;
    L.done[m] = 1;
    out[m].ticket = L.reqs[m].ticket;
    out[m].r = res[m];
    s->done.push_back(std::move(out[m]));
  }
  return TB_OK;
}

}  // namespace

extern "C" {

tb_status tb_server_create(tb_calculator* calc, const tb_options* opt, int64_t hbm_budget_bytes, int32_t max_batch,
                           tb_server** out) {
  if (!calc || !out) return fail(TB_BAD_INPUT, "null argument");
  if (hbm_budget_bytes <= 0 || max_batch <= 0) return fail(TB_BAD_INPUT, "budget and max_batch must be positive");
  auto* s = new tb_server();
  s->calc = calc;
  if (opt) s->opt = *opt; else tb_default_options(&s->opt);
  s->opt.profile = 0;
  s->budget = hbm_budget_bytes;
  s->max_batch = max_batch;
  *out = s;
  return TB_OK;
}

tb_status tb_server_submit(tb_server* s, const tb_structure* mol, int64_t* ticket) {
  if (!s || !mol || !ticket) return fail(TB_BAD_INPUT, "null argument");
  if (mol->nat <= 0 || !mol->id || !mol->xyz) return fail(TB_BAD_INPUT, "empty or null structure");
  tb_server::Req r;
  int32_t nsh = 0, nao = 0;
  const tb_status bs = tb_basis_size(s->calc, mol, &nsh, &nao);
  if (bs != TB_OK) return bs;
  r.nat = mol->nat; r.uhf = mol->uhf; r.charge = mol->charge; r.nsh = nsh; r.nao = nao;
  r.id.assign(mol->id, mol->id + mol->nat);
  r.xyz.assign(mol->xyz, mol->xyz + 3 * (size_t)mol->nat);
  r.bytes = workspace_estimate(s->opt, r.nat, nsh, nao);
  if (r.bytes > s->budget) return fail(TB_CAPACITY_EXCEEDED, "structure needs more device memory than the budget");
  r.ticket = s->next_ticket++;
  r.t_submit = std::chrono::steady_clock::now();
  *ticket = r.ticket;
  s->queue.push_back(std::move(r));
  return TB_OK;
}

tb_status tb_server_step(tb_server* s, int32_t* n_resident, int32_t* n_queued, int64_t* bytes_resident) {
  NvtxRange nv("tb.server_step");
  if (!s) return fail(TB_BAD_INPUT, "null server");
  tb_status st = server_admit(s);
  if (st != TB_OK) return st;
  // Micro-batches progress independently: a micro-batch whose iteration has
  // finished on its stream is collected and given its next iteration at once;
  // one still running is left alone (the step does not wait for it).
  for (size_t i = 0; i < s->live.size();) {
    tb_server::Live& L = s->live[i];
    if (L.inflight) {
      const cudaError_t q = cudaStreamQuery(L.st);
      if (q == cudaErrorNotReady) { ++i; continue; }
      if (q != cudaSuccess) return fail(TB_CUDA_ERROR, std::string("micro-batch: ") + cudaGetErrorString(q));
      int na = 0;
      st = finish_iteration(L.b, L.st, &na);
      if (st != TB_OK) return st;
      st = server_collect(s, L);
      if (st != TB_OK) return st;
      L.inflight = false;
      if (na > 0 && L.b->it < L.b->opt.max_iter) {
        st = server_compact(s, L);
        if (st != TB_OK) return st;
      }
      if (na <= 0 || L.b->it >= L.b->opt.max_iter) {
        delete L.b;
        s->streams.push_back(L.st);
        if (L.h_act) s->pinned.push_back({L.h_act, L.h_cap});
        s->resident -= L.bytes;
        s->pooled += (int64_t)L.ar->cap;
        s->pool.push_back(std::move(L.ar));
        s->live.erase(s->live.begin() + i);
        continue;
      }
    }
    st = server_launch(s, L);
    if (st != TB_OK) return st;
    L.inflight = true;
    ++i;
  }
  if (n_resident || bytes_resident) {
    int32_t nr = 0;
    for (auto& L : s->live)
      for (char d : L.done) nr += !d;
    if (n_resident) *n_resident = nr;
    if (bytes_resident) *bytes_resident = s->resident + s->pooled;
  }
  if (n_queued) *n_queued = (int32_t)s->queue.size();
  return TB_OK;
}

int64_t tb_server_compactions(const tb_server* s) { return s ? s->compactions : 0; }

int32_t tb_server_poll(tb_server* s, int32_t max, int64_t* tickets, tb_result* results) {
  if (!s || max <= 0) return 0;
  int32_t k = 0;
  while (k < max && !s->done.empty()) {
    tb_server::Done& d = s->done.front();
    if (tickets) tickets[k] = d.ticket;
    if (results) {
      tb_result& r = results[k];
      double *qat = r.qat, *qsh = r.qsh, *dpat = r.dpat, *qpat = r.qpat;
      r = d.r;
      r.qat = qat; r.qsh = qsh; r.dpat = dpat; r.qpat = qpat;
      if (qat) std::memcpy(qat, d.qat.data(), d.qat.size() * sizeof(double));
      if (qsh) std::memcpy(qsh, d.qsh.data(), d.qsh.size() * sizeof(double));
      if (dpat) std::memcpy(dpat, d.dpat.data(), d.dpat.size() * sizeof(double));
      if (qpat) std::memcpy(qpat, d.qpat.data(), d.qpat.size() * sizeof(double));
    }
    s->done.pop_front();
    ++k;
  }
  return k;
}

void tb_server_destroy(tb_server* s) { delete s; }

}  // extern "C"
