// Context, device tables, launch shapes and the C-ABI of the walker engine.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/qwg.h"
#include "qwg_deck.hpp"
#include "qwg_launch.cuh"
#include "qwg_mo.cuh"

using namespace qwg;

namespace {

struct CudaError : std::runtime_error {
  explicit CudaError(const std::string& m) : std::runtime_error(m) {}
};

#define CK(x)                                                                                  \
  do {                                                                                         \
    cudaError_t e_ = (x);                                                                      \
    if (e_ != cudaSuccess) throw CudaError(std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

struct DevBuf {
  void* p = nullptr;
  size_t n = 0;
  DevBuf() = default;
  DevBuf(const DevBuf&) = delete;
  DevBuf& operator=(const DevBuf&) = delete;
  ~DevBuf() { if (p) cudaFree(p); }
  void alloc(size_t bytes) {
    if (p) { cudaFree(p); p = nullptr; }
    n = bytes;
    if (bytes) CK(cudaMalloc(&p, bytes));
  }
  template <class T> T* as() const { return (T*)p; }
};

template <class T>
static void upload(DevBuf& b, const std::vector<T>& v, cudaStream_t st) {
  b.alloc(std::max<size_t>(v.size() * sizeof(T), 16));
  if (!v.empty()) CK(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
}

// Kernel families: 8/16/32 the shared-memory walker kernels; 0 the
// HBM-resident kernels (up to kMaxOrbHBM orbitals per spin); kComplexFamily
// their complex-orbital variant.  mmax_for gives the size class of m orbitals
// per spin, -1 beyond this build (checked before a family is chosen).
constexpr int kMaxOrbHBM = 256;
static int mo_stride_for(int mmax, int nmo_max) { return mmax > 0 ? mmax : (nmo_max + 3) / 4 * 4; }
// -1: the HBM-resident kernels with complex orbitals (CORBITALS, or real
// orbitals at a nonzero k-point)
constexpr int kComplexFamily = -1;
static bool hbm_family(int mmax) { return mmax <= 0; }
static bool needs_complex(const HostSystem& H) {
  return H.complex_orbitals || H.kpt[0] != 0.0 || H.kpt[1] != 0.0 || H.kpt[2] != 0.0;
}
// F and G shells and the CUTOFF_MO evaluator run on the HBM-resident kernels only
static bool has_high_l(const HostSystem& H) {
  if (H.cutoff_mo) return true;
  for (const Shell& s : H.shells)
    if (s.sym >= SYM_10F) return true;
  return false;
}
static int mmax_for(int m) {
  if (m <= 8) return 8;
  if (m <= 16) return 16;
  if (m <= 32) return 32;
  if (m <= kMaxOrbHBM) return 0;
  return -1;
}
// Kernel family of a system (within the 256-orbital limit).  The shared-memory
// kernels win only for the smallest molecules (up to 8 orbitals per spin);
// above that, and for periodic cells at every size, the HBM-resident kernels
// keep more walkers resident per SM and run faster (DMC on B200: 8-atom cell
// 1.4x mixed / 1.6x FP64, 24-electron molecule 1.3x / 1.1x, 43-electron
// molecule 1.3x / 2.0x; the 14-electron molecule runs 0.64x on them, so it
// stays on the shared-memory kernels).  Expansions, F/G shells and CUTOFF_MO
// need the HBM-resident kernels, complex orbitals their complex variant.
// QWG_KERNEL_FAMILY=hbm|smem overrides the size rule for tuning.
static int kernel_family(const HostSystem& H) {
  if (needs_complex(H)) return kComplexFamily;
  const int smem = mmax_for(std::max(H.nmo[0], H.nmo[1]));
  if (H.detwt.size() > 1 || has_high_l(H)) return 0;
  int mm = (H.periodic || smem > 8) ? 0 : smem;
  if (const char* fam = getenv("QWG_KERNEL_FAMILY")) {
    if (strcmp(fam, "hbm") == 0) mm = 0;
    if (strcmp(fam, "smem") == 0) mm = smem;
  }
  return mm;
}

}  // namespace

struct qwg_ctx {
  std::string err;
  HostSystem H;
  int precision = QWG_FP64;
  int max_walkers = 0;
  int nwalk = 0;
  int mmax = 8;
  int wpc = 4;
  int wpc_sweep = 4;        // walkers per CTA of the move-phase kernel (KM_SWEEP)
  size_t smem_sweep = 0;
  bool split = true;        // DMC steps as sweep + local-energy launches (else one fused launch per chunk)
  int vmc_depth = 2;        // VMC Split_sampler DEPTH / DIVIDER (Vmc_method.cpp:75-82 defaults)
  double vmc_divider = 2.0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  long long launches = 0;
  // tables
  DevBuf d_shell_i, d_shell_obj, d_shell_cut, d_spline, d_spline64, d_moc, d_moc_im, d_image_kfac;
  DevBuf d_image_pos, d_gvec, d_gweight, d_ion_sin, d_ion_cos;
  DevBuf d_sub_seg, d_sub_idx;  // sub-cell candidate lists of the image sums
  int sub_n[3] = {0, 0, 0};
  double sub_inv_h[3] = {0, 0, 0};
  DevBuf d_det_c, d_det_ud, d_ud_cols;  // determinant expansion tables
  DevSys<double> sys_d{};
  DevSys<float> sys_f{};
  WLayout L{};
  size_t smem_bytes = 0;
  // walkers
  DevBuf d_R, d_R2, d_state, d_state2, d_scratch, d_branch, d_tm_cand, d_tm_moves;
  bool state_valid = false;
  bool have_scalars = false;  // WScal.eold / weight written by a block
  // io scratch
  DevBuf d_io, d_acc, d_dyn, d_src, d_neww, d_energy;
  size_t io_bytes = 0;
  // dynamics
  uint64_t step_counter = 0;
  uint64_t noalloc_step_counter = 0;  // steps of qwg_vmc_block_noalloc (its own random streams)
  uint64_t last_refresh = 0;
  uint64_t branch_counter = 0;
  qwg_dmc_params dmc{};
  bool dmc_ready = false;
  DevBuf d_hist, d_stats;
  double* h_stats = nullptr;          // pinned block statistics
  cudaGraph_t graph = nullptr;        // one DMC block
  cudaGraphExec_t gexec = nullptr;
  long long launches_per_block = 0;
  bool block_pending = false;
  double eref = 0, branch_start = 0, branch_stop = 0;
  std::vector<double> block_energies, block_weights;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // tensor-core MO contraction (mixed precision, real orbitals): the MO
  // coefficients of each spin transposed to [bn][kpad] and split into TF32
  // high and low parts, with their TMA tensor maps
  bool tc_ready = false;
  int tc_kpad = 0, tc_bn[2] = {0, 0};
  DevBuf d_tc_b;                 // [spin][hi, lo][256][kpad] FP32
  CUtensorMap tc_map_b[2][2];
  DevBuf d_tc_err;               // expired-wait code of the GEMM kernel
  DevBuf d_mo_scratch;           // qwg_mo_eval work buffers
  // tensor-core move schedule (mixed precision, HBM-resident real single
  // determinant): per electron move, the basis rows of every walker's
  // proposal (A operand, hi and lo planes) and the GEMM's MO columns
  bool tc_moves = false;
  int tc_ldd = 0;
  // population control on the device-wide sort at every population size
  // (QWG_BRANCH_DEVICE_WIDE=1; by default only above kBranchSmemMax walkers)
  bool branch_device_wide = false;
  DevBuf d_phases;  // walker-kernel phase counters (profiling builds, -DQWG_PHASES)
  DevBuf d_tc_a, d_tc_d;
};

namespace {

constexpr int kHistCap = 1 << 16;  // block energies kept on the device for E_ref
constexpr int kStatsLen = QWG_NACC + 2;  // block sums, E_T, E_ref (k_block_end output)

static DRadial to_dradial(const Radial& r) {
  DRadial d{};
  d.kind = r.kind;
  d.rcut = r.rcut;
  d.inv_rcut = 1.0 / r.rcut;
  d.a = r.a;
  d.b = r.b;
  d.c = r.kind == RAD_CUTOFF_CUSP ? 1.0 / (3.0 + r.b) : 0.0;
  return d;
}

template <typename Real>
static void fill_sys(qwg_ctx* c, DevSys<Real>& S, const std::vector<int>& obj_base) {
  const HostSystem& H = c->H;
  memset(&S, 0, sizeof(S));
  S.nelec = H.nelec; S.nup = H.nup; S.ndn = H.ndn; S.natoms = H.natoms;
  S.nbasis = H.nbasis; S.nshell = (int)H.shells.size();
  S.m[0] = H.nel_s[0]; S.m[1] = H.nel_s[1];
  S.mstride = mo_stride_for(c->mmax, std::max(H.nmo[0], H.nmo[1]));
  S.ndet = (int)H.detwt.size();
  for (int s = 0; s < 2; s++) { S.nud[s] = (int)H.udet_cols[s].size(); S.nmo_u[s] = H.nmo[s]; }
  S.det_c = c->d_det_c.as<double>();
  S.det_ud = c->d_det_ud.as<int>();
  S.ud_cols = c->d_ud_cols.as<int>();
  S.ion_ion = H.ion_ion;
  S.shell_i = c->d_shell_i.as<int4>();
  S.shell_obj = c->d_shell_obj.as<int2>();
  S.shell_cut = c->d_shell_cut.as<double>();
  S.spline = c->d_spline.as<Real>();
  S.spline64 = c->d_spline64.as<double>();
  S.moc = c->d_moc.as<Real>();
  S.moc_im = c->d_moc_im.as<Real>();
  S.image_kfac = c->d_image_kfac.as<double>();
  for (int d = 0; d < 3; d++) S.kpt[d] = H.kpt[d];
  S.kint = 1;
  for (int d = 0; d < 3; d++)
    if (H.kpt[d] != std::floor(H.kpt[d])) S.kint = 0;
  S.real_orb = H.complex_orbitals ? 0 : 1;
  S.cutoff_mo = H.cutoff_mo ? 1 : 0;
  S.xl = has_high_l(H) ? 1 : 0;
  S.npts = H.spline_npts;
  S.spacing = H.spline_spacing;
  S.inv_spacing = 1.0 / H.spline_spacing;
  // ---- limits of the parameter bank
  if (H.natoms > QWG_MAXA) throw InputError("more than 64 atoms: beyond this engine build");
  if ((int)H.shells.size() > QWG_MAXSHELL) throw InputError("more than 1024 basis shells: beyond this engine build");
  if ((int)H.ee.size() > QWG_MAXEE) throw InputError("more than 8 e-e Jastrow functions");
  // atom types = distinct labels
  std::vector<std::string> types;
  for (int a = 0; a < H.natoms; a++) {
    int t = (int)(std::find(types.begin(), types.end(), H.labels[a]) - types.begin());
    if (t == (int)types.size()) types.push_back(H.labels[a]);
    if (t >= QWG_MAXT) throw InputError("more than 8 atom labels: beyond this engine build");
    S.atom_type[a] = t;
    for (int d = 0; d < 3; d++) S.atom_pos[a][d] = H.atom_pos[3 * a + d];
    S.atom_charge[a] = H.atom_charge[a];
  }
  // centers: one basis object per center, shells contiguous and in object order
  std::vector<int> seen(H.natoms, 0);
  for (size_t k = 0; k < H.shells.size(); k++) {
    const Shell& sh = H.shells[k];
    int4& cs = S.center_seg[sh.center];
    if (!seen[sh.center]) {
      seen[sh.center] = 1;
      cs = make_int4((int)k, 0, obj_base[sh.obj], H.obj_count[sh.obj]);
      S.center_cut[sh.center] = sh.cutoff;
    } else if (obj_base[sh.obj] != cs.z) {
      throw InputError("one BASIS section per atom label is supported");
    }
    cs.y++;
    if (sh.first >= (1 << 16) || sh.k >= 256) throw InputError("basis too large for the shell table");
    S.shell_pack[k] = sh.sym | (sh.first << 4) | (sh.k << 20);
  }
  // periodic cell and basis image centers
  S.periodic = H.periodic ? 1 : 0;
  for (int i = 0; i < 3; i++) {
    S.origin[i] = H.origin[i];
    for (int j = 0; j < 3; j++) {
      S.lat[i][j] = H.lat[3 * i + j];
      S.normvec[i][j] = H.normvec[3 * i + j];
      S.corners[i][j] = H.corners[3 * i + j];
    }
  }
  S.h2q = H.smallest_height * H.smallest_height * 0.25;
  S.ortho = 1;
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++)
      if (i != j && H.lat[3 * i + j] != 0.0) S.ortho = 0;
  for (int k = 0; k < 27 && H.periodic; k++)
    for (int d = 0; d < 3; d++) S.lattice_basis[k][d] = H.lattice_basis[3 * k + d];
  S.alpha = H.alpha;
  S.ewald_const = H.ewald_const;
  for (int a = 0; a < H.natoms; a++) S.atom_images[a] = make_int2(H.image_first[a], H.image_count[a]);
  S.image_pos = c->d_image_pos.as<double>();
  if (H.periodic) {
    for (int i = 0; i < 3; i++) { S.sub_n[i] = c->sub_n[i]; S.sub_inv_h[i] = c->sub_inv_h[i]; }
    S.sub_seg = c->d_sub_seg.as<int2>();
    S.sub_idx = c->d_sub_idx.as<int>();
  }
  S.ng = (int)H.gweight.size();
  S.gvec = c->d_gvec.as<double>();
  S.gweight = c->d_gweight.as<double>();
  S.ion_sin = c->d_ion_sin.as<double>();
  S.ion_cos = c->d_ion_cos.as<double>();
  if (H.periodic && c->mmax != kComplexFamily)
    for (int a = 0; a < H.natoms; a++) {
      int nf = 0;
      for (auto& sh : H.shells)
        if (sh.center == a) nf += sh.nfunc;
      if (nf > QWG_MAXF_ATOM) throw InputError("periodic cells support at most 16 basis functions per atom");
    }
  // Jastrow
  S.nee = (int)H.ee.size();
  double ee_rc = 0.0;
  for (const Radial& r : H.ee) ee_rc = std::max(ee_rc, r.rcut);
  S.ee_rc2 = ee_rc * ee_rc * (1.0 + 1e-12);
  for (int k = 0; k < S.nee; k++) {
    S.ee[k] = to_dradial(H.ee[k]);
    S.ee_like[k] = H.ee_like[k];
    S.ee_unlike[k] = H.ee_unlike[k];
  }
  S.has_tb = H.tb.empty() ? 0 : 1;
  S.tb_stale_ei = H.tb_stale_ei ? 1 : 0;
  S.has_pp = H.has_pp ? 1 : 0;
  std::vector<int> type_done(types.size(), 0);
  for (int a = 0; a < H.natoms; a++) {
    const int t = S.atom_type[a];
    if (type_done[t]) continue;
    type_done[t] = 1;
    if (H.ei_count[a] > QWG_MAXEI) throw InputError("more than 8 e-n Jastrow functions on one atom");
    S.ei_n[t] = H.ei_count[a];
    for (int k = 0; k < H.ei_count[a]; k++) {
      S.ei[t][k] = to_dradial(H.ei[H.ei_first[a] + k]);
      S.onebody[t][k] = H.onebody[H.ei_first[a] + k];
    }
    if (H.tb_count[a] > QWG_MAXTB) throw InputError("more than 12 e-e-n terms on one atom");
    S.tb_n[t] = H.tb_count[a];
    S.tb_rc[t] = 0.0;
    for (int n = 0; n < H.tb_count[a]; n++) {
      const ThreeBodyTerm& q = H.tb[H.tb_first[a] + n];
      S.tb[t][n] = DTB{q.k - H.ei_first[a], q.l - H.ei_first[a], q.m, q.c, q.cu};
      S.tb_rc[t] = std::max({S.tb_rc[t], S.ei[t][S.tb[t][n].k].rcut, S.ei[t][S.tb[t][n].l].rcut});
    }
    const PPAtom& P = H.pp[a];
    S.pp_nchan[t] = P.nchan;
    S.pp_aip[t] = P.aip;
    S.pp_cutoff[t] = P.cutoff;
    if (P.nchan > 5) throw InputError("pseudopotential channels beyond l=3 are not supported");
    if ((int)P.term_n.size() > QWG_MAXPPT) throw InputError("more than 24 pseudopotential terms on one atom (both spins)");
    if (P.aip > QWG_MAXQ) throw InputError("quadratures above 32 points are not supported");
    for (int l = 0; l <= P.nchan && P.nchan; l++) {
      S.pp_term_first[t][l] = P.term_first[l];
      S.pp_term_first_dn[t][l] = P.term_first_dn[l];
    }
    S.pp_addzeff[t] = P.add_zeff ? 1 : 0;
    for (size_t n = 0; n < P.term_n.size(); n++) {
      S.pp_term[t][n][0] = P.term_n[n];
      S.pp_term[t][n][1] = P.term_a[n];
      S.pp_term[t][n][2] = P.term_c[n];
    }
    for (int q = 0; q < P.aip; q++) {
      for (int d = 0; d < 3; d++) S.pp_quad[t][q][d] = P.quad[3 * q + d];
      S.pp_w[t][q] = P.weight[q];
    }
  }
}

// Sub-cell candidate lists of the periodic image sums (every periodic basis
// evaluation, both precisions).  The cell is cut into n0 x n1 x n2
// parallelepipeds about 1 bohr high; for sub-cell s and atom c the list holds
// the indices of c's image centers, in image order, within cutoff(c) + R +
// 1e-3 bohr of the sub-cell's center, R its circumradius and cutoff(c) the
// largest cutoff of c's shells.  A position inside s is within R of that
// center, so every image within cutoff of it is listed, and a sum over the
// listed images adds the same terms in the same order as one over all images.
struct SubcellLists {
  int n[3] = {0, 0, 0};
  double inv_h[3] = {0, 0, 0};
  std::vector<int2> seg;
  std::vector<int> idx;
};
static SubcellLists make_subcell_lists(const HostSystem& H) {
  SubcellLists L;
  if (!H.periodic) return L;
  const int A = H.natoms;
  const double* a = H.lat;
  double vol;
  {
    const double* u = a + 3; const double* v = a + 6;
    const double cx = u[1] * v[2] - u[2] * v[1], cy = u[2] * v[0] - u[0] * v[2], cz = u[0] * v[1] - u[1] * v[0];
    vol = std::fabs(a[0] * cx + a[1] * cy + a[2] * cz);
  }
  for (int i = 0; i < 3; i++) {
    const double* u = a + 3 * ((i + 1) % 3); const double* v = a + 3 * ((i + 2) % 3);
    const double cx = u[1] * v[2] - u[2] * v[1], cy = u[2] * v[0] - u[0] * v[2], cz = u[0] * v[1] - u[1] * v[0];
    const double h = vol / std::sqrt(cx * cx + cy * cy + cz * cz);
    L.n[i] = std::max(1, std::min(16, (int)std::ceil(h / 1.0)));
    const double* nv = H.normvec + 3 * i;
    L.inv_h[i] = 1.0 / (nv[0] * a[3 * i] + nv[1] * a[3 * i + 1] + nv[2] * a[3 * i + 2]);
  }
  double R = 0.0;  // circumradius of a sub-cell: the longest half body diagonal
  const int sg[4][3] = {{1, 1, 1}, {1, 1, -1}, {1, -1, 1}, {-1, 1, 1}};
  for (const auto& g : sg) {
    double v[3];
    for (int j = 0; j < 3; j++)
      v[j] = 0.5 * (g[0] * a[j] / L.n[0] + g[1] * a[3 + j] / L.n[1] + g[2] * a[6 + j] / L.n[2]);
    R = std::max(R, std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]));
  }
  std::vector<double> cmax(A, 0.0);
  for (const Shell& s : H.shells)
    cmax[s.center] = std::max(cmax[s.center], std::max(s.cutoff, H.cutoff_mo ? s.fcut : 0.0));
  const int nsub = L.n[0] * L.n[1] * L.n[2];
  L.seg.resize((size_t)nsub * A);
  for (int g0 = 0; g0 < L.n[0]; g0++)
    for (int g1 = 0; g1 < L.n[1]; g1++)
      for (int g2 = 0; g2 < L.n[2]; g2++) {
        const int s = (g0 * L.n[1] + g1) * L.n[2] + g2;
        double ctr[3];
        for (int j = 0; j < 3; j++)
          ctr[j] = H.origin[j] + (g0 + 0.5) / L.n[0] * a[j] + (g1 + 0.5) / L.n[1] * a[3 + j] +
                   (g2 + 0.5) / L.n[2] * a[6 + j];
        for (int c = 0; c < A; c++) {
          const int first = (int)L.idx.size();
          const double reach = cmax[c] + R + 1e-3;
          for (int m = H.image_first[c]; m < H.image_first[c] + H.image_count[c]; m++) {
            const double dx = H.image_pos[3 * m] - ctr[0], dy = H.image_pos[3 * m + 1] - ctr[1],
                         dz = H.image_pos[3 * m + 2] - ctr[2];
            if (dx * dx + dy * dy + dz * dz < reach * reach) L.idx.push_back(m);
          }
          L.seg[(size_t)s * A + c] = make_int2(first, (int)L.idx.size() - first);
        }
      }
  return L;
}

static void build_tables(qwg_ctx* c) {
  const HostSystem& H = c->H;
  cudaStream_t st = c->stream;
  const int A = H.natoms;
  // interval-major spline tables: object o occupies npts x count_o x 4 values
  const int npts = H.spline_npts;
  std::vector<int> obj_base(H.obj_first.size());
  size_t total4 = 0;
  for (size_t o = 0; o < H.obj_first.size(); o++) {
    obj_base[o] = (int)total4;
    total4 += (size_t)npts * H.obj_count[o];
  }
  std::vector<double> il(total4 * 4, 0.0);
  for (size_t o = 0; o < H.obj_first.size(); o++)
    for (int i = 0; i < npts; i++)
      for (int k = 0; k < H.obj_count[o]; k++)
        for (int q = 0; q < 4; q++)
          il[((size_t)obj_base[o] + (size_t)i * H.obj_count[o] + k) * 4 + q] =
              H.spline_coef[((size_t)(H.obj_first[o] + k) * npts + i) * 4 + q];
  std::vector<int4> si;
  std::vector<int2> so;
  std::vector<double> sc;
  for (size_t k = 0; k < H.shells.size(); k++) {
    const Shell& s = H.shells[k];
    si.push_back(make_int4(s.center, s.sym, s.first, s.k));
    so.push_back(make_int2(obj_base[s.obj], H.obj_count[s.obj]));
    sc.push_back(H.cutoff_mo ? s.fcut : s.cutoff);  // CUTOFF_MO: each function inside its own cutoff
  }
  (void)A;
  upload(c->d_shell_i, si, st);
  upload(c->d_shell_obj, so, st);
  upload(c->d_shell_cut, sc, st);
  // MO coefficients padded to the orbital stride, both spins
  const int mm = mo_stride_for(c->mmax, std::max(H.nmo[0], H.nmo[1]));
  std::vector<double> moc((size_t)2 * H.nbasis * mm, 0.0), moc_im(moc.size(), 0.0);
  for (int s = 0; s < 2; s++)
    for (int f = 0; f < H.nbasis; f++)
      for (int i = 0; i < H.nmo[s]; i++) {
        moc[((size_t)s * H.nbasis + f) * mm + i] = H.moc[s][(size_t)f * H.nmo[s] + i];
        moc_im[((size_t)s * H.nbasis + f) * mm + i] = H.moc_im[s][(size_t)f * H.nmo[s] + i];
      }
  if (c->mmax != kComplexFamily) moc_im.clear();
  // determinant expansion: weights, (up, down) spin-determinant of each
  // determinant, union columns of every distinct spin-determinant
  upload(c->d_det_c, H.detwt, st);
  upload(c->d_det_ud, H.det_ud, st);
  std::vector<int> ucols((size_t)2 * QWG_MAXUD * mm, 0);
  for (int s = 0; s < 2; s++)
    for (size_t u = 0; u < H.udet_cols[s].size(); u++)
      for (size_t i = 0; i < H.udet_cols[s][u].size(); i++) ucols[((size_t)s * QWG_MAXUD + u) * mm + i] = H.udet_cols[s][u][i];
  upload(c->d_ud_cols, ucols, st);
  upload(c->d_spline64, il, st);
  if (c->precision == QWG_FP64) {
    upload(c->d_spline, il, st);
    upload(c->d_moc, moc, st);
    upload(c->d_moc_im, moc_im, st);
  } else {
    std::vector<float> sf(il.begin(), il.end());
    std::vector<float> mf(moc.begin(), moc.end());
    std::vector<float> mfi(moc_im.begin(), moc_im.end());
    upload(c->d_spline, sf, st);
    upload(c->d_moc, mf, st);
    upload(c->d_moc_im, mfi, st);
  }
  upload(c->d_image_pos, H.image_pos, st);
  // k-point factor of every image center: e^{i pi k.n} (complex orbitals) or
  // cos(pi k.n) (real orbitals), n the image's lattice translation
  // (eval_kpoint_fac, MO_matrix.h:333-342)
  std::vector<double> kfac(H.image_pos.size() / 3 * 2, 0.0);
  for (size_t m = 0; m < kfac.size() / 2; m++) {
    const double dot = H.kpt[0] * H.image_shift[3 * m] + H.kpt[1] * H.image_shift[3 * m + 1] +
                       H.kpt[2] * H.image_shift[3 * m + 2];
    kfac[2 * m] = std::cos(dot * M_PI);
    kfac[2 * m + 1] = H.complex_orbitals ? std::sin(dot * M_PI) : 0.0;
  }
  upload(c->d_image_kfac, kfac, st);
  upload(c->d_gvec, H.gvec, st);
  upload(c->d_gweight, H.gweight, st);
  upload(c->d_ion_sin, H.ion_sin, st);
  upload(c->d_ion_cos, H.ion_cos, st);
  if (H.periodic) {
    const SubcellLists sl = make_subcell_lists(H);
    upload(c->d_sub_seg, sl.seg, st);
    upload(c->d_sub_idx, sl.idx, st);
    for (int i = 0; i < 3; i++) { c->sub_n[i] = sl.n[i]; c->sub_inv_h[i] = sl.inv_h[i]; }
  }
  fill_sys<double>(c, c->sys_d, obj_base);
  fill_sys<float>(c, c->sys_f, obj_base);
  const void* req[] = {c->sys_d.shell_i, c->sys_d.shell_obj, c->sys_d.shell_cut, c->sys_d.spline,
                       c->sys_d.spline64, c->sys_d.moc};
  for (const void* p : req)
    if (!p) throw std::runtime_error("internal: device table pointer left unset");
}

static int align16(int x) { return (x + 15) / 16 * 16; }

static void make_layout(qwg_ctx* c) {
  const HostSystem& H = c->H;
  const int N = H.nelec, A = H.natoms;
  const bool hbm = hbm_family(c->mmax);
  const int mm = mo_stride_for(c->mmax, std::max(H.nmo[0], H.nmo[1]));
  // complex orbitals: planar complex inverse, MO rows, basis rows and
  // projected coefficients (twice the real sizes)
  const int cf = c->mmax == kComplexFamily ? 2 : 1;
  const int rs = (c->precision == QWG_FP64 ? 8 : 4) * cf;
  WLayout& L = c->L;
  L.mstride = mm;
  int o = 0;
  L.scal = o; o = align16(o + (int)sizeof(WScal));
  L.R = o; o = align16(o + 8 * 3 * N);
  L.nud = std::max<int>(1, (int)std::max(H.udet_cols[0].size(), H.udet_cols[1].size()));
  L.inv = o; o = align16(o + rs * 2 * L.nud * mm * mm);
  L.mov = o; o = align16(o + rs * N * mm * 4);
  L.gU = o; o = align16(o + 8 * 3 * N);
  L.lU = o; o = align16(o + 8 * N);
  L.udl = L.mdt = L.mdv = L.mdr = 0;
  if (H.detwt.size() > 1) {
    L.udl = o; o = align16(o + 8 * 2 * L.nud * 2);
    L.mdt = o; o = align16(o + 8 * (QWG_MAXDET + 2 + 2 * QWG_MAXUD));
  }
  L.state_bytes = o;
  // scratch (offsets from its own start): the move/re-inversion phase and the
  // pseudopotential phase are never live together, so their buffers share
  // one region
  o = 0;
  L.bas = o; o = align16(o + rs * H.nbasis * 5);
  L.newcol = o; o = align16(o + rs * mm * 5);
  L.dG = o; o = align16(o + 8 * 4 * N);
  L.lu = o; o = align16(o + 8 * cf * (mm * 2 * mm + mm));
  if (H.detwt.size() > 1) {
    L.mdv = o; o = align16(o + 8 * mm * mm);
    L.mdr = o; o = align16(o + 8 * QWG_MAXUD * 5);
  }
  const int move_end = o;
  // pseudopotential phase for a chunk of wc electrons: items (wc x atoms),
  // Jastrow values, rotation, projected coefficients (wc x nbasis)
  auto pp_bytes = [&](int wc) {
    int q = align16((int)sizeof(PPItem) * wc * A);
    q = align16(q + 8 * N);
    q = align16(q + 8 * 9);
    return align16(q + rs * H.nbasis * wc);
  };
  if (hbm) {
    L.wchunk = std::min(N, 64);
  } else {
    // all electrons in one chunk if a walker still fits the budget of 4
    // walkers x 4 CTAs per SM, else as many as fit (at least 4)
    const int budget = (227 * 1024 - 1024) / 16 - L.state_bytes;
    const int room = std::max(budget, move_end);
    int wc = N;
    while (wc > 4 && pp_bytes(wc) > room) wc--;
    L.wchunk = std::max(1, std::min(N, wc));
  }
  L.items = 0;
  o = align16((int)sizeof(PPItem) * L.wchunk * A);
  L.Ue = o; o = align16(o + 8 * N);
  L.rot = o; o = align16(o + 8 * 9);
  L.wproj = o; o = align16(o + rs * H.nbasis * L.wchunk * L.nud);
  L.scratch_bytes = std::max(o, move_end);
  L.bytes = L.state_bytes + L.scratch_bytes;
  L.sweep_bytes = L.state_bytes + move_end;
  if (hbm) {
    c->wpc = c->wpc_sweep = 4;
    c->smem_bytes = c->smem_sweep = 0;
    return;
  }
  int wps = 4;  // same rule for the move kernel's smaller footprint
  while (wps > 1 && (size_t)wps * L.sweep_bytes > 110 * 1024) wps--;
  c->wpc_sweep = wps;
  c->smem_sweep = (size_t)wps * L.sweep_bytes;
  // walkers per CTA: up to 4 while the CTA stays under ~110 KB (2 CTAs/SM)
  int wpc = 4;
  while (wpc > 1 && (size_t)wpc * L.bytes > 110 * 1024) wpc--;
  c->wpc = wpc;
  c->smem_bytes = (size_t)wpc * L.bytes;
  if (c->smem_bytes > 227 * 1024) throw InputError("system too large for the shared-memory walker kernel");
}

// Dynamic shared memory of the branching kernel for W walkers, or 0 when the
// sort runs in global memory (populations above kBranchSmemMax walkers).
constexpr int kBranchSmemMax = 8192;
constexpr int kMaxDmcWalkers = 1 << 18;
static size_t branch_bytes(int W) {
  int p2 = 1;
  while (p2 < W) p2 <<= 1;
  return (size_t)p2 * (8 + 4) + (size_t)W * 4 + 16 + (size_t)W * 8;
}
static size_t branch_smem(int W) { return W <= kBranchSmemMax ? branch_bytes(W) : 0; }

// Device-wide population control (populations above kBranchSmemMax): the
// sort's double buffers, counts, new weights, digit counts and partial sums
// in the context's branch buffer.
static size_t align256(size_t b) { return (b + 255) / 256 * 256; }
static size_t branch_big_bytes(int W, BranchBig* G, unsigned char* base) {
  const int ntiles = (W + RADIX_TILE - 1) / RADIX_TILE, nprep = (W + 255) / 256, npb = (W / 2 + 255) / 256 + 1;
  size_t o = 0;
  auto take = [&](size_t bytes) { size_t at = o; o += align256(bytes); return at; };
  const size_t k0 = take((size_t)W * 8), k1 = take((size_t)W * 8), i0 = take((size_t)W * 4),
               i1 = take((size_t)W * 4), cn = take((size_t)W * 4), nw = take((size_t)W * 8),
               hi = take((size_t)256 * ntiles * 4), ps = take((size_t)nprep * 8), np = take((size_t)npb * 4);
  if (G && base) {
    G->key[0] = (unsigned long long*)(base + k0); G->key[1] = (unsigned long long*)(base + k1);
    G->idx[0] = (int*)(base + i0); G->idx[1] = (int*)(base + i1);
    G->cnt = (int*)(base + cn); G->nw = (double*)(base + nw); G->hist = (int*)(base + hi);
    G->psum = (double*)(base + ps); G->npair = (int*)(base + np);
    G->ntiles = ntiles; G->nprep = nprep; G->npairblk = npb;
  }
  return o;
}

// Device bytes a context holds for max_walkers walkers (the allocations of
// qwg_create plus the evaluation buffers qwg_dmc_init sizes).
constexpr int kTcMinWalkers = 1024;

// The tensor-core move schedule serves the mixed-precision HBM-resident
// kernels with real orbitals and one determinant, by default when the
// contraction of a move (basis functions x orbitals per spin) is at least
// kTcMinContraction: measured on one B200 (DMC, mixed), the schedule is 1.10x
// the one-launch CUDA-core sweep on a 128-electron cell (416 x 64), 0.92-0.98x
// on a 72-electron molecule (180 x 36) and 0.98-1.00x on a 32-electron cell
// (104 x 16), since it pays three launches per electron.  QWG_TC_MOVES=1
// forces it on, QWG_TC_MOVES=0 off (to time either beside the other).
constexpr size_t kTcMinContraction = 16384;
static bool tc_moves_eligible(const qwg_ctx* c) {
  if (!(c->precision == QWG_MIXED && c->mmax == 0 && c->H.detwt.size() <= 1 && c->H.nmo[0] <= 256 &&
        c->H.nmo[1] <= 256))
    return false;
  const char* env = std::getenv("QWG_TC_MOVES");
  if (env && env[0] == '0') return false;
  if (env && env[0] == '1') return true;
  return (size_t)c->H.nbasis * (size_t)std::max(c->H.nmo[0], c->H.nmo[1]) >= kTcMinContraction;
}

static size_t tc_moves_bytes(const qwg_ctx* c, size_t W) {
  const size_t kpad = ((size_t)c->H.nbasis + 31) / 32 * 32;
  size_t ldd = 16;
  for (int s = 0; s < 2; s++) ldd = std::max(ldd, ((size_t)c->H.nmo[s] + 15) / 16 * 16);
  return W * 5 * (kpad * 8 + ldd * 4) + 2 * 2 * 256 * kpad * 4 + 16;
}

static size_t footprint_bytes(const qwg_ctx* c, int max_walkers) {
  const HostSystem& H = c->H;
  const size_t rs = c->precision == QWG_FP64 ? 8 : 4, N = H.nelec, W = max_walkers;
  size_t total4 = 0;
  for (size_t o = 0; o < H.obj_first.size(); o++) total4 += (size_t)H.spline_npts * H.obj_count[o];
  const size_t ms = mo_stride_for(c->mmax, std::max(H.nmo[0], H.nmo[1]));
  const size_t cf = c->mmax == kComplexFamily ? 2 : 1;
  size_t b = total4 * 4 * (8 + rs) + 2 * (size_t)H.nbasis * ms * rs * cf + H.shells.size() * 32 +
             H.image_pos.size() * 8 * 5 / 3 + H.gvec.size() * 8 + 3 * H.gweight.size() * 8;
  if (H.periodic) {
    const SubcellLists sl = make_subcell_lists(H);
    b += sl.seg.size() * sizeof(int2) + sl.idx.size() * sizeof(int);
  }
  b += W * (2 * 3 * N * 8 + 2 * (size_t)c->L.state_bytes + (hbm_family(c->mmax) ? (size_t)c->L.scratch_bytes : 0) + 20);
  b += W * 8 * (9 + 5 + 4 * N);  // evaluation outputs (qwg_eval / qwg_dmc_init)
  if (tc_moves_eligible(c)) b += tc_moves_bytes(c, W);
  b += sizeof(BlockAcc) * 1024 + DYN_COUNT * 8 + (size_t)kHistCap * 8 + kStatsLen * 8;
  if (max_walkers > kBranchSmemMax) b += branch_big_bytes(max_walkers, nullptr, nullptr);
  return b;
}

// Raise a kernel's dynamic shared-memory limit once to the largest size any
// context asked for (never during a stream capture: callers make a plain
// launch of every kernel before capturing it).
template <class K>
static void ensure_smem_attr(K kern, size_t bytes) {
  static std::mutex mu;
  static std::map<const void*, size_t> done;
  std::lock_guard<std::mutex> lock(mu);
  size_t& have = done[(const void*)kern];
  if (bytes > have) {
    CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes));
    have = bytes;
  }
}

template <typename Real, int MM>
static void launch_walkers_t(qwg_ctx* c, const DevSys<Real>& S, const StepParams& P, const EvalIO& io, int mode,
                             int nwalk) {
  const bool sw = mode == KM_SWEEP || mode == KM_TMOVE;  // move-phase shared-memory layout
  CK((launch_walker_kernels<Real, MM>(S, c->L, P, io, mode, nwalk, sw ? c->wpc_sweep : c->wpc,
                                      sw ? c->smem_sweep : c->smem_bytes, c->stream)));
  if (nwalk > 0) c->launches++;
}

static void launch_walkers(qwg_ctx* c, const StepParams& P, const EvalIO& io, int mode, int nwalk) {
  if (c->precision == QWG_FP64) {
    switch (c->mmax) {
      case 8: launch_walkers_t<double, 8>(c, c->sys_d, P, io, mode, nwalk); break;
      case 16: launch_walkers_t<double, 16>(c, c->sys_d, P, io, mode, nwalk); break;
      case 32: launch_walkers_t<double, 32>(c, c->sys_d, P, io, mode, nwalk); break;
      case kComplexFamily: launch_walkers_t<double, -1>(c, c->sys_d, P, io, mode, nwalk); break;
      default: launch_walkers_t<double, 0>(c, c->sys_d, P, io, mode, nwalk); break;
    }
  } else {
    switch (c->mmax) {
      case 8: launch_walkers_t<float, 8>(c, c->sys_f, P, io, mode, nwalk); break;
      case 16: launch_walkers_t<float, 16>(c, c->sys_f, P, io, mode, nwalk); break;
      case 32: launch_walkers_t<float, 32>(c, c->sys_f, P, io, mode, nwalk); break;
      case kComplexFamily: launch_walkers_t<float, -1>(c, c->sys_f, P, io, mode, nwalk); break;
      default: launch_walkers_t<float, 0>(c, c->sys_f, P, io, mode, nwalk); break;
    }
  }
}

static StepParams base_params(qwg_ctx* c) {
  StepParams P{};
  P.nwalk = c->nwalk;
  P.R = c->d_R.as<double>();
  P.state = c->d_state.as<unsigned char>();
  P.scratch = c->d_scratch.p ? c->d_scratch.as<unsigned char>() : nullptr;
  P.acc = c->d_acc.as<BlockAcc>();
  P.etrial = c->d_dyn.as<double>();
  P.refresh = 1;
  P.vmc_depth = c->vmc_depth;
  P.vmc_divider = c->vmc_divider;
  P.phases = c->d_phases.p ? c->d_phases.as<unsigned long long>() : nullptr;
  if (c->tc_moves) {
    P.tc_kpad = c->tc_kpad;
    P.tc_ldd = c->tc_ldd;
    P.tc_ahi = c->d_tc_a.as<float>();
    P.tc_alo = P.tc_ahi + (size_t)c->max_walkers * 5 * c->tc_kpad;
    P.tc_D = c->d_tc_d.as<float>();
  }
  return P;
}

// ---------------------------------------------------------------------------
// Tensor-core MO contraction: tensor maps and the split-TF32 coefficients.

typedef CUresult (*TensorMapEncodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                         const cuuint64_t*, const cuuint32_t*, const cuuint32_t*,
                                         CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                         CUtensorMapFloatOOBfill);

static TensorMapEncodeTiled tensor_map_encoder() {
  static TensorMapEncodeTiled fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (TensorMapEncodeTiled)p;
  });
  return fn;
}

// Tensor map of a row-major FP32 array [outer][inner] read in boxes of 32 x
// box_outer elements with the 128-byte swizzle (inner must be a multiple of
// 32 and the base 16-byte aligned; rows past outer read as zeros).
static void tc_map(CUtensorMap* m, const float* base, uint64_t inner, uint64_t outer, uint32_t box_outer) {
  TensorMapEncodeTiled enc = tensor_map_encoder();
  if (!enc) throw CudaError("cuTensorMapEncodeTiled is not available from the driver");
  if (inner % TC_BK != 0 || ((uintptr_t)base & 15) != 0) throw CudaError("tensor map: bad inner extent or alignment");
  cuuint64_t dims[2] = {inner, outer};
  cuuint64_t strides[1] = {inner * sizeof(float)};
  cuuint32_t box[2] = {(cuuint32_t)TC_BK, box_outer};
  cuuint32_t es[2] = {1, 1};
  const CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, (void*)base, dims, strides, box, es,
                         CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                         CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw CudaError("cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
}

// FP32 rounded to TF32 (10 explicit mantissa bits), to nearest, ties away.
static float tf32_round(float x) {
  uint32_t u;
  std::memcpy(&u, &x, 4);
  if ((u & 0x7f800000u) != 0x7f800000u) {
    u += 0x1000u;
    u &= 0xffffe000u;
  }
  float r;
  std::memcpy(&r, &u, 4);
  return r;
}

static void tc_setup(qwg_ctx* c) {
  if (c->tc_ready) return;
  const HostSystem& H = c->H;
  const int kpad = (H.nbasis + TC_BK - 1) / TC_BK * TC_BK;
  c->tc_kpad = kpad;
  std::vector<float> b((size_t)2 * 2 * 256 * kpad, 0.f);
  for (int s = 0; s < 2; s++) {
    if (H.nmo[s] > 256) throw InputError("the tensor-core MO contraction takes at most 256 orbitals per spin");
    c->tc_bn[s] = std::max(16, (H.nmo[s] + 15) / 16 * 16);
    for (int j = 0; j < H.nmo[s]; j++)
      for (int f = 0; f < H.nbasis; f++) {
        const double v = H.moc[s][(size_t)f * H.nmo[s] + j];
        const float hi = tf32_round((float)v);
        b[(((size_t)s * 2 + 0) * 256 + j) * kpad + f] = hi;
        b[(((size_t)s * 2 + 1) * 256 + j) * kpad + f] = tf32_round((float)(v - (double)hi));
      }
  }
  upload(c->d_tc_b, b, c->stream);
  for (int s = 0; s < 2; s++)
    for (int h = 0; h < 2; h++)
      tc_map(&c->tc_map_b[s][h], c->d_tc_b.as<float>() + ((size_t)s * 2 + h) * 256 * kpad, kpad, c->tc_bn[s],
             (uint32_t)c->tc_bn[s]);
  c->d_tc_err.alloc(16);
  c->tc_ready = true;
}

// D[r][j] (row stride ldd) = sum_k (a_hi + a_lo)[r][k] (b_hi + b_lo)[j][k]
// for the orbitals j of one spin, rows r < rows; split-TF32 tensor cores.
static void tc_gemm(qwg_ctx* c, const float* a_hi, const float* a_lo, int rows, int spin, float* D, int ldd) {
  const int bn = c->tc_bn[spin];
  const int stages = bn <= 64 ? 4 : bn <= 128 ? 3 : 2;
  const size_t smem = tc_smem_bytes(bn, stages);
  CUtensorMap ma, ml;
  tc_map(&ma, a_hi, c->tc_kpad, rows, TC_BM);
  tc_map(&ml, a_lo, c->tc_kpad, rows, TC_BM);
  TcGemmArgs g{rows, c->tc_kpad / TC_BK, c->H.nmo[spin], bn, ldd, stages, D, c->d_tc_err.as<int>()};
  CK(cudaFuncSetAttribute(k_mo_gemm_tf32x3, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  k_mo_gemm_tf32x3<<<(rows + TC_BM - 1) / TC_BM, TC_THREADS, smem, c->stream>>>(ma, ml, c->tc_map_b[spin][0],
                                                                               c->tc_map_b[spin][1], g);
  CK(cudaGetLastError());
  c->launches++;
}

static int fail(qwg_ctx* c, int code, const std::string& m) {
  if (c) c->err = m;
  return code;
}

// After a synchronised block: a tensor-core pipeline wait that expired
// (bounded waits in the GEMM kernel) becomes a CUDA-class error.
static int tc_check(qwg_ctx* c) {
  if (!c->tc_moves) return QWG_OK;
  int err = 0;
  CK(cudaMemcpyAsync(&err, c->d_tc_err.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
  CK(cudaStreamSynchronize(c->stream));
  if (!err) return QWG_OK;
  return fail(c, QWG_ERR_CUDA, "tensor-core MO contraction: a pipeline wait expired (code " + std::to_string(err) + ")");
}

template <class F>
static int guarded(qwg_ctx* c, F&& f) {
  try {
    return f();
  } catch (const InputError& e) {
    return fail(c, QWG_ERR_INPUT, e.what());
  } catch (const CudaError& e) {
    return fail(c, QWG_ERR_CUDA, e.what());
  } catch (const std::exception& e) {
    return fail(c, QWG_ERR_ARG, e.what());
  }
}

static void ensure_io(qwg_ctx* c, size_t bytes) {
  if (c->io_bytes < bytes) {
    c->d_io.alloc(bytes);
    c->io_bytes = bytes;
  }
}

// One chunk of steps on the resident population (plus DMC branching).
// Candidate and target buffers of the T-moves for nw walkers.
static int tmove_cap(const qwg_ctx* c) { return c->L.wchunk * c->H.natoms * QWG_MAXQ; }
static void ensure_tmove_buffers(qwg_ctx* c, int nw) {
  const size_t cand = (size_t)nw * tmove_cap(c) * 8, mv = (size_t)nw * c->H.nelec * 4 * 8;
  if (c->d_tm_cand.n < cand) c->d_tm_cand.alloc(cand);
  if (c->d_tm_moves.n < mv) c->d_tm_moves.alloc(mv);
}
static void set_tmoves(qwg_ctx* c, StepParams& P) {
  P.tmoves = c->dmc.tmoves;
  if (!P.tmoves) return;
  P.tm_cap = tmove_cap(c);
  P.tm_cand = c->d_tm_cand.as<double>();
  P.tm_moves = c->d_tm_moves.as<double>();
}

// P.nsteps steps of every walker: one fused launch, or (split schedule) a
// move launch and a local-energy launch per step.
static void launch_steps(qwg_ctx* c, StepParams P, const EvalIO& io, int nwalk) {
  // VMC with delayed rejection runs on the fused step kernel, which alone
  // carries the second-stage move (the DMC move kernel keeps depth 1)
  if (!c->split || (!P.dmc && P.vmc_depth > 1)) {
    launch_walkers(c, P, io, KM_STEPS, nwalk);
    return;
  }
  // the per-electron GEMM fills the GPU only with enough walkers (5 rows
  // each, 128-row tiles): below kTcMinWalkers the one-launch sweep is faster
  const bool tc = P.tc_ahi && P.tc_D && nwalk <= c->max_walkers && nwalk >= kTcMinWalkers;
  for (int st = 0; st < P.nsteps; st++) {
    P.st = st;
    if (tc) {
      // per electron: proposals + basis rows, one tensor-core GEMM over all
      // walkers' rows, decisions + Sherman-Morrison updates
      for (int e = 0; e < c->H.nelec; e++) {
        P.tc_e = e;
        P.tc_phase = 1;
        launch_walkers(c, P, io, KM_SWEEP, nwalk);
        tc_gemm(c, P.tc_ahi, P.tc_alo, nwalk * 5, e < c->H.nup ? 0 : 1, (float*)P.tc_D, P.tc_ldd);
        P.tc_phase = 2;
        launch_walkers(c, P, io, KM_SWEEP, nwalk);
      }
      P.tc_phase = 0;
    } else {
      launch_walkers(c, P, io, KM_SWEEP, nwalk);
    }
    launch_walkers(c, P, io, P.tmoves ? KM_ELOC_TM : KM_ELOC, nwalk);
    if (P.tmoves) launch_walkers(c, P, io, KM_TMOVE, nwalk);
  }
}

static void run_chunk(qwg_ctx* c, int nsteps, double tau, uint64_t seed, int det_pp, bool dmc, BlockAcc* acc,
                      double* energy_out) {
  StepParams P = base_params(c);
  P.nsteps = nsteps;
  P.tau = tau;
  P.dmc = dmc ? 1 : 0;
  P.deterministic_pp = det_pp;
  P.seed = seed;
  P.step0 = c->step_counter;
  P.acc = acc;
  P.branch_start = c->branch_start;
  P.branch_stop = c->branch_stop;
  P.max_weight = dmc ? c->dmc.max_poss_weight : 1.0;
  // full recompute (FP64 re-inversion) when the resident state is stale or
  // refresh_interval steps have passed since the last one
  int refresh_every = std::max(1, dmc ? c->dmc.refresh_interval : nsteps);
  P.refresh = (!c->state_valid || c->step_counter - c->last_refresh >= (uint64_t)refresh_every) ? 1 : 0;
  if (P.refresh) c->last_refresh = c->step_counter;
  EvalIO io{};
  io.energy = energy_out;
  launch_steps(c, P, io, c->nwalk);
  c->state_valid = true;
  c->have_scalars = true;
  c->step_counter += nsteps;
}

static void run_branch(qwg_ctx* c, const BlockAcc* acc, int nsteps) {
  BranchParams B{};
  B.nwalk = c->nwalk;
  int p2 = 1;
  while (p2 < c->nwalk) p2 <<= 1;
  B.npow2 = p2;
  B.nsteps = nsteps;
  B.feedback = c->dmc.feedback;
  B.timestep = c->dmc.timestep;
  B.seed = c->dmc.seed ^ 0x5bd1e995ull;
  B.state = c->d_state.as<unsigned char>();
  B.state_bytes = c->L.state_bytes;
  B.scal_off = c->L.scal;
  B.acc = acc;
  B.dyn = c->d_dyn.as<double>();
  B.src_of = c->d_src.as<int>();
  B.new_w = c->d_neww.as<double>();
  size_t sm = c->branch_device_wide ? 0 : branch_smem(c->nwalk);
  if (sm == 0) {
    // large population: the device-wide sort (8 stable 8-bit passes), the
    // pairing over all CTAs and a one-CTA gather map
    BranchBig G{};
    branch_big_bytes(c->nwalk, &G, c->d_branch.as<unsigned char>());
    const int W = c->nwalk;
    k_branch_prep<<<G.nprep, 256, 0, c->stream>>>(B, G);
    for (int pass = 0; pass < 8; pass++) {
      const int a = pass & 1;
      k_radix_hist<<<G.ntiles, 256, 0, c->stream>>>(G.key[a], W, 8 * pass, G.hist, G.ntiles);
      k_radix_scan<<<1, 1024, 0, c->stream>>>(G.hist, 256 * G.ntiles);
      k_radix_scatter<<<G.ntiles, 256, 0, c->stream>>>(G.key[a], G.idx[a], G.key[1 - a], G.idx[1 - a], W, 8 * pass,
                                                        G.hist, G.ntiles);
    }
    k_branch_pairs<<<G.npairblk, 256, 0, c->stream>>>(B, G, 0);
    k_branch_finish<<<1, 1024, 0, c->stream>>>(B, G);
    CK(cudaGetLastError());
    c->launches += 2 + 3 * 8 + 1;
  } else {
    ensure_smem_attr(k_branch, sm);
    k_branch<<<1, 1024, sm, c->stream>>>(B);
    CK(cudaGetLastError());
  }
  const int n3 = 3 * c->H.nelec;
  k_gather<<<c->nwalk, 128, 0, c->stream>>>(c->nwalk, n3, c->L.state_bytes, c->L.scal, c->d_src.as<int>(),
                                            c->d_neww.as<double>(), c->d_R.as<double>(),
                                            c->d_state.as<unsigned char>(), c->d_R2.as<double>(),
                                            c->d_state2.as<unsigned char>());
  CK(cudaGetLastError());
  c->launches += 2;
  // back into the primary buffers (keeps the buffers fixed for graph replay)
  CK(cudaMemcpyAsync(c->d_R.p, c->d_R2.p, (size_t)c->nwalk * n3 * 8, cudaMemcpyDeviceToDevice, c->stream));
  CK(cudaMemcpyAsync(c->d_state.p, c->d_state2.p, (size_t)c->nwalk * c->L.state_bytes, cudaMemcpyDeviceToDevice,
                     c->stream));
}

// One DMC block on the stream, entirely device-driven: per feedback interval
// the step kernel (step counter and refresh from dyn[]), then branching and
// the population gather; at the end the block statistics and E_ref/E_T
// update, and the statistics copied to pinned host memory.
static void enqueue_dmc_block(qwg_ctx* c) {
  const int nstep = c->dmc.nstep, fi = c->dmc.feedback_interval;
  const int nchunk = (nstep + fi - 1) / fi;
  BlockAcc* acc = c->d_acc.as<BlockAcc>();
  CK(cudaMemsetAsync(acc, 0, sizeof(BlockAcc) * nchunk, c->stream));
  for (int ch = 0, step = 0; ch < nchunk; ch++) {
    const int np = std::min(fi, nstep - step);
    StepParams P = base_params(c);
    P.nsteps = np;
    P.tau = c->dmc.timestep;
    P.dmc = 1;
    P.dyn_step = 1;
    P.refresh = 2;
    P.refresh_every = std::max(1, c->dmc.refresh_interval);
    P.deterministic_pp = c->dmc.deterministic_pp;
    P.seed = c->dmc.seed;
    P.acc = acc + ch;
    P.branch_start = c->branch_start;
    P.branch_stop = c->branch_stop;
    P.max_weight = c->dmc.max_poss_weight;
    set_tmoves(c, P);
    EvalIO io{};
    launch_steps(c, P, io, c->nwalk);
    run_branch(c, acc + ch, np);
    step += np;
  }
  k_block_end<<<1, 32, 0, c->stream>>>(acc, nchunk, c->d_dyn.as<double>(), c->d_hist.as<double>(), kHistCap,
                                       c->dmc.feedback, c->nwalk, c->d_stats.as<double>());
  CK(cudaGetLastError());
  c->launches++;
  CK(cudaMemcpyAsync(c->h_stats, c->d_stats.p, kStatsLen * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
}

// Block statistics from the BlockAcc sums t[0..QWG_NACC-1]: weighted averages
// as Properties_manager::endBlock (Properties.cpp:578-640), and the point
// variances of its log entry: (mean x^2 - mean^2) n / (n - 1) over the
// block's walker-steps, unweighted (condense_variance, :574-577).
static void stats_from_sums(const double* t, qwg_block_stats* s) {
  memset(s, 0, sizeof(*s));
  double W = t[0] > 0 ? t[0] : 1.0;
  s->energy = t[1] / W;
  s->kinetic = t[2] / W;
  s->potential = t[3] / W;
  s->nonlocal = t[4] / W;
  s->energy_var = t[5] / W - s->energy * s->energy;
  s->weight = t[9] > 0 ? t[0] / t[9] : 0.0;
  s->acceptance = t[7] > 0 ? t[6] / t[7] : 0.0;
  s->nonfinite = (int)t[8];
  s->npoints = t[9];
  const double n = t[9];
  auto pvar = [&](double sx, double sx2) {
    if (n < 2) return 0.0;
    const double m = sx / n;
    return (sx2 / n - m * m) * (n / (n - 1.0));
  };
  s->var_energy = pvar(t[10], t[11]);
  s->var_kinetic = pvar(t[12], t[13]);
  s->var_potential = pvar(t[14], t[15]);
  s->var_nonlocal = pvar(t[16], t[17]);
  s->var_weight = pvar(t[18], t[19]);
  s->etrial = t[QWG_NACC];
}

static void acc_to_stats(const std::vector<BlockAcc>& v, qwg_block_stats* s) {
  double t[QWG_NACC + 2] = {0};
  for (auto& a : v) {
    const double* p = (const double*)&a;
    for (int k = 0; k < QWG_NACC; k++) t[k] += p[k];
  }
  stats_from_sums(t, s);
}

}  // namespace

// ===========================================================================
// C-ABI

extern "C" {

const char* qwg_version(void) { return "mainline_b200 qwg 0.1 (sm_100a)"; }

// Error text of the last failed qwg_create on this thread (context is NULL then).
static thread_local std::string g_create_error;

const char* qwg_last_error(const qwg_ctx* ctx) { return ctx ? ctx->err.c_str() : g_create_error.c_str(); }

int qwg_inspect_deck(const char* deck_path, qwg_info* info, char* err, int errlen) {
  try {
    HostSystem H = build_system(deck_path);
    if (info) {
      memset(info, 0, sizeof(*info));
      info->nelec = H.nelec; info->nup = H.nup; info->ndown = H.ndn; info->natoms = H.natoms;
      info->nbasis = H.nbasis; info->nshell = (int)H.shells.size(); info->nmo_up = H.nmo[0];
      info->nmo_down = H.nmo[1]; info->has_pseudo = H.has_pp; info->ion_ion = H.ion_ion;
      info->complex_orbitals = needs_complex(H) ? 1 : 0;
    }
    return QWG_OK;
  } catch (const std::exception& e) {
    if (err && errlen > 0) { strncpy(err, e.what(), errlen - 1); err[errlen - 1] = 0; }
    return QWG_ERR_INPUT;
  }
}

int qwg_footprint(const char* deck_path, int precision, int max_walkers, unsigned long long* bytes) {
  if (!deck_path || !bytes || max_walkers <= 0) return QWG_ERR_ARG;
  if (precision != QWG_FP64 && precision != QWG_MIXED) return QWG_ERR_ARG;
  try {
    std::unique_ptr<qwg_ctx> c(new qwg_ctx());
    c->precision = precision;
    c->H = build_system(deck_path);
    if (mmax_for(std::max(c->H.nmo[0], c->H.nmo[1])) < 0) return QWG_ERR_INPUT;
    c->mmax = kernel_family(c->H);
    make_layout(c.get());
    *bytes = footprint_bytes(c.get(), max_walkers);
    return QWG_OK;
  } catch (const std::exception&) {
    return QWG_ERR_INPUT;
  }
}

int qwg_inspect_spline(const char* deck_path, int shell, double* coef, int maxpts, int* npts, double* spacing,
                       double* cutoff) {
  try {
    HostSystem H = build_system(deck_path);
    if (shell < 0 || shell >= (int)H.shells.size()) return QWG_ERR_ARG;
    const Shell& s = H.shells[shell];
    int n = std::min(maxpts, H.spline_npts);
    if (coef) memcpy(coef, H.spline_coef.data() + (size_t)s.spline * H.spline_npts * 4, sizeof(double) * 4 * n);
    if (npts) *npts = H.spline_npts;
    if (spacing) *spacing = H.spline_spacing;
    if (cutoff) *cutoff = s.cutoff;
    return QWG_OK;
  } catch (const std::exception&) {
    return QWG_ERR_INPUT;
  }
}

int qwg_create(const char* deck_path, int precision, int max_walkers, void* stream, qwg_ctx** out) {
  if (!out || !deck_path) return QWG_ERR_ARG;
  *out = nullptr;
  if (precision != QWG_FP64 && precision != QWG_MIXED) return QWG_ERR_ARG;
  if (max_walkers <= 0 || max_walkers > (1 << 22)) return QWG_ERR_ARG;
  std::unique_ptr<qwg_ctx> c(new qwg_ctx());
  c->precision = precision;
  c->max_walkers = max_walkers;
  int rc = guarded(c.get(), [&]() -> int {
    c->H = build_system(deck_path);
    if (mmax_for(std::max(c->H.nmo[0], c->H.nmo[1])) < 0)
      throw InputError("more than 256 electrons (or expansion orbitals) of one spin: beyond this engine build");
    if (c->H.detwt.size() > 1 && c->H.periodic)
      throw InputError("determinant expansions are supported for molecules only");
    c->mmax = kernel_family(c->H);
    if (const char* sched = getenv("QWG_DMC_SCHEDULE")) c->split = strcmp(sched, "fused") != 0;
    if (stream) {
      c->stream = (cudaStream_t)stream;
    } else {
      CK(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
      c->own_stream = true;
    }
    build_tables(c.get());
    make_layout(c.get());
    const int N = c->H.nelec;
    c->d_R.alloc((size_t)max_walkers * 3 * N * 8);
    c->d_R2.alloc((size_t)max_walkers * 3 * N * 8);
    c->d_state.alloc((size_t)max_walkers * c->L.state_bytes);
    c->d_state2.alloc((size_t)max_walkers * c->L.state_bytes);
    if (hbm_family(c->mmax)) c->d_scratch.alloc((size_t)max_walkers * c->L.scratch_bytes);
    if (const char* bw = std::getenv("QWG_BRANCH_DEVICE_WIDE")) c->branch_device_wide = bw[0] == '1';
#ifdef QWG_PHASES
    c->d_phases.alloc(PH_COUNT * sizeof(unsigned long long));
    CK(cudaMemsetAsync(c->d_phases.p, 0, PH_COUNT * sizeof(unsigned long long), c->stream));
#endif
    if (tc_moves_eligible(c.get())) {
      tc_setup(c.get());
      c->tc_ldd = std::max(c->tc_bn[0], c->tc_bn[1]);
      c->d_tc_a.alloc((size_t)max_walkers * 5 * c->tc_kpad * 2 * sizeof(float));
      c->d_tc_d.alloc((size_t)max_walkers * 5 * c->tc_ldd * sizeof(float));
      CK(cudaMemsetAsync(c->d_tc_err.p, 0, sizeof(int), c->stream));
      c->tc_moves = true;
    }
    c->d_acc.alloc(sizeof(BlockAcc) * 1024);
    c->d_dyn.alloc(DYN_COUNT * 8);
    CK(cudaMemsetAsync(c->d_dyn.p, 0, DYN_COUNT * 8, c->stream));
    c->d_src.alloc((size_t)max_walkers * 4);
    c->d_neww.alloc((size_t)max_walkers * 8);
    c->d_energy.alloc((size_t)max_walkers * 8);
    c->d_hist.alloc((size_t)kHistCap * 8);
    c->d_stats.alloc(kStatsLen * 8);
    CK(cudaMallocHost((void**)&c->h_stats, kStatsLen * sizeof(double)));
    CK(cudaEventCreate(&c->ev0));
    CK(cudaEventCreate(&c->ev1));
    CK(cudaStreamSynchronize(c->stream));
    return QWG_OK;
  });
  if (rc != QWG_OK) {
    g_create_error = c->err;
    return rc;
  }
  *out = c.release();
  return QWG_OK;
}

int qwg_destroy(qwg_ctx* ctx) {
  if (!ctx) return QWG_OK;
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->gexec) cudaGraphExecDestroy(ctx->gexec);
  if (ctx->graph) cudaGraphDestroy(ctx->graph);
  if (ctx->h_stats) cudaFreeHost(ctx->h_stats);
  if (ctx->ev0) cudaEventDestroy(ctx->ev0);
  if (ctx->ev1) cudaEventDestroy(ctx->ev1);
  cudaStream_t st = ctx->own_stream ? ctx->stream : nullptr;
  delete ctx;
  if (st) cudaStreamDestroy(st);
  return QWG_OK;
}

int qwg_get_info(const qwg_ctx* c, qwg_info* info) {
  if (!c || !info) return QWG_ERR_ARG;
  memset(info, 0, sizeof(*info));
  const HostSystem& H = c->H;
  info->nelec = H.nelec; info->nup = H.nup; info->ndown = H.ndn; info->natoms = H.natoms;
  info->nbasis = H.nbasis; info->nshell = (int)H.shells.size(); info->nmo_up = H.nmo[0]; info->nmo_down = H.nmo[1];
  info->has_pseudo = H.has_pp; info->max_walkers = c->max_walkers; info->precision = c->precision;
  info->walkers_per_cta = c->wpc; info->ion_ion = H.ion_ion;
  info->device_bytes = footprint_bytes(c, c->max_walkers);
  info->complex_orbitals = c->mmax == kComplexFamily ? 1 : 0;
  return QWG_OK;
}

int qwg_set_walkers(qwg_ctx* c, const double* R, int nw) {
  if (!c || !R || nw <= 0 || nw > c->max_walkers) return fail(c, QWG_ERR_ARG, "qwg_set_walkers: bad walker count");
  return guarded(c, [&]() -> int {
    const size_t bytes = (size_t)nw * 3 * c->H.nelec * 8;
    CK(cudaMemcpyAsync(c->d_R.p, R, bytes, cudaMemcpyHostToDevice, c->stream));
    c->nwalk = nw;
    c->state_valid = false;
    c->have_scalars = false;
    c->dmc_ready = false;
    return QWG_OK;
  });
}

int qwg_set_walkers_device(qwg_ctx* c, const double* dR, int nw) {
  if (!c || !dR || nw <= 0 || nw > c->max_walkers) return fail(c, QWG_ERR_ARG, "qwg_set_walkers_device: bad walker count");
  return guarded(c, [&]() -> int {
    CK(cudaMemcpyAsync(c->d_R.p, dR, (size_t)nw * 3 * c->H.nelec * 8, cudaMemcpyDeviceToDevice, c->stream));
    c->nwalk = nw;
    c->state_valid = false;
    c->have_scalars = false;
    c->dmc_ready = false;
    return QWG_OK;
  });
}

int qwg_get_walkers(qwg_ctx* c, double* R, int nw) {
  if (!c || !R || nw <= 0 || nw > c->nwalk) return fail(c, QWG_ERR_ARG, "qwg_get_walkers: bad walker count");
  return guarded(c, [&]() -> int {
    CK(cudaMemcpyAsync(R, c->d_R.p, (size_t)nw * 3 * c->H.nelec * 8, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    return QWG_OK;
  });
}

int qwg_get_walker_scalars(qwg_ctx* c, double* energy, double* weight, int nw) {
  if (!c || nw <= 0 || nw > c->nwalk) return fail(c, QWG_ERR_ARG, "qwg_get_walker_scalars: bad walker count");
  if (!c->have_scalars) return fail(c, QWG_ERR_STATE, "qwg_get_walker_scalars: no block has run on these walkers");
  return guarded(c, [&]() -> int {
    // one strided copy of (eold, weight) out of every walker's state
    std::vector<double> ew((size_t)nw * 2);
    const unsigned char* src = c->d_state.as<unsigned char>() + c->L.scal + offsetof(WScal, eold);
    static_assert(offsetof(WScal, weight) == offsetof(WScal, eold) + sizeof(double), "WScal layout");
    CK(cudaMemcpy2DAsync(ew.data(), 16, src, c->L.state_bytes, 16, nw, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (int w = 0; w < nw; w++) {
      if (energy) energy[w] = ew[2 * (size_t)w];
      if (weight) weight[w] = ew[2 * (size_t)w + 1];
    }
    return QWG_OK;
  });
}

int qwg_store_configs(qwg_ctx* c, const char* path, int dmc) {
  if (!c || !path) return QWG_ERR_ARG;
  if (c->nwalk <= 0) return fail(c, QWG_ERR_STATE, "qwg_store_configs: no walkers");
  if (dmc && !c->have_scalars) return fail(c, QWG_ERR_STATE, "qwg_store_configs: no DMC weights yet");
  return guarded(c, [&]() -> int {
    const int W = c->nwalk, N = c->H.nelec;
    std::vector<double> R((size_t)W * N * 3), wt, sg;
    CK(cudaMemcpyAsync(R.data(), c->d_R.p, R.size() * 8, cudaMemcpyDeviceToHost, c->stream));
    if (dmc) {
      // weight and both determinant signs out of every walker's scalars
      std::vector<WScal> sc(W);
      CK(cudaMemcpy2DAsync(sc.data(), sizeof(WScal), c->d_state.as<unsigned char>() + c->L.scal, c->L.state_bytes,
                           sizeof(WScal), W, cudaMemcpyDeviceToHost, c->stream));
      CK(cudaStreamSynchronize(c->stream));
      wt.resize(W);
      sg.resize(W);
      for (int w = 0; w < W; w++) {
        wt[w] = sc[w].weight;
        sg[w] = sc[w].sign[0] * sc[w].sign[1];
      }
    }
    CK(cudaStreamSynchronize(c->stream));
    const int rc = qwg_write_configs(path, R.data(), dmc ? wt.data() : nullptr, dmc ? sg.data() : nullptr, W, N);
    if (rc != QWG_OK) return fail(c, rc, std::string("qwg_store_configs: cannot write ") + path);
    return QWG_OK;
  });
}

int qwg_eval(qwg_ctx* c, const double* rot, qwg_eval_out* out) {
  if (!c || !out) return QWG_ERR_ARG;
  if (c->nwalk <= 0) return fail(c, QWG_ERR_STATE, "qwg_eval: no walkers");
  return guarded(c, [&]() -> int {
    const int W = c->nwalk, N = c->H.nelec;
    size_t n_rot = (size_t)W * 9, n_g = (size_t)W * N * 3, n_l = (size_t)W * N;
    size_t total = 8 * (n_rot + 5 * (size_t)W + n_g + n_l);
    ensure_io(c, total);
    double* base = c->d_io.as<double>();
    double* d_rot = base;
    double* d_lp = d_rot + n_rot;
    double* d_sg = d_lp + W;
    double* d_k = d_sg + W;
    double* d_v = d_k + W;
    double* d_nl = d_v + W;
    double* d_g = d_nl + W;
    double* d_l = d_g + n_g;
    if (rot) CK(cudaMemcpyAsync(d_rot, rot, 8 * n_rot, cudaMemcpyHostToDevice, c->stream));
    EvalIO io{};
    io.rot = rot ? d_rot : nullptr;
    io.logpsi = d_lp; io.sign = d_sg; io.kinetic = d_k; io.potential = d_v; io.nonlocal = d_nl;
    io.grad = d_g; io.lap = d_l;
    StepParams P = base_params(c);
    launch_walkers(c, P, io, KM_EVAL, W);
    auto dl = [&](double* h, const double* d, size_t n) {
      if (h) CK(cudaMemcpyAsync(h, d, 8 * n, cudaMemcpyDeviceToHost, c->stream));
    };
    dl(out->logpsi, d_lp, W); dl(out->sign, d_sg, W); dl(out->kinetic, d_k, W); dl(out->potential, d_v, W);
    dl(out->nonlocal, d_nl, W); dl(out->grad, d_g, n_g); dl(out->lap, d_l, n_l);
    CK(cudaStreamSynchronize(c->stream));
    c->state_valid = false;  // eval leaves scratch state unsaved
    return QWG_OK;
  });
}

int qwg_phase_counters(qwg_ctx* c, unsigned long long* out, int n, int reset) {
  if (!c || (n > 0 && !out)) return QWG_ERR_ARG;
  if (!c->d_phases.p) return fail(c, QWG_ERR_STATE, "qwg_phase_counters: this library was built without phase "
                                                    "counters (build libqwg_phases.so)");
  return guarded(c, [&]() -> int {
    CK(cudaStreamSynchronize(c->stream));
    const int m = std::min(n, (int)PH_COUNT);
    if (m > 0) CK(cudaMemcpy(out, c->d_phases.p, m * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    if (reset) CK(cudaMemset(c->d_phases.p, 0, PH_COUNT * sizeof(unsigned long long)));
    return QWG_OK;
  });
}

int qwg_mo_eval(qwg_ctx* c, const double* pos, int npos, int spin, double* out) {
  if (!c || !pos || !out || npos <= 0 || spin < 0 || spin > 1) return QWG_ERR_ARG;
  if (c->mmax == kComplexFamily) return fail(c, QWG_ERR_ARG, "qwg_mo_eval: complex orbitals are not supported");
  if ((size_t)npos * 5 > (size_t)INT32_MAX / 2) return fail(c, QWG_ERR_ARG, "qwg_mo_eval: too many positions");
  const int nmo = c->H.nmo[spin];
  if (nmo == 0) return QWG_OK;
  return guarded(c, [&]() -> int {
    const int nb = c->H.nbasis;
    const size_t n_out = (size_t)npos * nmo * 5;
    std::vector<double> host_out;
    if (c->precision == QWG_FP64) {
      const int ms = c->sys_d.mstride;
      const size_t bytes = 8 * ((size_t)npos * 3 + (size_t)npos * nb * 5 + (size_t)npos * ms * 5 + n_out);
      if (c->d_mo_scratch.n < bytes) c->d_mo_scratch.alloc(bytes);
      double* d_pos = c->d_mo_scratch.as<double>();
      double* bas = d_pos + (size_t)npos * 3;
      double* osc = bas + (size_t)npos * nb * 5;
      double* dout = osc + (size_t)npos * ms * 5;
      CK(cudaMemcpyAsync(d_pos, pos, 8 * (size_t)npos * 3, cudaMemcpyHostToDevice, c->stream));
      k_mo_rows_cuda<double><<<(npos + 3) / 4, 128, 0, c->stream>>>(
          c->sys_d, c->sys_d.moc + (size_t)spin * nb * ms, d_pos, npos, nmo, bas, osc, dout);
      CK(cudaGetLastError());
      c->launches++;
      CK(cudaMemcpyAsync(out, dout, 8 * n_out, cudaMemcpyDeviceToHost, c->stream));
      CK(cudaStreamSynchronize(c->stream));
      return QWG_OK;
    }
    tc_setup(c);
    const int kpad = c->tc_kpad, bn = c->tc_bn[spin];
    const size_t rows = (size_t)npos * 5;
    // doubles: positions, basis rows; floats (256-byte aligned): a_hi, a_lo, D
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t o_bas = al(8 * (size_t)npos * 3), o_ahi = o_bas + al(8 * (size_t)npos * nb * 5);
    const size_t o_alo = o_ahi + al(4 * rows * kpad), o_d = o_alo + al(4 * rows * kpad);
    const size_t bytes = o_d + al(4 * rows * bn);
    if (c->d_mo_scratch.n < bytes) c->d_mo_scratch.alloc(bytes);
    unsigned char* base = c->d_mo_scratch.as<unsigned char>();
    double* d_pos = (double*)base;
    float* a_hi = (float*)(base + o_ahi);
    float* a_lo = (float*)(base + o_alo);
    float* D = (float*)(base + o_d);
    CK(cudaMemcpyAsync(d_pos, pos, 8 * (size_t)npos * 3, cudaMemcpyHostToDevice, c->stream));
    k_basis_rows_tf32<float><<<(npos + 3) / 4, 128, 0, c->stream>>>(c->sys_f, d_pos, npos, kpad,
                                                                    (double*)(base + o_bas), a_hi, a_lo);
    CK(cudaGetLastError());
    c->launches++;
    CK(cudaMemsetAsync(c->d_tc_err.p, 0, sizeof(int), c->stream));
    tc_gemm(c, a_hi, a_lo, (int)rows, spin, D, bn);
    std::vector<float> hD(rows * bn);
    int err = 0;
    CK(cudaMemcpyAsync(hD.data(), D, 4 * rows * bn, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(&err, c->d_tc_err.p, sizeof(int), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (err) return fail(c, QWG_ERR_CUDA, "qwg_mo_eval: a tensor-core pipeline wait expired (code " +
                                              std::to_string(err) + ")");
    for (int p = 0; p < npos; p++)
      for (int j = 0; j < nmo; j++)
        for (int q = 0; q < 5; q++) out[((size_t)p * nmo + j) * 5 + q] = hD[((size_t)p * 5 + q) * bn + j];
    return QWG_OK;
  });
}

int qwg_ratio(qwg_ctx* c, const int* e, const double* Rnew, double* dlogpsi, double* sign, double* grad,
              double* lap) {
  if (!c || !e || !Rnew) return QWG_ERR_ARG;
  if (c->nwalk <= 0) return fail(c, QWG_ERR_STATE, "qwg_ratio: no walkers");
  for (int w = 0; w < c->nwalk; w++)
    if (e[w] < 0 || e[w] >= c->H.nelec) return fail(c, QWG_ERR_ARG, "qwg_ratio: electron index out of range");
  return guarded(c, [&]() -> int {
    const int W = c->nwalk;
    size_t total = 8 * ((size_t)W * 3 + (size_t)W * 3 + 3 * (size_t)W) + 4 * (size_t)W + 64;
    ensure_io(c, total);
    double* d_r = c->d_io.as<double>();
    double* d_lp = d_r + 3 * W;
    double* d_sg = d_lp + W;
    double* d_g = d_sg + W;
    double* d_l = d_g + 3 * W;
    int* d_e = (int*)(d_l + W);
    CK(cudaMemcpyAsync(d_r, Rnew, 8 * 3 * (size_t)W, cudaMemcpyHostToDevice, c->stream));
    CK(cudaMemcpyAsync(d_e, e, 4 * (size_t)W, cudaMemcpyHostToDevice, c->stream));
    EvalIO io{};
    io.move_e = d_e; io.move_r = d_r; io.logpsi = d_lp; io.sign = d_sg; io.grad = d_g; io.lap = d_l;
    StepParams P = base_params(c);
    launch_walkers(c, P, io, KM_RATIO, W);
    if (dlogpsi) CK(cudaMemcpyAsync(dlogpsi, d_lp, 8 * (size_t)W, cudaMemcpyDeviceToHost, c->stream));
    if (sign) CK(cudaMemcpyAsync(sign, d_sg, 8 * (size_t)W, cudaMemcpyDeviceToHost, c->stream));
    if (grad) CK(cudaMemcpyAsync(grad, d_g, 8 * 3 * (size_t)W, cudaMemcpyDeviceToHost, c->stream));
    if (lap) CK(cudaMemcpyAsync(lap, d_l, 8 * (size_t)W, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->state_valid = false;
    return QWG_OK;
  });
}

int qwg_set_vmc_dynamics(qwg_ctx* c, int depth, double divider) {
  if (!c || depth < 1 || depth > 2 || !(divider > 0))
    return fail(c, QWG_ERR_ARG, "qwg_set_vmc_dynamics: depth must be 1 or 2 and divider positive");
  c->vmc_depth = depth;
  c->vmc_divider = divider;
  return QWG_OK;
}

int qwg_vmc_block(qwg_ctx* c, int nstep, double timestep, uint64_t seed, int deterministic_pp,
                  qwg_block_stats* stats) {
  if (!c || nstep <= 0 || !(timestep > 0)) return fail(c, QWG_ERR_ARG, "qwg_vmc_block: bad arguments");
  if (c->nwalk <= 0) return fail(c, QWG_ERR_STATE, "qwg_vmc_block: no walkers");
  return guarded(c, [&]() -> int {
    BlockAcc* acc = c->d_acc.as<BlockAcc>();
    CK(cudaMemsetAsync(acc, 0, sizeof(BlockAcc), c->stream));
    CK(cudaEventRecord(c->ev0, c->stream));
    c->state_valid = false;  // VMC: full recompute at the start of each block
    run_chunk(c, nstep, timestep, seed, deterministic_pp, false, acc, nullptr);
    CK(cudaEventRecord(c->ev1, c->stream));
    std::vector<BlockAcc> h(1);
    CK(cudaMemcpyAsync(h.data(), acc, sizeof(BlockAcc), cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    if (int rc = tc_check(c)) return rc;
    if (stats) {
      memset(stats, 0, sizeof(*stats));
      acc_to_stats(h, stats);
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
      stats->block_ms = ms;
      stats->nsteps = nstep;
      stats->nwalkers = c->nwalk;
    }
    c->dmc_ready = false;
    return QWG_OK;
  });
}

int qwg_dmc_init(qwg_ctx* c, const qwg_dmc_params* p) {
  if (!c || !p || !(p->timestep > 0)) return fail(c, QWG_ERR_ARG, "qwg_dmc_init: bad parameters");
  if (c->nwalk <= 0) return fail(c, QWG_ERR_STATE, "qwg_dmc_init: no walkers");
  return guarded(c, [&]() -> int {
    c->dmc = *p;
    if (c->dmc.nstep <= 0) c->dmc.nstep = std::max(int(1.0 / p->timestep + 0.5), 1);
    if (c->dmc.feedback_interval <= 0) c->dmc.feedback_interval = 5;
    if (c->dmc.max_poss_weight <= 0) c->dmc.max_poss_weight = 7.0;
    if (c->dmc.branch_start_cutoff <= 0) c->dmc.branch_start_cutoff = 10.0;
    if (c->dmc.refresh_interval <= 0)
      c->dmc.refresh_interval = c->precision == QWG_FP64 ? c->dmc.feedback_interval : 32;
    if (c->dmc.tmoves < 0 || c->dmc.tmoves > 2) throw InputError("tmoves must be 0, 1 or 2");
    if (c->dmc.tmoves && !c->H.has_pp) throw InputError("T-moves need a pseudopotential");
    if (c->dmc.tmoves && !c->split) throw InputError("T-moves need the split step schedule");
    if (c->dmc.tmoves) ensure_tmove_buffers(c, c->nwalk);
    const int W = c->nwalk;
    const int nchunk = (c->dmc.nstep + c->dmc.feedback_interval - 1) / c->dmc.feedback_interval;
    if (nchunk > 1024) throw std::runtime_error("too many feedback intervals per block");
    if (c->graph) { cudaGraphDestroy(c->graph); c->graph = nullptr; }
    if (c->gexec) { cudaGraphExecDestroy(c->gexec); c->gexec = nullptr; }
    // local energies of the starting walkers (gatherData for every walker in
    // Dmc_method::restorecheckpoint; deterministic PP for a clean start)
    size_t n_g = (size_t)W * c->H.nelec * 3, n_l = (size_t)W * c->H.nelec;
    ensure_io(c, 8 * (5 * (size_t)W + n_g + n_l));
    double* base = c->d_io.as<double>();
    EvalIO io{};
    io.logpsi = base; io.sign = base + W; io.kinetic = base + 2 * W; io.potential = base + 3 * W;
    io.nonlocal = base + 4 * W; io.grad = base + 5 * W; io.lap = io.grad + n_g;
    StepParams P = base_params(c);
    launch_walkers(c, P, io, KM_EVAL, W);
    std::vector<double> k(W), v(W), nl(W), el(W), lp(W);
    CK(cudaMemcpyAsync(k.data(), io.kinetic, 8 * W, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(v.data(), io.potential, 8 * W, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(nl.data(), io.nonlocal, 8 * W, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaMemcpyAsync(lp.data(), io.logpsi, 8 * W, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    double sum = 0;
    int good = 0;
    for (int w = 0; w < W; w++) {
      el[w] = k[w] + v[w] + nl[w];
      // a zero determinant (log|D| = -1e201, the exact zero of the inversion)
      // leaves no usable local energy
      if (!(lp[w] > -1e200)) el[w] = NAN;
      if (std::isfinite(el[w])) { sum += el[w]; good++; }
    }
    if (!good)
      return fail(c, QWG_ERR_NUMERIC,
                  "qwg_dmc_init: no walker has a finite local energy (non-finite values or a zero determinant)");
    // find_cutoffs (Dmc_method.cpp:262-300)
    double eavg = sum / good, var = 0;
    for (int w = 0; w < W; w++)
      if (std::isfinite(el[w])) var += (el[w] - eavg) * (el[w] - eavg);
      else el[w] = eavg;
    var /= W;
    double sigma = std::sqrt(var);
    c->eref = eavg;
    c->branch_start = c->dmc.branch_start_cutoff * sigma;
    c->branch_stop = c->branch_start * 1.5;
    CK(cudaMemcpyAsync(c->d_energy.p, el.data(), 8 * W, cudaMemcpyHostToDevice, c->stream));
    // resident state: one zero-step launch builds it; weights 1, E_old = E_L
    StepParams P2 = base_params(c);
    P2.nsteps = 0;
    P2.refresh = 1;
    P2.acc = c->d_acc.as<BlockAcc>();
    EvalIO io2{};
    launch_walkers(c, P2, io2, KM_STEPS, W);
    k_init_weights<<<(W + 255) / 256, 256, 0, c->stream>>>(c->d_state.as<unsigned char>(), W, c->L.state_bytes,
                                                           c->L.scal, c->d_energy.as<double>());
    CK(cudaGetLastError());
    c->launches++;
    c->have_scalars = true;
    // device scalars: E_T = E_ref (start_feedback * log 1), counters
    double dyn0[DYN_COUNT] = {0};
    dyn0[DYN_ETRIAL] = c->eref;
    dyn0[DYN_TEFF] = c->dmc.timestep;
    dyn0[DYN_SUMW] = double(W);
    dyn0[DYN_EREF] = c->eref;
    dyn0[DYN_STEP] = double(c->step_counter);
    dyn0[DYN_BRANCH] = double(c->branch_counter);
    CK(cudaMemcpyAsync(c->d_dyn.p, dyn0, sizeof(dyn0), cudaMemcpyHostToDevice, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    c->state_valid = true;
    // capture one block as a CUDA graph (every kernel in it has been
    // launched before, so no attribute changes happen during the capture)
    {
      BlockAcc* acc = c->d_acc.as<BlockAcc>();
      StepParams Pw = base_params(c);
      Pw.nsteps = 0; Pw.refresh = 0; Pw.acc = acc;
      EvalIO iw{};
      launch_walkers(c, Pw, iw, KM_STEPS, W);  // same kernel variant as the block's chunks
      launch_walkers(c, Pw, iw, KM_SWEEP, 0);  // shared-memory attributes of the split kernels
      launch_walkers(c, Pw, iw, KM_ELOC, 0);
      launch_walkers(c, Pw, iw, KM_ELOC_TM, 0);
      launch_walkers(c, Pw, iw, KM_TMOVE, 0);
      CK(cudaStreamSynchronize(c->stream));
    }
    if (W > kMaxDmcWalkers) throw InputError("DMC populations above 262144 walkers are beyond this engine build");
    if (branch_smem(W) && !c->branch_device_wide) {
      ensure_smem_attr(k_branch, branch_smem(W));
    } else if (c->d_branch.n < branch_big_bytes(W, nullptr, nullptr)) {
      c->d_branch.alloc(branch_big_bytes(W, nullptr, nullptr));
    }
    const long long l0 = c->launches;
    CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal));
    try {
      enqueue_dmc_block(c);
    } catch (...) {
      cudaGraph_t g = nullptr;
      cudaStreamEndCapture(c->stream, &g);
      if (g) cudaGraphDestroy(g);
      throw;
    }
    CK(cudaStreamEndCapture(c->stream, &c->graph));
    CK(cudaGraphInstantiate(&c->gexec, c->graph, 0));
    c->launches_per_block = c->launches - l0;
    c->launches = l0;
    c->dmc_ready = true;
    c->block_pending = false;
    return QWG_OK;
  });
}

int qwg_dmc_block_async(qwg_ctx* c) {
  if (!c) return QWG_ERR_ARG;
  if (!c->dmc_ready) return fail(c, QWG_ERR_STATE, "qwg_dmc_block_async: call qwg_dmc_init first");
  if (c->block_pending) return fail(c, QWG_ERR_STATE, "qwg_dmc_block_async: previous block not collected");
  return guarded(c, [&]() -> int {
    CK(cudaEventRecord(c->ev0, c->stream));
    CK(cudaGraphLaunch(c->gexec, c->stream));
    CK(cudaEventRecord(c->ev1, c->stream));
    c->launches += c->launches_per_block;
    c->block_pending = true;
    return QWG_OK;
  });
}

int qwg_dmc_block_wait(qwg_ctx* c, qwg_block_stats* stats) {
  if (!c) return QWG_ERR_ARG;
  if (!c->block_pending) return fail(c, QWG_ERR_STATE, "qwg_dmc_block_wait: no block in flight");
  return guarded(c, [&]() -> int {
    CK(cudaEventSynchronize(c->ev1));
    c->block_pending = false;
    c->step_counter += c->dmc.nstep;
    if (int rc = tc_check(c)) return rc;
    if (stats) {
      stats_from_sums(c->h_stats, stats);
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
      stats->block_ms = ms;
      stats->nsteps = c->dmc.nstep;
      stats->nwalkers = c->nwalk;
    }
    return QWG_OK;
  });
}

int qwg_dmc_block_ready(qwg_ctx* c) {
  if (!c) return QWG_ERR_ARG;
  if (!c->block_pending) return fail(c, QWG_ERR_STATE, "qwg_dmc_block_ready: no block in flight");
  cudaError_t e = cudaEventQuery(c->ev1);
  if (e == cudaSuccess) return 1;
  if (e == cudaErrorNotReady) return 0;
  return fail(c, QWG_ERR_CUDA, std::string("qwg_dmc_block_ready: ") + cudaGetErrorString(e));
}

int qwg_dmc_block(qwg_ctx* c, qwg_block_stats* stats) {
  int rc = qwg_dmc_block_async(c);
  if (rc != QWG_OK) return rc;
  return qwg_dmc_block_wait(c, stats);
}

// ---------------------------------------------------------------------------
// Allocation-free VMC block: the walker state and the accumulators live in one
// file-scope device array instead of the context's buffers.  In host code
// g_noalloc_scratch names a host-side stand-in, not a device address; the
// device address is looked up once per device and passed to the kernel.

static __device__ __align__(256) unsigned char g_noalloc_scratch[QWG_NOALLOC_SCRATCH_BYTES];

namespace {
constexpr int kNoallocMaxDevices = 64;
std::mutex g_noalloc_mu;
void* g_noalloc_ptr[kNoallocMaxDevices] = {};

// Device address of the scratch array on the current device (first call per
// device does the lookup).
void* noalloc_scratch_device_ptr(std::string& err) {
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kNoallocMaxDevices) {
    err = std::string("qwg_vmc_block_noalloc: no usable current device: ") + cudaGetErrorString(e);
    return nullptr;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (!g_noalloc_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      err = std::string("qwg_vmc_block_noalloc: cudaGetSymbolAddress failed: ") + cudaGetErrorString(e);
      return nullptr;
    }
    g_noalloc_ptr[dev] = p;
  }
  return g_noalloc_ptr[dev];
}
}  // namespace

int qwg_vmc_block_noalloc(qwg_ctx* c, double* d_R, int nw, int nstep, double timestep, uint64_t seed,
                          int deterministic_pp, double* d_energy, double* d_sums) {
  if (!c) return QWG_ERR_ARG;
  if (!d_R || !d_sums || nw <= 0 || nstep <= 0 || !(timestep > 0))
    return fail(c, QWG_ERR_ARG, "qwg_vmc_block_noalloc: bad arguments");
  const size_t acc_bytes = 256;  // BlockAcc at the start, walker state after it
  static_assert(sizeof(BlockAcc) <= 256, "accumulator block exceeds its scratch slot");
  // HBM-resident walkers (more than 32 orbitals per spin) also need their
  // scratch region in the fixed buffer, after the walker states
  const size_t per = (size_t)c->L.state_bytes + (hbm_family(c->mmax) ? (size_t)c->L.scratch_bytes : 0);
  const size_t need = acc_bytes + (size_t)nw * per;
  if (need > QWG_NOALLOC_SCRATCH_BYTES) {
    const size_t maxw = (QWG_NOALLOC_SCRATCH_BYTES - acc_bytes) / per;
    return fail(c, QWG_ERR_ARG, "qwg_vmc_block_noalloc: " + std::to_string(nw) + " walkers need " +
                                    std::to_string(need) + " bytes of scratch; the fixed scratch holds " +
                                    std::to_string(QWG_NOALLOC_SCRATCH_BYTES) + " bytes (at most " +
                                    std::to_string(maxw) + " walkers of this system)");
  }
  std::string err;
  unsigned char* base = (unsigned char*)noalloc_scratch_device_ptr(err);
  if (!base) return fail(c, QWG_ERR_CUDA, err);
  return guarded(c, [&]() -> int {
    BlockAcc* acc = (BlockAcc*)base;
    CK(cudaMemsetAsync(acc, 0, sizeof(BlockAcc), c->stream));
    StepParams P{};
    P.nwalk = nw;
    P.nsteps = nstep;
    P.refresh = 1;
    P.dmc = 0;
    P.vmc_depth = c->vmc_depth;
    P.vmc_divider = c->vmc_divider;
    P.deterministic_pp = deterministic_pp;
    P.tau = timestep;
    P.seed = seed;
    P.step0 = c->noalloc_step_counter;
    P.max_weight = 1.0;
    P.R = d_R;
    P.state = base + acc_bytes;
    P.scratch = hbm_family(c->mmax) ? base + acc_bytes + (size_t)nw * c->L.state_bytes : nullptr;
    P.acc = acc;
    P.etrial = c->d_dyn.as<double>();
    EvalIO io{};
    io.energy = d_energy;
    launch_steps(c, P, io, nw);
    CK(cudaMemcpyAsync(d_sums, acc, 10 * sizeof(double), cudaMemcpyDeviceToDevice, c->stream));
    c->noalloc_step_counter += nstep;
    return QWG_OK;
  });
}

// ---------------------------------------------------------------------------
// batched systems: one graph, one block of every context

}  // extern "C"

struct qwg_batch {
  std::vector<qwg_ctx*> ctxs;
  cudaStream_t origin = nullptr;
  std::vector<cudaEvent_t> events;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  std::string err;
};

extern "C" {

int qwg_batch_create(qwg_ctx* const* ctxs, int n, qwg_batch** out) {
  if (!ctxs || n <= 0 || !out) return QWG_ERR_ARG;
  *out = nullptr;
  std::unique_ptr<qwg_batch> b(new qwg_batch());
  for (int i = 0; i < n; i++) {
    if (!ctxs[i] || !ctxs[i]->dmc_ready) {
      g_create_error = "qwg_batch_create: context " + std::to_string(i) + " has no qwg_dmc_init";
      return QWG_ERR_STATE;
    }
    b->ctxs.push_back(ctxs[i]);
  }
  try {
    CK(cudaStreamCreateWithFlags(&b->origin, cudaStreamNonBlocking));
    CK(cudaEventCreate(&b->ev0));
    CK(cudaEventCreate(&b->ev1));
    b->events.resize(n + 1);
    for (auto& e : b->events) CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (auto* c : b->ctxs) CK(cudaStreamSynchronize(c->stream));
    CK(cudaStreamBeginCapture(b->origin, cudaStreamCaptureModeThreadLocal));
    CK(cudaEventRecord(b->events[n], b->origin));
    for (int i = 0; i < n; i++) {
      qwg_ctx* c = b->ctxs[i];
      CK(cudaStreamWaitEvent(c->stream, b->events[n], 0));  // fork
      enqueue_dmc_block(c);
      CK(cudaEventRecord(b->events[i], c->stream));
      CK(cudaStreamWaitEvent(b->origin, b->events[i], 0));   // join
    }
    CK(cudaStreamEndCapture(b->origin, &b->graph));
    CK(cudaGraphInstantiate(&b->gexec, b->graph, 0));
  } catch (const std::exception& e) {
    g_create_error = std::string("qwg_batch_create: ") + e.what();
    cudaGraph_t g = nullptr;
    if (b->origin) {
      cudaStreamCaptureStatus st;
      if (cudaStreamIsCapturing(b->origin, &st) == cudaSuccess && st != cudaStreamCaptureStatusNone)
        cudaStreamEndCapture(b->origin, &g);
    }
    if (g) cudaGraphDestroy(g);
    qwg_batch_destroy(b.release());
    return QWG_ERR_CUDA;
  }
  for (auto* c : b->ctxs) c->launches -= c->launches_per_block;  // counted at capture
  *out = b.release();
  return QWG_OK;
}

int qwg_batch_block(qwg_batch* b, qwg_block_stats* stats) {
  if (!b) return QWG_ERR_ARG;
  for (auto* c : b->ctxs)
    if (c->block_pending) { b->err = "qwg_batch_block: a context has a block in flight"; return QWG_ERR_STATE; }
  try {
    CK(cudaEventRecord(b->ev0, b->origin));
    CK(cudaGraphLaunch(b->gexec, b->origin));
    CK(cudaEventRecord(b->ev1, b->origin));
    CK(cudaEventSynchronize(b->ev1));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    for (size_t i = 0; i < b->ctxs.size(); i++) {
      qwg_ctx* c = b->ctxs[i];
      c->launches += c->launches_per_block;
      c->step_counter += c->dmc.nstep;
      if (stats) {
        stats_from_sums(c->h_stats, &stats[i]);
        stats[i].block_ms = ms;
        stats[i].nsteps = c->dmc.nstep;
        stats[i].nwalkers = c->nwalk;
      }
    }
  } catch (const std::exception& e) {
    b->err = e.what();
    return QWG_ERR_CUDA;
  }
  return QWG_OK;
}

int qwg_batch_destroy(qwg_batch* b) {
  if (!b) return QWG_OK;
  if (b->origin) cudaStreamSynchronize(b->origin);
  if (b->gexec) cudaGraphExecDestroy(b->gexec);
  if (b->graph) cudaGraphDestroy(b->graph);
  for (auto e : b->events)
    if (e) cudaEventDestroy(e);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  if (b->origin) cudaStreamDestroy(b->origin);
  delete b;
  return QWG_OK;
}

int qwg_tmove_select(qwg_ctx* c, const double* rot, int mode, double tau, uint64_t seed, int* moved, double* pos) {
  if (!c || !moved || !pos || (mode != 1 && mode != 2) || !(tau > 0)) return QWG_ERR_ARG;
  if (c->nwalk <= 0) return fail(c, QWG_ERR_STATE, "qwg_tmove_select: no walkers");
  if (!c->H.has_pp) return fail(c, QWG_ERR_INPUT, "qwg_tmove_select: the deck has no pseudopotential");
  return guarded(c, [&]() -> int {
    const int W = c->nwalk, N = c->H.nelec;
    ensure_tmove_buffers(c, W);
    const size_t n_rot = (size_t)W * 9, n_g = (size_t)W * N * 3, n_l = (size_t)W * N;
    ensure_io(c, 8 * (n_rot + 5 * (size_t)W + n_g + n_l));
    double* base = c->d_io.as<double>();
    EvalIO io{};
    io.logpsi = base; io.sign = base + W; io.kinetic = base + 2 * W; io.potential = base + 3 * W;
    io.nonlocal = base + 4 * W; io.grad = base + 5 * W; io.lap = io.grad + n_g;
    if (rot) {
      double* drot = io.lap + n_l;
      CK(cudaMemcpyAsync(drot, rot, 8 * n_rot, cudaMemcpyHostToDevice, c->stream));
      io.rot = drot;
    }
    StepParams P = base_params(c);
    P.tmoves = mode;
    P.tau = tau;
    P.seed = seed;
    P.tm_cap = tmove_cap(c);
    P.tm_cand = c->d_tm_cand.as<double>();
    P.tm_moves = c->d_tm_moves.as<double>();
    launch_walkers(c, P, io, KM_EVAL, W);
    std::vector<double> mv((size_t)W * N * 4);
    CK(cudaMemcpyAsync(mv.data(), P.tm_moves, mv.size() * 8, cudaMemcpyDeviceToHost, c->stream));
    CK(cudaStreamSynchronize(c->stream));
    for (size_t k = 0; k < (size_t)W * N; k++) {
      moved[k] = mv[4 * k + 3] != 0.0 ? 1 : 0;
      for (int d = 0; d < 3; d++) pos[3 * k + d] = mv[4 * k + d];
    }
    c->state_valid = false;  // the evaluation used the resident state slots as scratch
    return QWG_OK;
  });
}

int qwg_time_kernels(qwg_ctx* c, int nstep, double* sweep_ms, double* eloc_ms) {
  if (!c || nstep <= 0) return QWG_ERR_ARG;
  if (!c->dmc_ready) return fail(c, QWG_ERR_STATE, "qwg_time_kernels: call qwg_dmc_init first");
  if (c->block_pending) return fail(c, QWG_ERR_STATE, "qwg_time_kernels: a block is in flight");
  return guarded(c, [&]() -> int {
    BlockAcc* acc = c->d_acc.as<BlockAcc>();
    CK(cudaMemsetAsync(acc, 0, sizeof(BlockAcc), c->stream));
    StepParams P = base_params(c);
    P.nsteps = nstep;
    P.tau = c->dmc.timestep;
    P.dmc = 1;
    P.dyn_step = 1;
    P.refresh = 0;
    P.deterministic_pp = c->dmc.deterministic_pp;
    P.seed = c->dmc.seed ^ 0x7157ull;  // a stream of its own
    P.acc = acc;
    P.branch_start = c->branch_start;
    P.branch_stop = c->branch_stop;
    P.max_weight = c->dmc.max_poss_weight;
    EvalIO io{};
    std::vector<cudaEvent_t> ev(3 * nstep);
    for (auto& e : ev) CK(cudaEventCreate(&e));
    for (int st = 0; st < nstep; st++) {
      P.st = st;
      CK(cudaEventRecord(ev[3 * st], c->stream));
      launch_walkers(c, P, io, KM_SWEEP, c->nwalk);
      CK(cudaEventRecord(ev[3 * st + 1], c->stream));
      launch_walkers(c, P, io, KM_ELOC, c->nwalk);
      CK(cudaEventRecord(ev[3 * st + 2], c->stream));
    }
    CK(cudaStreamSynchronize(c->stream));
    double ts = 0, te = 0;
    for (int st = 0; st < nstep; st++) {
      float a = 0, b = 0;
      CK(cudaEventElapsedTime(&a, ev[3 * st], ev[3 * st + 1]));
      CK(cudaEventElapsedTime(&b, ev[3 * st + 1], ev[3 * st + 2]));
      ts += a; te += b;
    }
    for (auto& e : ev) cudaEventDestroy(e);
    if (sweep_ms) *sweep_ms = ts / nstep;
    if (eloc_ms) *eloc_ms = te / nstep;
    return QWG_OK;
  });
}

int qwg_autotune(qwg_ctx* c, int* walkers_per_cta) {
  if (!c) return QWG_ERR_ARG;
  if (c->nwalk <= 0) return fail(c, QWG_ERR_STATE, "qwg_autotune: no walkers");
  return guarded(c, [&]() -> int {
    const int W = c->nwalk;
    size_t n_g = (size_t)W * c->H.nelec * 3, n_l = (size_t)W * c->H.nelec;
    ensure_io(c, 8 * (5 * (size_t)W + n_g + n_l));
    double* base = c->d_io.as<double>();
    EvalIO io{};
    io.logpsi = base; io.sign = base + W; io.kinetic = base + 2 * W; io.potential = base + 3 * W;
    io.nonlocal = base + 4 * W; io.grad = base + 5 * W; io.lap = io.grad + n_g;
    // shared memory per walker (none for HBM-resident walkers)
    const size_t per = hbm_family(c->mmax) ? 0 : (size_t)c->L.bytes;
    int best = c->wpc;
    float best_ms = 1e30f;
    for (int cand : {1, 2, 4}) {
      if ((size_t)cand * per > 227 * 1024) continue;
      c->wpc = cand;
      c->smem_bytes = (size_t)cand * per;
      StepParams P = base_params(c);
      launch_walkers(c, P, io, KM_EVAL, W);  // warm-up (and attribute)
      CK(cudaEventRecord(c->ev0, c->stream));
      for (int r = 0; r < 3; r++) launch_walkers(c, P, io, KM_EVAL, W);
      CK(cudaEventRecord(c->ev1, c->stream));
      CK(cudaEventSynchronize(c->ev1));
      float ms = 0;
      CK(cudaEventElapsedTime(&ms, c->ev0, c->ev1));
      if (ms < best_ms) { best_ms = ms; best = cand; }
    }
    c->wpc = best;
    c->smem_bytes = (size_t)best * per;
    c->state_valid = false;
    c->dmc_ready = false;
    if (walkers_per_cta) *walkers_per_cta = best;
    return QWG_OK;
  });
}

long long qwg_launch_count(const qwg_ctx* c) { return c ? c->launches : 0; }
void qwg_reset_launch_count(qwg_ctx* c) { if (c) c->launches = 0; }

}  // extern "C"
