// Device code of the B200 walker engine.
//
// Execution model: one warp owns one walker for a whole kernel (a DMC
// feedback interval or a VMC block).  The walker's state -- positions, the
// transposed inverse Slater matrices of both spins, the MO gradient/Laplacian
// rows of every electron, the Jastrow gradient/Laplacian sums -- lives in
// shared memory while the warp works on it and is written back to its HBM
// slot once at the end.  Read-only tables (radial spline coefficients, MO
// coefficients, Jastrow and pseudopotential parameters) are shared by all
// walkers: MO coefficients are staged into shared memory per CTA, splines are
// read through L1/L2 (they fit in L2 many times over).
//
// Within a walker, lanes split the independent pieces of each phase: basis
// shells for one position, (MO, component) outputs of the MO contraction,
// electrons or pairs for the Jastrow, quadrature points for the pseudopotential
// (one lane evaluates a whole point: basis values dotted with the electron's
// projected coefficients, and the Jastrow).  Phases communicate through
// shared memory with __syncwarp().
//
// Real = double: everything in FP64.  Real = float (mixed precision): basis,
// MO values, determinant ratios, inverse and its Sherman-Morrison updates in
// FP32; the periodic full re-inversion (Gauss-Jordan), log|det|, Jastrow sums,
// local energies and weights in FP64.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>
#include <math_constants.h>

namespace qwg {

// ---------------------------------------------------------------------------
// tables

struct DRadial {
  int kind;         // 0 CUTOFF_CUSP, 1 POLYPADE, 2 PADE
  double rcut, inv_rcut;
  double a, b, c;   // CUTOFF_CUSP: cusp, gamma, 1/(3+gamma) ; POLYPADE: beta ; PADE: alpha
};
struct DTB {
  int k, l, m;      // e-n functions k, l of the atom's type, e-e function m
  double c, cu;     // coefficient for equal-spin / opposite-spin pairs
};

// Capacities of the tables carried in the kernel parameter bank.
constexpr int QWG_MAXA = 64;       // atoms
constexpr int QWG_MAXT = 8;        // atom types (labels)
constexpr int QWG_MAXEE = 8;       // e-e radial functions
constexpr int QWG_MAXEI = 8;       // e-n radial functions per type
constexpr int QWG_MAXTB = 12;      // e-e-n terms per type
constexpr int QWG_MAXPPT = 24;     // pseudopotential Gaussian terms per type (both spins of SPIN_DEP)
constexpr int QWG_MAXQ = 32;       // quadrature points
constexpr int QWG_MAXSHELL = 1024; // basis shells
constexpr int QWG_MAXDET = 64;     // determinants of an expansion
constexpr int QWG_MAXUD = 16;      // distinct determinants of one spin

// System tables.  Large tables (splines, MO coefficients, the per-shell
// arrays read by lanes that each take a different shell) live in HBM; the
// small ones are carried by value in the kernel's __grid_constant__
// parameter, so the uniform reads of the Jastrow, pseudopotential and
// per-center loops come from the constant cache instead of L1/L2.
template <typename Real>
struct DevSys {
  int nelec, nup, ndn, natoms, nbasis, nshell;
  int m[2];                      // electrons per spin (Slater matrix size)
  int mstride;                   // padded MO stride of moc rows (= MMAX)
  // determinant expansion (HBM-resident kernels only when ndet > 1):
  // psi_D = sum_k det_c[k] D_up(det_ud[2k]) D_down(det_ud[2k+1]); nmo_u[s]
  // orbitals per spin (union), ud_cols[(s * QWG_MAXUD + u) * mstride + i] =
  // union column of orbital i of spin-determinant u
  int ndet;
  int nud[2];
  int nmo_u[2];
  const double* det_c;
  const int* det_ud;
  const int* ud_cols;
  double ion_ion;
  const int4* shell_i;           // (center, sym, first, k) per shell, sorted by center
  const int2* shell_obj;         // (table base in 4-tuples, splines in the object)
  const double* shell_cut;       // [nshell]
  // radial spline tables, interval-major per basis object: the 4 cubic
  // coefficients of every spline of an object for interval i are contiguous
  // (one row of nk x 4 values), so all shells of a center read one row.
  const Real* spline;            // Real copy (value-only quadrature points)
  const double* spline64;        // FP64 copy (value/gradient/Laplacian)
  int npts;
  double spacing, inv_spacing;
  const Real* moc;               // [2][nbasis][mstride]
  // ---- parameter-bank tables
  double atom_pos[QWG_MAXA][3];
  double atom_charge[QWG_MAXA];
  int atom_type[QWG_MAXA];
  int4 center_seg[QWG_MAXA];     // (first shell, shells, spline-object base, splines in the object)
  double center_cut[QWG_MAXA];   // basis-object threshold of the center
  int shell_pack[QWG_MAXSHELL];  // sym | first << 4 | k << 20
  // Jastrow
  int nee;
  DRadial ee[QWG_MAXEE];
  double ee_like[QWG_MAXEE], ee_unlike[QWG_MAXEE];
  int ei_n[QWG_MAXT];
  DRadial ei[QWG_MAXT][QWG_MAXEI];
  double onebody[QWG_MAXT][QWG_MAXEI];
  int tb_n[QWG_MAXT];
  double tb_rc[QWG_MAXT];        // largest e-i cutoff the type's e-e-n terms use
  double ee_rc2;                 // (largest e-e cutoff)^2 (1 + 1e-12): every pair term (two- and
                                 // three-body) vanishes for electrons at least that far apart
  DTB tb[QWG_MAXT][QWG_MAXTB];
  int has_tb;
  // value-only ratios (pseudopotential quadrature): the e-e-n terms take the
  // moved electron's e-n basis at its current position.  The reference's
  // Jastrow2_wf::updateVal (Jastrow2_wf.cpp:877-882, 931-936) refreshes the
  // saved e-n basis only when a group has a plain THREEBODY term, so with
  // THREEBODY_SPIN alone its quadrature ratios see the stale values.
  int tb_stale_ei;
  // pseudopotential per type (nchan 0: none)
  int has_pp;
  int pp_nchan[QWG_MAXT], pp_aip[QWG_MAXT];
  double pp_cutoff[QWG_MAXT];
  int pp_term_first[QWG_MAXT][8];      // spin-up electrons
  int pp_term_first_dn[QWG_MAXT][8];   // spin-down electrons (SPIN_DEP; else the same)
  int pp_addzeff[QWG_MAXT];            // ADD_ZEFF: +Z_ion/r in the local channel
  double pp_term[QWG_MAXT][QWG_MAXPPT][3];  // (n, a, c)
  double pp_quad[QWG_MAXT][QWG_MAXQ][3];
  double pp_w[QWG_MAXT][QWG_MAXQ];
  // periodic cell (periodic == 0: molecule, one image per atom = the atom)
  int periodic;
  double lat[3][3], normvec[3][3], origin[3], corners[3][3];
  double h2q;                    // (smallest cell height / 2)^2: minimum-image shortcut
  int ortho;                     // lattice vectors along x, y, z (orthorhombic cell)
  double lattice_basis[27][3];
  double alpha, ewald_const;
  int2 atom_images[QWG_MAXA];    // (first, count) into image_pos
  const double* image_pos;       // [nimage][3] basis centers (atoms and their images)
  // sub-cell candidate lists of the image sums: the cell cut into sub_n[0] x
  // sub_n[1] x sub_n[2] parallelepipeds; sub_seg[s * natoms + c] = (first,
  // count) into sub_idx, the image indices of atom c (in image order) within
  // reach of some point of sub-cell s.  Null for molecules.
  int sub_n[3];
  double sub_inv_h[3];           // 1 / (normvec[i] . lat[i])
  const int2* sub_seg;
  const int* sub_idx;
  // complex-orbital kernels (CORBITALS, or real orbitals at a nonzero k-point):
  // planar complex tables (imaginary plane of the MO coefficients in moc_im,
  // same layout as moc); image_kfac[m] = k-point factor of image center m,
  // e^{i pi k.n} for complex orbitals and cos(pi k.n) for real ones, n its
  // lattice translation (MO_matrix.h:333-342, MO_matrix_blas.h:179-188)
  const Real* moc_im;
  const double* image_kfac;      // [nimage][2]
  double kpt[3];                 // KPOINT
  int kint;                      // every k component an integer: the overall sign
                                 // cos(pi k.n) of a wrap enters node checks and PP signs
  int real_orb;                  // orbitals real (ORBITALS at a nonzero k-point)
  int xl;                        // F/G shells or CUTOFF_MO: the FP32 HBM-resident kernels compiled with their code
  int cutoff_mo;                 // CUTOFF_MO evaluator (HBM-resident kernels): shell_cut holds
                                 // each spline's own cutoff, no |value| <= 1e-8 skip
  int ng;                        // Ewald G-vectors
  const double* gvec;            // [ng][3]
  const double* gweight;         // [ng]
  const double* ion_sin;         // [ng]
  const double* ion_cos;         // [ng]
};

// Minimum-image vector (Periodic_sample::minimum_image,
// system/Periodic_sample.cpp:259-287); identity for molecules.
template <typename Real>
__device__ __forceinline__ void min_image(const DevSys<Real>& S, double& x, double& y, double& z) {
  if (!S.periodic) return;
  const double d2 = x * x + y * y + z * z;
  if (d2 < S.h2q) return;
  if (S.ortho) {
    // orthorhombic cell: the 27-image search reduces to one independent
    // choice per axis among x - L, x, x + L (the same sums it would form)
    const double lx = S.lat[0][0], ly = S.lat[1][1], lz = S.lat[2][2];
    if (x > 0.5 * lx) x -= lx; else if (x < -0.5 * lx) x += lx;
    if (y > 0.5 * ly) y -= ly; else if (y < -0.5 * ly) y += ly;
    if (z > 0.5 * lz) z -= lz; else if (z < -0.5 * lz) z += lz;
    return;
  }
  double bx = x, by = y, bz = z, bd = 1e99;
  for (int a = 0; a < 27; a++) {
    const double tx = x + S.lattice_basis[a][0], ty = y + S.lattice_basis[a][1], tz = z + S.lattice_basis[a][2];
    const double td = tx * tx + ty * ty + tz * tz;
    if (td < bd) {
      bx = tx; by = ty; bz = tz; bd = td;
      if (td < S.h2q) break;
    }
  }
  x = bx; y = by; z = bz;
}

// Put a position inside the cell (Periodic_system::enforcePbc,
// system/Periodic_system.cpp:521-570).  At most 64 shifts per direction.
template <typename Real>
__device__ __forceinline__ void wrap_pos(const DevSys<Real>& S, double& x, double& y, double& z) {
  if (!S.periodic) return;
  for (int i = 0; i < 3; i++) {
    for (int it = 0; it < 64; it++) {
      const double* n = S.normvec[i];
      const double sh = n[0] * (x - S.origin[0]) + n[1] * (y - S.origin[1]) + n[2] * (z - S.origin[2]);
      const double fa = n[0] * (x - S.corners[i][0]) + n[1] * (y - S.corners[i][1]) + n[2] * (z - S.corners[i][2]);
      if (sh < -1e-12) { x += S.lat[i][0]; y += S.lat[i][1]; z += S.lat[i][2]; }
      else if (fa > 1e-12) { x -= S.lat[i][0]; y -= S.lat[i][1]; z -= S.lat[i][2]; }
      else break;
    }
  }
}

// Sub-cell of a position inside the cell (the frame of wrap_pos), or -1
// outside it or without lists (molecules).
template <typename Real>
__device__ __forceinline__ int subcell_of(const DevSys<Real>& S, double x, double y, double z) {
  if (S.sub_seg == nullptr) return -1;
  int id = 0;
  for (int i = 0; i < 3; i++) {
    const double* n = S.normvec[i];
    const double f = (n[0] * (x - S.origin[0]) + n[1] * (y - S.origin[1]) + n[2] * (z - S.origin[2])) * S.sub_inv_h[i];
    if (!(f > -1e-9 && f < 1.0 + 1e-9)) return -1;
    id = id * S.sub_n[i] + min(S.sub_n[i] - 1, max(0, int(f * double(S.sub_n[i]))));
  }
  return id;
}

// The image centers of atom c a position of sub-cell sc can reach: the
// listed subset (same order) or, for sc < 0, all of the atom's images.
struct ImgRange {
  const int* idx;
  int first, count;
  __device__ __forceinline__ int operator[](int t) const { return idx ? __ldg(idx + first + t) : first + t; }
};
template <typename Real>
__device__ __forceinline__ ImgRange images_of(const DevSys<Real>& S, int sc, int c) {
  if (sc >= 0) {
    const int2 g = __ldg(&S.sub_seg[(size_t)sc * S.natoms + c]);
    return {S.sub_idx, g.x, g.y};
  }
  const int2 im = S.atom_images[c];
  return {nullptr, im.x, im.y};
}

// wrap_pos that also returns the lattice translations applied (nshift[i] +1
// for each +L_i, Periodic_system::enforcePbc, Periodic_system.cpp:521-570);
// their k-point phase pi k.n enters the pseudopotential ratios
// (Periodic_sample::translateElectron, Periodic_sample.cpp:388-420).
template <typename Real>
__device__ __forceinline__ double wrap_pos_kphase(const DevSys<Real>& S, double& x, double& y, double& z) {
  if (!S.periodic) return 0.0;
  int ns[3] = {0, 0, 0};
  for (int i = 0; i < 3; i++) {
    for (int it = 0; it < 64; it++) {
      const double* n = S.normvec[i];
      const double sh = n[0] * (x - S.origin[0]) + n[1] * (y - S.origin[1]) + n[2] * (z - S.origin[2]);
      const double fa = n[0] * (x - S.corners[i][0]) + n[1] * (y - S.corners[i][1]) + n[2] * (z - S.corners[i][2]);
      if (sh < -1e-12) { x += S.lat[i][0]; y += S.lat[i][1]; z += S.lat[i][2]; ns[i]++; }
      else if (fa > 1e-12) { x -= S.lat[i][0]; y -= S.lat[i][1]; z -= S.lat[i][2]; ns[i]--; }
      else break;
    }
  }
  return CUDART_PI * (S.kpt[0] * ns[0] + S.kpt[1] * ns[1] + S.kpt[2] * ns[2]);
}

// erfc approximation of the Ewald sum (A&S 7.1.26, Periodic_system.h:221-227)
__device__ __forceinline__ double erfc_poly(double x) {
  const double p = .3275911, a = .254829592, b = -.284496736, c = 1.421413741, d = -1.453152027, e = 1.061405429;
  double y = 1. / (1. + p * x);
  return y * (a + y * (b + y * (c + y * (d + y * e)))) * exp(-x * x);
}

// Per-walker shared-memory layout (byte offsets, host computed).
// Byte offsets of one walker's arrays.  R, inv, mov, gU, lU and scal are
// offsets into the persistent state (state_bytes per walker); bas, newcol,
// dG, lu, items, Ue, rot and wproj into the walker's scratch (scratch_bytes).
// Walkers with <= 32 orbitals per spin keep state + scratch together in
// shared memory (bytes = state_bytes + scratch_bytes per warp); larger ones
// work in place in HBM with one scratch region per walker.
struct WLayout {
  int R, inv, mov, gU, lU, scal, bas, newcol, dG, Ue, lu, items, rot, wproj, wchunk, bytes;
  int sweep_bytes;    // state + the move-phase scratch (shared memory per walker of the sweep kernel)
  int state_bytes;    // persistent walker state
  int scratch_bytes;  // per-walker scratch
  int mstride;        // row stride of the inverse / MO-derivative rows (orbitals, padded)
  // determinant expansions: nud distinct determinants per spin (1 for a single
  // determinant); state: udl [2][nud][2] (log|D|, sign), mdt [QWG_MAXDET + 2 +
  // 2 * QWG_MAXUD] (weights t_k, W, log reference, per-spin weight sums);
  // scratch: mdv [mstride][mstride] orbital values, mdr [QWG_MAXUD][5] ratios
  int nud, udl, mdt, mdv, mdr;
};

// Persistent scalars of a walker (inside the state prefix).
struct WScal {
  double logdet[2];
  double sign[2];
  double U;
  double eold;      // previous local energy (DMC weight)
  double weight;
  double phase;     // arg psi_D (complex-orbital kernels; 0 otherwise)
};

struct BlockAcc {   // per-launch reduction target (double atomics)
  double sum_w, sum_we, sum_wk, sum_wv, sum_wnl, sum_we2, accepted, attempted;
  double nonfinite, npts;
  // unweighted point sums for the block variances of the log
  // (Properties_manager::insertPoint / endBlock, Properties.cpp:437-640)
  double sum_e, sum_e2, sum_k, sum_k2, sum_v, sum_v2, sum_nl, sum_nl2, sum_wt, sum_wt2;
};
constexpr int QWG_NACC = 20;  // doubles in BlockAcc

// Device-resident DMC scalars (dyn[]): the whole block runs without a host
// round trip, so it can be replayed as one CUDA graph.
enum DynSlot {
  DYN_ETRIAL = 0,   // E_T
  DYN_TEFF = 1,     // effective time step of the weights
  DYN_SUMW = 2,     // sum of the walker weights after the last branching
  DYN_PAIRS = 3,    // split/kill pairs so far
  DYN_EREF = 4,     // E_ref (average of the block energies)
  DYN_STEP = 5,     // global step counter (RNG counter)
  DYN_BRANCH = 6,   // branching counter (RNG counter)
  DYN_NBLOCK = 7,   // blocks completed
  DYN_COUNT = 16
};

// Launch parameters shared by the step kernels.
// Phase counters of the walker kernels, compiled in with -DQWG_PHASES only
// (the profiling build libqwg_phases.so): each counter sums the clock64()
// cycles lane 0 of a walker's warp spends in one phase, over every walker.
enum QwgPhase {
  PH_MO = 0,          // basis rows + MO contraction of a proposal (or its read from the GEMM)
  PH_PROPOSE_REST,    // ratio, drift, Jastrow of the moved electron
  PH_ACCEPT,          // Sherman-Morrison update and state bookkeeping
  PH_KINETIC,
  PH_POTENTIAL,       // Coulomb or Ewald
  PH_PP_JASTROW,      // quadrature: Jastrow values of the electrons at their positions
  PH_PP_ITEMS,        // quadrature: (electron, atom) pairs inside the cutoff
  PH_PP_PROJECT,      // quadrature: projected coefficients C A^-1
  PH_PP_POINTS,       // quadrature: point ratios (basis values, Jastrow)
  PH_REFRESH,         // full recompute and re-inversion
  PH_WALKER,          // a walker's whole step-mode launch (moves or local energy)
  PH_PP_POINT_JAS,    // the Jastrow part of PH_PP_POINTS (lane 0's share of the warp)
  PH_COUNT = 16
};
#ifdef QWG_PHASES
#define QWG_PHASE_BEGIN(t) const long long t = clock64();
#define QWG_PHASE_END(t, slot, ctr) \
  if ((ctr) && (threadIdx.x & 31) == 0) atomicAdd(&(ctr)[slot], (unsigned long long)(clock64() - t));
#else
#define QWG_PHASE_BEGIN(t)
#define QWG_PHASE_END(t, slot, ctr)
#endif

struct StepParams {
  int nwalk;
  int nsteps;
  int st;               // KM_SWEEP / KM_ELOC: step of the chunk this launch performs
  int refresh;          // 1: full recompute at start, 0: load state, 2: recompute when the
                        //    chunk reaches a multiple of refresh_every steps (device counter)
  int refresh_every;
  int dmc;              // 1: DMC weights + node restriction
  int dyn_step;         // 1: take the step counter from etrial[DYN_STEP]
  int deterministic_pp;
  double tau;           // move time step
  double teff;          // DMC effective time step (weights)
  const double* etrial; // device scalars dyn[DYN_COUNT]
  double branch_start, branch_stop, max_weight;
  uint64_t seed;
  uint64_t step0;       // global step counter of the first step (dyn_step == 0)
  double* R;            // [W][N][3]
  unsigned char* state; // [W][state_bytes]
  unsigned char* scratch;  // [W][scratch_bytes] (HBM-resident walkers only)
  BlockAcc* acc;
  // T-moves (Dmc_method::doTmove, Dmc_method.cpp:850-906): 0 off, 1 one move
  // per walker (TMOVES), 2 one per electron (TMOVESSC)
  int tmoves;
  int tm_cap;           // quadrature terms per walker the candidate buffer holds
  // VMC dynamics (Split_sampler DEPTH / DIVIDER, the reference's VMC default
  // 2 / 2): a rejected move is retried from the same point with timestep
  // tau / divider (delayed rejection); the fused step kernel only
  int vmc_depth;
  double vmc_divider;
  double* tm_cand;      // [W][tm_cap] the current electron chunk's point terms
  double* tm_moves;     // [W][N][4] selected targets (x, y, z, 1) or flag 0
  // Tensor-core move schedule (KM_SWEEP, HBM-resident FP32 kernels): one
  // electron tc_e per launch.  Phase 1 proposes the move and writes the five
  // basis rows of the proposed position as split-TF32 pairs into the GEMM's
  // A operand (rows walker * 5 + component, kpad columns); the tensor-core
  // GEMM contracts them with the MO coefficients into tc_D (row stride
  // tc_ldd); phase 2 recomputes the same proposal and decides it with the
  // MO column read from tc_D.  tc_phase 0: the whole sweep in one launch.
  int tc_phase, tc_e, tc_kpad, tc_ldd;
  float* tc_ahi;
  float* tc_alo;
  const float* tc_D;
  unsigned long long* phases;  // [PH_COUNT] counters (profiling builds), or null
};

// ---------------------------------------------------------------------------
// counter-based RNG: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11) and
// Box-Muller normals.

struct U4 { uint32_t x, y, z, w; };

__device__ __forceinline__ U4 philox4x32(U4 c, uint32_t k0, uint32_t k1) {
  const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
  for (int r = 0; r < 10; r++) {
    uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
    uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
    U4 n;
    n.x = hi1 ^ c.y ^ k0;
    n.y = lo1;
    n.z = hi0 ^ c.w ^ k1;
    n.w = lo0;
    c = n;
    k0 += W0;
    k1 += W1;
  }
  return c;
}

// uniform in (0, 1]
__device__ __forceinline__ double u01(uint32_t a) { return (double(a) + 1.0) * (1.0 / 4294967296.0); }

struct Rand4 { double u[4]; };

__device__ __forceinline__ Rand4 rand4(uint64_t seed, uint32_t walker, uint64_t step, uint32_t e, uint32_t purpose) {
  U4 c;
  c.x = walker;
  c.y = (uint32_t)step;
  c.z = (uint32_t)(step >> 32) ^ (e << 8) ^ purpose;
  c.w = purpose * 0x9E3779B9u + e;
  U4 r = philox4x32(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  Rand4 o;
  o.u[0] = u01(r.x); o.u[1] = u01(r.y); o.u[2] = u01(r.z); o.u[3] = u01(r.w);
  return o;
}

// Two normal deviates from two uniforms (Box-Muller), in FP32 with the fast
// intrinsics, the angle taken in [-pi, pi) where __sincosf is accurate to
// ~2^-21 (a half turn of the angle maps the pair to its negative, so the
// deviates keep their distribution).  They only draw the proposal; the
// acceptance uses the realised displacement, and the FP32 rounding (~1e-7
// relative) perturbs the proposal density far below any statistical error,
// while the FP64 transcendentals leave the move loop.  Both precisions draw
// the same deviates.
__device__ __forceinline__ void box_muller(double u1, double u2, double& g1, double& g2) {
  const float rad = sqrtf(-2.0f * __logf(float(u1)));
  float s, c;
  __sincosf(6.2831853071795864f * (float(u2) - 0.5f), &s, &c);
  g1 = double(rad * c);
  g2 = double(rad * s);
}

// ---------------------------------------------------------------------------
// warp helpers

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// ---------------------------------------------------------------------------
// radial functions

// Quotient of the Jastrow radials: the fast FP32 divide (__fdividef, 2 ulp
// for the O(1) denominators here) in the working precision of the mixed path,
// the IEEE divide in FP64.
template <typename T>
__device__ __forceinline__ T jdiv(T x, T y) {
  if constexpr (sizeof(T) == 4) return __fdividef(x, y);
  else return x / y;
}

// Jastrow radial function (value, f'/r, 3D Laplacian).  Zero at r >= rcut.
template <typename T>
__device__ __forceinline__ void radial_lap(const DRadial& q, T r, T& f, T& fd, T& lap) {
  if (!(r < T(q.rcut))) { f = fd = lap = T(0); return; }
  const T ircut = T(q.inv_rcut);
  const T zz = r * ircut, zz2 = zz * zz;
  const T ir = jdiv(T(1), r);
  if (q.kind == 0) {  // CUTOFF_CUSP (cusp a, gamma b, 1/(3+gamma) c)
    const T cusp = T(q.a), gamma = T(q.b);
    T pp = zz - zz2 + zz * zz2 * T(1.0 / 3.0);
    T pade = jdiv(T(1), T(1) + gamma * pp);
    f = cusp * T(q.rcut) * (pp * pade - T(q.c));
    T pade2 = pade * pade;
    T ppd = T(1) - T(2) * zz + zz2;
    T ppdd = T(-2) + T(2) * zz;
    T dadr = ppd * pade2 * ir;
    fd = cusp * dadr;
    lap = cusp * ((ppdd * pade2 - T(2) * gamma * ppd * ppd * pade2 * pade) * ircut + T(2) * dadr);
  } else if (q.kind == 2) {  // PADE (alpha a): f = (a r / (1 + a r))^2
    const T pade = jdiv(T(1), T(1) + T(q.a) * r);
    const T app = T(q.a) * T(q.a) * pade * pade;
    f = app * r * r;
    fd = T(2) * app * pade;
    lap = T(3) * fd * pade;
  } else {            // POLYPADE (beta a)
    const T beta = T(q.a);
    T zpp = zz2 * (T(6) - T(8) * zz + T(3) * zz2);
    T zppd = T(12) * zz * (T(1) - T(2) * zz + zz2);
    T zppdd2 = T(6) - T(24) * zz + T(18) * zz2;
    T zpade = jdiv(T(1), T(1) + beta * zpp), zpade2 = zpade * zpade;
    f = (T(1) - zpp) * zpade;
    fd = -zppd * zpade2 * (beta + T(1)) * ir * ircut;
    T crsdd2 = -zpade2 * (zppdd2 - beta * zppd * zppd * zpade) * (beta + T(1)) * ircut * ircut;
    lap = T(2) * (crsdd2 + fd);
  }
}
template <typename T>
__device__ __forceinline__ T radial_val(const DRadial& q, T r) {
  if (!(r < T(q.rcut))) return T(0);
  const T zz = r * T(q.inv_rcut), zz2 = zz * zz;
  if (q.kind == 0) {
    T pp = zz - zz2 + zz * zz2 * T(1.0 / 3.0);
    return T(q.a) * T(q.rcut) * (jdiv(pp, T(1) + T(q.b) * pp) - T(q.c));
  }
  if (q.kind == 2) {
    const T ap = jdiv(T(q.a), T(1) + T(q.a) * r);
    return ap * ap * r * r;
  }
  T zpp = zz2 * (T(6) - T(8) * zz + T(3) * zz2);
  return jdiv(T(1) - zpp, T(1) + T(q.a) * zpp);
}

// ---------------------------------------------------------------------------
// Basis functions: Cartesian Gaussian-type A(x,y,z) f(r) from the spline's
// f, f'/r, f''.  Value, gradient (dA f + A f'/r r_vec) and Laplacian
// lap = A f'' + (2l+2) A f'/r + f lap(A) for a homogeneous A of degree l.
// Orderings follow the GAMESS conventions of Cubic_spline_build.cpp:660-760.

// Writes the 5 components of one function to out[0..4] (a basis row).
// ACC: add to out (image sums; the |value| rule is applied by the caller to
// the sums) instead of storing with the |value| <= 1e-8 rule of the dense
// evaluator (MO_matrix_blas.h:468-470).
template <typename Real, bool ACC>
__device__ __forceinline__ void put_lap(Real* out, double A, double ax, double ay, double az, double lapA, int l,
                                        double x, double y, double z, double f, double fd, double f2) {
  double v = A * f;
  double h = A * fd;
  double g0 = h * x + ax * f, g1 = h * y + ay * f, g2 = h * z + az * f;
  double lp = A * f2 + double(2 * l + 2) * h + lapA * f;
  if (ACC) {
    out[0] += Real(v); out[1] += Real(g0); out[2] += Real(g1); out[3] += Real(g2); out[4] += Real(lp);
  } else {
    bool keep = fabs(v) > 1e-8;
    out[0] = Real(keep ? v : 0.0);
    out[1] = Real(keep ? g0 : 0.0);
    out[2] = Real(keep ? g1 : 0.0);
    out[3] = Real(keep ? g2 : 0.0);
    out[4] = Real(keep ? lp : 0.0);
  }
}

template <typename Real, bool ACC>
__device__ __forceinline__ void shell_lap_store(int sym, double x, double y, double z, double f, double fd, double f2,
                                                Real* b /* [nf][5] */) {
  switch (sym) {
    case 0: put_lap<Real, ACC>(b, 1.0, 0.0, 0.0, 0.0, 0.0, 0, x, y, z, f, fd, f2); break;
    case 1:
      put_lap<Real, ACC>(b, x, 1.0, 0.0, 0.0, 0.0, 1, x, y, z, f, fd, f2);
      put_lap<Real, ACC>(b + 5, y, 0.0, 1.0, 0.0, 0.0, 1, x, y, z, f, fd, f2);
      put_lap<Real, ACC>(b + 10, z, 0.0, 0.0, 1.0, 0.0, 1, x, y, z, f, fd, f2);
      break;
    case 2:
      put_lap<Real, ACC>(b, x * x, 2 * x, 0.0, 0.0, 2.0, 2, x, y, z, f, fd, f2);
      put_lap<Real, ACC>(b + 5, y * y, 0.0, 2 * y, 0.0, 2.0, 2, x, y, z, f, fd, f2);
      put_lap<Real, ACC>(b + 10, z * z, 0.0, 0.0, 2 * z, 2.0, 2, x, y, z, f, fd, f2);
      put_lap<Real, ACC>(b + 15, x * y, y, x, 0.0, 0.0, 2, x, y, z, f, fd, f2);
      put_lap<Real, ACC>(b + 20, x * z, z, 0.0, x, 0.0, 2, x, y, z, f, fd, f2);
      put_lap<Real, ACC>(b + 25, y * z, 0.0, z, y, 0.0, 2, x, y, z, f, fd, f2);
      break;
    default:
      put_lap<Real, ACC>(b, 2 * z * z - x * x - y * y, -2 * x, -2 * y, 4 * z, 0.0, 2, x, y, z, f, fd, f2);
      put_lap<Real, ACC>(b + 5, x * z, z, 0.0, x, 0.0, 2, x, y, z, f, fd, f2);
      put_lap<Real, ACC>(b + 10, y * z, 0.0, z, y, 0.0, 2, x, y, z, f, fd, f2);
      put_lap<Real, ACC>(b + 15, x * x - y * y, 2 * x, -2 * y, 0.0, 0.0, 2, x, y, z, f, fd, f2);
      put_lap<Real, ACC>(b + 20, x * y, y, x, 0.0, 0.0, 2, x, y, z, f, fd, f2);
      break;
  }
}

__device__ __forceinline__ int sym_nfunc(int sym) {
  return sym == 0 ? 1 : sym == 1 ? 3 : sym == 2 ? 6 : sym == 3 ? 5 : sym == 4 ? 10 : sym <= 6 ? 7 : sym == 7 ? 15 : 9;
}

// ---- F and G shells (sym >= 4), compiled into the HBM-resident kernels only
// (decks with such shells run there).  Function q of the shell maps to one
// angular polynomial A (Cubic_spline_calc.cpp:106-296 values, 600-1080 with
// derivatives); its gradient and Laplacian enter put_lap.  Index of A:
// 0-9 Cartesian F (xxx yyy zzz xxy xxz yyx yyz zzx zzy xyz), 10 Fm3, 11 Fm1,
// 12 F0, 13 Fp1, 14 Fp2, 15 Fp3mod; 16-30 Cartesian G (xxxx yyyy zzzz xxxy
// xxxz yyyx yyyz zzzx zzzy xxyy xxzz yyzz xxyz yyxz zzxy); 31-39 G0..G8.
__device__ __forceinline__ int fg_index(int sym, int q) {
  // 7F: F0 Fm3 Fp3mod Fp2 Fxyz Fm1 Fp1; 7F_crystal: F0 Fp1 Fm1 Fp2 Fxyz Fp3mod Fm3
  // (Cubic_spline_build.cpp:702-721), packed 3 bits per function, offset 9
  constexpr int P7F = 3 | 1 << 3 | 6 << 6 | 5 << 9 | 0 << 12 | 2 << 15 | 4 << 18;
  constexpr int P7FC = 3 | 4 << 3 | 2 << 6 | 5 << 9 | 0 << 12 | 6 << 15 | 1 << 18;
  switch (sym) {
    case 4: return q;
    case 5: return 9 + ((P7F >> (3 * q)) & 7);
    case 6: return 9 + ((P7FC >> (3 * q)) & 7);
    case 7: return 16 + q;
    default: return 31 + q;
  }
}

// value of angular polynomial idx (same expressions as the reference's values)
template <typename T>
__device__ __forceinline__ T fg_value(int idx, T x, T y, T z) {
  const T v1 = x * x, v2 = y * y, v3 = z * z;
  switch (idx) {
    case 0: return v1 * x;
    case 1: return v2 * y;
    case 2: return v3 * z;
    case 3: return v1 * y;
    case 4: return v1 * z;
    case 5: return v2 * x;
    case 6: return v2 * z;
    case 7: return x * v3;
    case 8: return v3 * y;
    case 9: return x * y * z;
    case 10: return y * (T(3) * v1 - v2);
    case 11: return y * (T(4) * v3 - v1 - v2);
    case 12: return z * (T(2) * v3 - T(3) * (v1 + v2));
    case 13: return x * (T(4) * v3 - v1 - v2);
    case 14: return z * (v1 - v2);
    case 15: return x * (v1 - T(3) * v2);
    case 16: return v1 * v1;
    case 17: return v2 * v2;
    case 18: return v3 * v3;
    case 19: return v1 * x * y;
    case 20: return v1 * x * z;
    case 21: return v2 * y * x;
    case 22: return v2 * y * z;
    case 23: return v3 * z * x;
    case 24: return v3 * z * y;
    case 25: return v1 * v2;
    case 26: return v1 * v3;
    case 27: return v2 * v3;
    case 28: return v1 * y * z;
    case 29: return v2 * x * z;
    case 30: return v3 * x * y;
    case 31: { const T v5 = v1 + v2 + v3; return T(35) * v3 * v3 - T(30) * v3 * v5 + T(3) * v5 * v5; }
    case 32: { const T v5 = v1 + v2 + v3; return x * z * (T(7) * v3 - T(3) * v5); }
    case 33: { const T v5 = v1 + v2 + v3; return y * z * (T(7) * v3 - T(3) * v5); }
    case 34: { const T v5 = v1 + v2 + v3; return (v1 - v2) * (T(7) * v3 - v5); }
    case 35: { const T v5 = v1 + v2 + v3; return x * y * (T(7) * v3 - v5); }
    case 36: return (v1 - T(3) * v2) * x * z;
    case 37: return (T(3) * v1 - v2) * y * z;
    case 38: return (v1 - T(3) * v2) * v1 - (T(3) * v1 - v2) * v2;
    default: return (v1 - v2) * x * y;
  }
}

// value, gradient and Laplacian of angular polynomial idx
__device__ __forceinline__ void fg_lap(int idx, double x, double y, double z, double& A, double& ax, double& ay,
                                       double& az, double& lA) {
  const double v1 = x * x, v2 = y * y, v3 = z * z;
  A = fg_value<double>(idx, x, y, z);
  lA = 0.0;  // the real-harmonic F and G polynomials are harmonic
  switch (idx) {
    case 0: ax = 3 * v1; ay = 0; az = 0; lA = 6 * x; break;
    case 1: ax = 0; ay = 3 * v2; az = 0; lA = 6 * y; break;
    case 2: ax = 0; ay = 0; az = 3 * v3; lA = 6 * z; break;
    case 3: ax = 2 * x * y; ay = v1; az = 0; lA = 2 * y; break;
    case 4: ax = 2 * x * z; ay = 0; az = v1; lA = 2 * z; break;
    case 5: ax = v2; ay = 2 * x * y; az = 0; lA = 2 * x; break;
    case 6: ax = 0; ay = 2 * y * z; az = v2; lA = 2 * z; break;
    case 7: ax = v3; ay = 0; az = 2 * x * z; lA = 2 * x; break;
    case 8: ax = 0; ay = v3; az = 2 * y * z; lA = 2 * y; break;
    case 9: ax = y * z; ay = x * z; az = x * y; break;
    case 10: ax = 6 * x * y; ay = 3 * (v1 - v2); az = 0; break;
    case 11: ax = -2 * x * y; ay = 4 * v3 - v1 - 3 * v2; az = 8 * y * z; break;
    case 12: ax = -6 * x * z; ay = -6 * y * z; az = 6 * v3 - 3 * (v1 + v2); break;
    case 13: ax = 4 * v3 - 3 * v1 - v2; ay = -2 * x * y; az = 8 * x * z; break;
    case 14: ax = 2 * x * z; ay = -2 * y * z; az = v1 - v2; break;
    case 15: ax = 3 * (v1 - v2); ay = -6 * x * y; az = 0; break;
    case 16: ax = 4 * v1 * x; ay = 0; az = 0; lA = 12 * v1; break;
    case 17: ax = 0; ay = 4 * v2 * y; az = 0; lA = 12 * v2; break;
    case 18: ax = 0; ay = 0; az = 4 * v3 * z; lA = 12 * v3; break;
    case 19: ax = 3 * v1 * y; ay = v1 * x; az = 0; lA = 6 * x * y; break;
    case 20: ax = 3 * v1 * z; ay = 0; az = v1 * x; lA = 6 * x * z; break;
    case 21: ax = v2 * y; ay = 3 * v2 * x; az = 0; lA = 6 * x * y; break;
    case 22: ax = 0; ay = 3 * v2 * z; az = v2 * y; lA = 6 * y * z; break;
    case 23: ax = v3 * z; ay = 0; az = 3 * v3 * x; lA = 6 * x * z; break;
    case 24: ax = 0; ay = v3 * z; az = 3 * v3 * y; lA = 6 * y * z; break;
    case 25: ax = 2 * x * v2; ay = 2 * v1 * y; az = 0; lA = 2 * (v1 + v2); break;
    case 26: ax = 2 * x * v3; ay = 0; az = 2 * v1 * z; lA = 2 * (v1 + v3); break;
    case 27: ax = 0; ay = 2 * y * v3; az = 2 * v2 * z; lA = 2 * (v2 + v3); break;
    case 28: ax = 2 * x * y * z; ay = v1 * z; az = v1 * y; lA = 2 * y * z; break;
    case 29: ax = v2 * z; ay = 2 * x * y * z; az = x * v2; lA = 2 * x * z; break;
    case 30: ax = y * v3; ay = x * v3; az = 2 * x * y * z; lA = 2 * x * y; break;
    case 31:
      ax = 12 * (v1 + v2 - 4 * v3) * x; ay = 12 * (v1 + v2 - 4 * v3) * y; az = -48 * (v1 + v2 + v3) * z + 80 * v3 * z;
      break;
    case 32: ax = (-9 * v1 - 3 * v2 + 4 * v3) * z; ay = -6 * x * y * z; az = (-3 * v1 - 3 * v2 + 12 * v3) * x; break;
    case 33: ax = -6 * x * y * z; ay = (-3 * v1 - 9 * v2 + 4 * v3) * z; az = (-3 * v1 - 3 * v2 + 12 * v3) * y; break;
    case 34: ax = 4 * x * (3 * v3 - v1); ay = -4 * y * (3 * v3 - v2); az = 12 * z * (v1 - v2); break;
    case 35: ax = y * (6 * v3 - 3 * v1 - v2); ay = x * (6 * v3 - v1 - 3 * v2); az = 12 * x * y * z; break;
    case 36: ax = 3 * (v1 - v2) * z; ay = -6 * x * y * z; az = (v1 - 3 * v2) * x; break;
    case 37: ax = 6 * x * y * z; ay = 3 * (v1 - v2) * z; az = (3 * v1 - v2) * y; break;
    case 38: ax = 4 * x * (v1 - 3 * v2); ay = 4 * y * (v2 - 3 * v1); az = 0; break;
    default: ax = (3 * v1 - v2) * y; ay = (v1 - 3 * v2) * x; az = 0; break;
  }
}

template <typename Real, bool ACC>
__device__ __forceinline__ void shell_lap_store_fg(int sym, double x, double y, double z, double f, double fd,
                                                   double f2, Real* b) {
  const int nf = sym_nfunc(sym), l = sym <= 6 ? 3 : 4;
  for (int q = 0; q < nf; q++) {
    double A, ax, ay, az, lA;
    fg_lap(fg_index(sym, q), x, y, z, A, ax, ay, az, lA);
    put_lap<Real, ACC>(b + 5 * q, A, ax, ay, az, lA, l, x, y, z, f, fd, f2);
  }
}

// Basis value, gradient and Laplacian of every basis function at one
// position, warp-cooperative: lanes split the shells (radial spline and
// angular factors in FP64: the Laplacian of the tight shells cancels
// strongly); the rows go to bas [nbasis][5] in the output type O.
// PER: 0 molecule, 1 periodic cell (compiled for that case only), 2 decided
// at run time from S.periodic.
template <typename O, int PER, bool HL, typename Real>
__device__ void basis_lap_warp(const DevSys<Real>& S, double px, double py, double pz, O* bas, int lane) {
  const int sc = PER == 0 ? -1 : subcell_of(S, px, py, pz);
  for (int s = lane; s < S.nshell; s += 32) {
    int4 si = S.shell_i[s];
    int2 so = S.shell_obj[s];
    O* b = bas + si.z * 5;
    const int nf = sym_nfunc(si.y);
    const double cut = S.shell_cut[s];
    if (PER == 0 || (PER == 2 && !S.periodic)) {
      const double* ap = S.atom_pos[si.x];
      double dx = px - ap[0], dy = py - ap[1], dz = pz - ap[2];
      double r = sqrt(dx * dx + dy * dy + dz * dz);
      if (r < cut) {
        int i = int(r * S.inv_spacing);
        double h = r - double(i) * S.spacing;
        const double2* c2p = reinterpret_cast<const double2*>(S.spline64 + ((size_t)so.x + (size_t)i * so.y + si.w) * 4);
        double2 ca = __ldg(c2p), cb = __ldg(c2p + 1);
        double f = ca.x + h * (ca.y + h * (cb.x + h * cb.y));
        double fd = (ca.y + h * (2.0 * cb.x + h * (3.0 * cb.y))) / r;
        double f2 = 2.0 * cb.x + 6.0 * h * cb.y;
        if (HL && (si.y >= 4 || S.cutoff_mo)) {
          // accumulate into zeros: no |value| skip for CUTOFF_MO
          if (S.cutoff_mo)
            for (int k = 0; k < 5 * nf; k++) b[k] = O(0);
          if (si.y >= 4) {
            if (S.cutoff_mo) shell_lap_store_fg<O, true>(si.y, dx, dy, dz, f, fd, f2, b);
            else shell_lap_store_fg<O, false>(si.y, dx, dy, dz, f, fd, f2, b);
          } else {
            shell_lap_store<O, true>(si.y, dx, dy, dz, f, fd, f2, b);
          }
        } else {
          shell_lap_store<O, false>(si.y, dx, dy, dz, f, fd, f2, b);
        }
      } else {
        for (int k = 0; k < 5 * nf; k++) b[k] = O(0);
      }
    } else {
      // periodic: sum the shell over the atom's image centers, then apply the
      // |value| <= 1e-8 rule to the sums (MO_matrix_blas.h:444-474)
      for (int k = 0; k < 5 * nf; k++) b[k] = O(0);
      const ImgRange im = images_of(S, sc, si.x);
      const double cut2 = cut * cut * (1.0 + 1e-12);  // beyond it r < cut is certainly false
      for (int t = 0; t < im.count; t++) {
        const double* cp = S.image_pos + 3 * im[t];
        double dx = px - cp[0], dy = py - cp[1], dz = pz - cp[2];
        const double r2 = dx * dx + dy * dy + dz * dz;
        if (!(r2 < cut2)) continue;
        double r = sqrt(r2);
        if (!(r < cut)) continue;
        int i = int(r * S.inv_spacing);
        double h = r - double(i) * S.spacing;
        const double2* c2p = reinterpret_cast<const double2*>(S.spline64 + ((size_t)so.x + (size_t)i * so.y + si.w) * 4);
        double2 ca = __ldg(c2p), cb = __ldg(c2p + 1);
        double f = ca.x + h * (ca.y + h * (cb.x + h * cb.y));
        double fd = (ca.y + h * (2.0 * cb.x + h * (3.0 * cb.y))) / r;
        double f2 = 2.0 * cb.x + 6.0 * h * cb.y;
        if (HL && si.y >= 4) shell_lap_store_fg<O, true>(si.y, dx, dy, dz, f, fd, f2, b);
        else shell_lap_store<O, true>(si.y, dx, dy, dz, f, fd, f2, b);
      }
      if (!(HL && S.cutoff_mo))
        for (int k = 0; k < nf; k++)
          if (!(fabs(double(b[5 * k])) > 1e-8))
            for (int c = 0; c < 5; c++) b[5 * k + c] = O(0);
    }
  }
  __syncwarp();
}

// MO value, gradient and Laplacian of one position, warp-cooperative: the
// basis rows (basis_lap_warp) in bas [nbasis][5] as Real, then lanes split
// the (MO, component) outputs of the contraction with the MO coefficients
// moc_s [nbasis][mstride].
template <typename Real, int PER, bool HL = false>
__device__ void mo_lap_warp(const DevSys<Real>& S, const Real* moc_s, double px, double py, double pz, int M,
                            Real* bas, Real* out, int lane) {
  basis_lap_warp<Real, PER, HL>(S, px, py, pz, bas, lane);
  __syncwarp();
  if (M > 32) {
    // many orbitals: lanes over MOs (coalesced coefficient rows), the basis
    // values are warp-uniform reads
    for (int mo = lane; mo < M; mo += 32) {
      Real a0 = Real(0), a1 = Real(0), a2 = Real(0), a3 = Real(0), a4 = Real(0);
      const Real* w = moc_s + mo;
      for (int f = 0; f < S.nbasis; f++) {
        const Real c = w[(size_t)f * S.mstride];
        const Real* bb = bas + f * 5;
        a0 += bb[0] * c; a1 += bb[1] * c; a2 += bb[2] * c; a3 += bb[3] * c; a4 += bb[4] * c;
      }
      out[mo * 5] = a0; out[mo * 5 + 1] = a1; out[mo * 5 + 2] = a2; out[mo * 5 + 3] = a3; out[mo * 5 + 4] = a4;
    }
    __syncwarp();
    return;
  }
  // contraction: lane (mo, chunk) sums the 5 components of one MO over a
  // slice of the basis (5 independent accumulators), then the slices of an
  // MO are added with shuffles
  const int nch = M > 16 ? 1 : M > 8 ? 2 : M > 4 ? 4 : 8;  // lanes per MO (M * nch <= 32)
  const int mo = lane / nch, ch = lane - mo * nch;
  const int fper = (S.nbasis + nch - 1) / nch;
  Real a0 = Real(0), a1 = Real(0), a2 = Real(0), a3 = Real(0), a4 = Real(0);
  if (mo < M) {
    const int f0 = ch * fper, f1 = min(S.nbasis, f0 + fper);
    const Real* w = moc_s + mo;
    for (int f = f0; f < f1; f++) {
      const Real c = w[f * S.mstride];
      const Real* bb = bas + f * 5;
      a0 += bb[0] * c; a1 += bb[1] * c; a2 += bb[2] * c; a3 += bb[3] * c; a4 += bb[4] * c;
    }
  }
  for (int o = 1; o < nch; o <<= 1) {
    a0 += __shfl_xor_sync(0xffffffffu, a0, o);
    a1 += __shfl_xor_sync(0xffffffffu, a1, o);
    a2 += __shfl_xor_sync(0xffffffffu, a2, o);
    a3 += __shfl_xor_sync(0xffffffffu, a3, o);
    a4 += __shfl_xor_sync(0xffffffffu, a4, o);
  }
  if (mo < M && ch == 0) {
    out[mo * 5] = a0; out[mo * 5 + 1] = a1; out[mo * 5 + 2] = a2; out[mo * 5 + 3] = a3; out[mo * 5 + 4] = a4;
  }
  __syncwarp();
}

// Cubic spline value at offset h from the row's 4 coefficients c (16-byte
// aligned): one 16-byte load in FP32, two in FP64.
template <typename Real>
__device__ __forceinline__ Real spline_val(const Real* c, Real h) {
  if constexpr (sizeof(Real) == 4) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(c));
    return v.x + h * (v.y + h * (v.z + h * v.w));
  } else {
    const double2 a = __ldg(reinterpret_cast<const double2*>(c)), b = __ldg(reinterpret_cast<const double2*>(c) + 1);
    return a.x + h * (a.y + h * (b.x + h * b.y));
  }
}

// Determinant ratio of one electron moved to p, evaluated entirely by the
// calling lane (pseudopotential quadrature points): with the projected
// coefficients w_f = sum_m C[f][m] (A^-1)[m][e] of that electron,
//   psi_D(p)/psi_D = sum_m phi_m(p) (A^-1)[m][e] = sum_f b_f(p) w_f,
// an nbasis-term dot product instead of the nbasis x M MO contraction.
template <typename Real, bool HL = false>
__device__ __forceinline__ Real basis_dot_lane(const DevSys<Real>& S, double px, double py, double pz,
                                               const Real* w) {
  Real acc = Real(0);
  const bool cmo = HL && S.cutoff_mo;  // CUTOFF_MO: no |value| skip, per-function cutoffs
  auto add = [&](int f, Real v) { acc += (cmo || fabs(v) > Real(1e-8) ? v : Real(0)) * w[f]; };
  constexpr int B = sizeof(Real) == 4 ? 6 : 4;  // spline rows loaded per batch
  for (int c = 0; c < S.natoms; c++) {
    const int4 cs = S.center_seg[c];  // first shell, shells, object base, splines per row
    if (cs.y == 0) continue;
    const double* ap = S.atom_pos[c];
    const Real x = Real(px - ap[0]), y = Real(py - ap[1]), z = Real(pz - ap[2]);
    const Real rd = sqrt(x * x + y * y + z * z);
    if (!(rd < Real(S.center_cut[c]))) continue;
    const int i = int(rd * Real(S.inv_spacing));
    const Real h = rd - Real(i) * Real(S.spacing);
    const Real* row = S.spline + ((size_t)cs.z + (size_t)i * cs.w) * 4;
    for (int k0 = 0; k0 < cs.y; k0 += B) {
      Real cf[B][4];
#pragma unroll
      for (int j = 0; j < B; j++)
        if (k0 + j < cs.y) {
          const int k = (S.shell_pack[cs.x + k0 + j] >> 20) & 0xff;
          if constexpr (sizeof(Real) == 4) {
            const float4 v = __ldg(reinterpret_cast<const float4*>(row + 4 * k));
            cf[j][0] = v.x; cf[j][1] = v.y; cf[j][2] = v.z; cf[j][3] = v.w;
          } else {
            const double2 a = __ldg(reinterpret_cast<const double2*>(row + 4 * k));
            const double2 b = __ldg(reinterpret_cast<const double2*>(row + 4 * k) + 1);
            cf[j][0] = a.x; cf[j][1] = a.y; cf[j][2] = b.x; cf[j][3] = b.y;
          }
        }
#pragma unroll
      for (int j = 0; j < B; j++) {
        if (k0 + j >= cs.y) break;
        if constexpr (HL)
          if (cmo && !(rd < Real(S.shell_cut[cs.x + k0 + j]))) continue;
        const int pk = S.shell_pack[cs.x + k0 + j];
        const int sym = pk & 0xf, fb = (pk >> 4) & 0xffff;
        const Real f = cf[j][0] + h * (cf[j][1] + h * (cf[j][2] + h * cf[j][3]));
        switch (sym) {
          case 0: add(fb, f); break;
          case 1: add(fb, x * f); add(fb + 1, y * f); add(fb + 2, z * f); break;
          case 2:
            add(fb, x * x * f); add(fb + 1, y * y * f); add(fb + 2, z * z * f);
            add(fb + 3, x * y * f); add(fb + 4, x * z * f); add(fb + 5, y * z * f);
            break;
          default:
            if constexpr (HL) {
              if (sym >= 4) {
                for (int q = 0; q < sym_nfunc(sym); q++) add(fb + q, fg_value<Real>(fg_index(sym, q), x, y, z) * f);
                break;
              }
            }
            add(fb, (Real(2) * z * z - x * x - y * y) * f); add(fb + 1, x * z * f); add(fb + 2, y * z * f);
            add(fb + 3, (x * x - y * y) * f); add(fb + 4, x * y * f);
            break;
        }
      }
    }
  }
  return acc;
}

// basis_dot_lane for several projected-coefficient vectors at once (the
// distinct spin-determinants of an expansion): acc[u] = sum_f b_f(p) w[u *
// wstride + f] for u < nu (molecules).
template <typename Real>
__device__ __forceinline__ void basis_dot_lane_multi(const DevSys<Real>& S, double px, double py, double pz,
                                                     const Real* w, int wstride, int nu, Real* acc) {
#pragma unroll
  for (int u = 0; u < QWG_MAXUD; u++) acc[u] = Real(0);
  const bool cmo = S.cutoff_mo;  // HBM-resident kernels only
  auto add = [&](int f, Real v) {
    const Real vv = cmo || fabs(v) > Real(1e-8) ? v : Real(0);
#pragma unroll
    for (int u = 0; u < QWG_MAXUD; u++)
      if (u < nu) acc[u] += vv * w[(size_t)u * wstride + f];
  };
  for (int c = 0; c < S.natoms; c++) {
    const int4 cs = S.center_seg[c];
    if (cs.y == 0) continue;
    const double* ap = S.atom_pos[c];
    const Real x = Real(px - ap[0]), y = Real(py - ap[1]), z = Real(pz - ap[2]);
    const Real rd = sqrt(x * x + y * y + z * z);
    if (!(rd < Real(S.center_cut[c]))) continue;
    const int i = int(rd * Real(S.inv_spacing));
    const Real h = rd - Real(i) * Real(S.spacing);
    const Real* row = S.spline + ((size_t)cs.z + (size_t)i * cs.w) * 4;
    for (int k0 = 0; k0 < cs.y; k0++) {
      if (cmo && !(rd < Real(S.shell_cut[cs.x + k0]))) continue;
      const int pk = S.shell_pack[cs.x + k0];
      const int sym = pk & 0xf, fb = (pk >> 4) & 0xffff, kk = (pk >> 20) & 0xff;
      const Real* cf = row + 4 * kk;
      const Real f = spline_val(cf, h);
      switch (sym) {
        case 0: add(fb, f); break;
        case 1: add(fb, x * f); add(fb + 1, y * f); add(fb + 2, z * f); break;
        case 2:
          add(fb, x * x * f); add(fb + 1, y * y * f); add(fb + 2, z * z * f);
          add(fb + 3, x * y * f); add(fb + 4, x * z * f); add(fb + 5, y * z * f);
          break;
        case 3:
          add(fb, (Real(2) * z * z - x * x - y * y) * f); add(fb + 1, x * z * f); add(fb + 2, y * z * f);
          add(fb + 3, (x * x - y * y) * f); add(fb + 4, x * y * f);
          break;
        default:
          for (int q = 0; q < sym_nfunc(sym); q++) add(fb + q, fg_value<Real>(fg_index(sym, q), x, y, z) * f);
          break;
      }
    }
  }
}

// Periodic version of basis_dot_lane: each atom's functions are summed over
// its image centers before the |value| rule and the dot with w.
constexpr int QWG_MAXF_ATOM = 16;  // basis functions per atom on the periodic path
template <typename Real, bool HL = false>
__device__ __forceinline__ Real basis_dot_lane_periodic(const DevSys<Real>& S, double px, double py, double pz,
                                                        const Real* w) {
  Real acc = Real(0);
  const int sc = subcell_of(S, px, py, pz);
  for (int c = 0; c < S.natoms; c++) {
    const int4 cs = S.center_seg[c];  // first shell, shells, object base, splines per row
    if (cs.y == 0) continue;
    Real fs[QWG_MAXF_ATOM];
    int nfa = 0;
    for (int k = 0; k < cs.y; k++) nfa += sym_nfunc(S.shell_pack[cs.x + k] & 0xf);
    for (int q = 0; q < QWG_MAXF_ATOM; q++) fs[q] = Real(0);
    const int fb0 = (S.shell_pack[cs.x] >> 4) & 0xffff;
    const ImgRange im = images_of(S, sc, c);
    const Real cut = Real(S.center_cut[c]);
    const Real cut2 = cut * cut * Real(1.000001);  // beyond it rd < cut is certainly false
    for (int t = 0; t < im.count; t++) {
      const double* cp = S.image_pos + 3 * im[t];
      const Real x = Real(px - cp[0]), y = Real(py - cp[1]), z = Real(pz - cp[2]);
      const Real rd2 = x * x + y * y + z * z;
      if (!(rd2 < cut2)) continue;
      const Real rd = sqrt(rd2);
      if (!(rd < cut)) continue;
      const int i = int(rd * Real(S.inv_spacing));
      const Real h = rd - Real(i) * Real(S.spacing);
      const Real* row = S.spline + ((size_t)cs.z + (size_t)i * cs.w) * 4;
      for (int k = 0; k < cs.y; k++) {
        if constexpr (HL)
          if (S.cutoff_mo && !(rd < Real(S.shell_cut[cs.x + k]))) continue;
        const int pk = S.shell_pack[cs.x + k];
        const int sym = pk & 0xf, fo = ((pk >> 4) & 0xffff) - fb0, kk = (pk >> 20) & 0xff;
        const Real* cf = row + 4 * kk;
        const Real f = spline_val(cf, h);
        switch (sym) {
          case 0: fs[fo] += f; break;
          case 1: fs[fo] += x * f; fs[fo + 1] += y * f; fs[fo + 2] += z * f; break;
          case 2:
            fs[fo] += x * x * f; fs[fo + 1] += y * y * f; fs[fo + 2] += z * z * f;
            fs[fo + 3] += x * y * f; fs[fo + 4] += x * z * f; fs[fo + 5] += y * z * f;
            break;
          default:
            if constexpr (HL) {
              if (sym >= 4) {
                for (int q = 0; q < sym_nfunc(sym) && fo + q < QWG_MAXF_ATOM; q++)
                  fs[fo + q] += fg_value<Real>(fg_index(sym, q), x, y, z) * f;
                break;
              }
            }
            fs[fo] += (Real(2) * z * z - x * x - y * y) * f; fs[fo + 1] += x * z * f; fs[fo + 2] += y * z * f;
            fs[fo + 3] += (x * x - y * y) * f; fs[fo + 4] += x * y * f;
            break;
        }
      }
    }
    const bool cmo = HL && S.cutoff_mo;
    for (int q = 0; q < nfa; q++) acc += (cmo || fabs(fs[q]) > Real(1e-8) ? fs[q] : Real(0)) * w[fb0 + q];
  }
  return acc;
}

// ---------------------------------------------------------------------------
// Complex orbitals (MO_matrix_blas<dcomplex>, MO_matrix_blas.h:336-491).
// Complex arrays are planar: the real plane, then the imaginary plane.

// Spline value f, f'/r and f'' of one shell at distance r (r < cutoff).
template <typename Real>
__device__ __forceinline__ void shell_radial64(const DevSys<Real>& S, int2 so, int k, double r, double& f, double& fd,
                                               double& f2) {
  const int i = int(r * S.inv_spacing);
  const double h = r - double(i) * S.spacing;
  const double2* c2p = reinterpret_cast<const double2*>(S.spline64 + ((size_t)so.x + (size_t)i * so.y + k) * 4);
  const double2 ca = __ldg(c2p), cb = __ldg(c2p + 1);
  f = ca.x + h * (ca.y + h * (cb.x + h * cb.y));
  fd = (ca.y + h * (2.0 * cb.x + h * (3.0 * cb.y))) / r;
  f2 = 2.0 * cb.x + 6.0 * h * cb.y;
}

// MO values, gradients and Laplacians of one position: each shell summed
// over its atom's image centers times the image's k-point factor, the
// |value| <= 1e-8 rule on the modulus of the sums (MO_matrix_blas.h:444-474),
// then the complex contraction with the coefficients.  Molecules have one
// image per atom (the atom, factor 1).  bas: [nbasis][5] + imaginary plane at
// bas + 5 nbasis; out: [M][5] + imaginary plane at out + 5 ms.
template <typename Real>
__device__ void mo_lap_warp_cpx(const DevSys<Real>& S, const Real* moc_re, const Real* moc_im, double px, double py,
                                double pz, int M, int ms, Real* bas, Real* out, int lane) {
  const int nb5 = 5 * S.nbasis;
  const int sc = subcell_of(S, px, py, pz);
  for (int s = lane; s < S.nshell; s += 32) {
    const int4 si = S.shell_i[s];
    const int2 so = S.shell_obj[s];
    Real* br = bas + si.z * 5;
    Real* bi = br + nb5;
    const int nf = sym_nfunc(si.y);
    for (int k = 0; k < 5 * nf; k++) br[k] = bi[k] = Real(0);
    const double cut = S.shell_cut[s];
    const double cut2 = cut * cut * (1.0 + 1e-12);
    const ImgRange im = images_of(S, sc, si.x);
    for (int t = 0; t < im.count; t++) {
      const int m = im[t];
      const double* cp = S.image_pos + 3 * m;
      const double dx = px - cp[0], dy = py - cp[1], dz = pz - cp[2];
      const double r2 = dx * dx + dy * dy + dz * dz;
      if (!(r2 < cut2)) continue;
      const double r = sqrt(r2);
      if (!(r < cut)) continue;
      double f, fd, f2;
      shell_radial64(S, so, si.w, r, f, fd, f2);
      const double kc = S.image_kfac[2 * m], ks = S.image_kfac[2 * m + 1];
      if (si.y >= 4) {
        shell_lap_store_fg<Real, true>(si.y, dx, dy, dz, f * kc, fd * kc, f2 * kc, br);
        if (ks != 0.0) shell_lap_store_fg<Real, true>(si.y, dx, dy, dz, f * ks, fd * ks, f2 * ks, bi);
      } else {
        shell_lap_store<Real, true>(si.y, dx, dy, dz, f * kc, fd * kc, f2 * kc, br);
        if (ks != 0.0) shell_lap_store<Real, true>(si.y, dx, dy, dz, f * ks, fd * ks, f2 * ks, bi);
      }
    }
    for (int k = 0; k < nf && !S.cutoff_mo; k++) {
      const double vr = double(br[5 * k]), vi = double(bi[5 * k]);
      if (!(sqrt(vr * vr + vi * vi) > 1e-8))
        for (int c = 0; c < 5; c++) br[5 * k + c] = bi[5 * k + c] = Real(0);
    }
  }
  __syncwarp();
  for (int mo = lane; mo < M; mo += 32) {
    Real ar[5] = {Real(0), Real(0), Real(0), Real(0), Real(0)}, ai[5] = {Real(0), Real(0), Real(0), Real(0), Real(0)};
    for (int f = 0; f < S.nbasis; f++) {
      const Real cr = moc_re[(size_t)f * ms + mo], ci = moc_im[(size_t)f * ms + mo];
      const Real* b = bas + f * 5;
#pragma unroll
      for (int q = 0; q < 5; q++) {
        const Real xr = b[q], xi = b[nb5 + q];
        ar[q] += cr * xr - ci * xi;
        ai[q] += cr * xi + ci * xr;
      }
    }
#pragma unroll
    for (int q = 0; q < 5; q++) { out[mo * 5 + q] = ar[q]; out[5 * ms + mo * 5 + q] = ai[q]; }
  }
  __syncwarp();
}

// Determinant ratio of one electron moved to p, by the calling lane, with
// the projected coefficients w (complex, planar with imaginary plane at
// w_im): sum_f b_f(p) w_f over the k-phased image sums of every shell.
template <typename Real>
__device__ __forceinline__ void basis_dot_lane_cpx(const DevSys<Real>& S, double px, double py, double pz,
                                                   const Real* w_re, const Real* w_im, Real& out_re, Real& out_im) {
  Real acr = Real(0), aci = Real(0);
  const int sc = subcell_of(S, px, py, pz);
  for (int c = 0; c < S.natoms; c++) {
    const int4 cs = S.center_seg[c];  // first shell, shells, object base, splines per row
    if (cs.y == 0) continue;
    const ImgRange im = images_of(S, sc, c);
    const Real cut = Real(S.center_cut[c]);
    for (int k = 0; k < cs.y; k++) {
      const int pk = S.shell_pack[cs.x + k];
      const int sym = pk & 0xf, fb = (pk >> 4) & 0xffff, kk = (pk >> 20) & 0xff;
      // CUTOFF_MO: the shell's own cutoff and no |value| skip
      const Real scut = S.cutoff_mo ? Real(S.shell_cut[cs.x + k]) : cut;
      const Real scut2 = scut * scut * Real(1.000001);
      const Real tiny = S.cutoff_mo ? Real(-1) : Real(1e-8);
      if (sym >= 4) {
        // F and G shells: one function at a time over the images
        for (int q = 0; q < sym_nfunc(sym); q++) {
          const int idx = fg_index(sym, q);
          Real gr = Real(0), gi = Real(0);
          for (int t = 0; t < im.count; t++) {
            const int m = im[t];
            const double* cp = S.image_pos + 3 * m;
            const Real x = Real(px - cp[0]), y = Real(py - cp[1]), z = Real(pz - cp[2]);
            const Real rd2 = x * x + y * y + z * z;
            if (!(rd2 < scut2)) continue;
            const Real rd = sqrt(rd2);
            if (!(rd < scut)) continue;
            const int i = int(rd * Real(S.inv_spacing));
            const Real h = rd - Real(i) * Real(S.spacing);
            const Real* cf = S.spline + ((size_t)cs.z + (size_t)i * cs.w) * 4 + 4 * kk;
            const Real f = spline_val(cf, h);
            const Real a = fg_value<Real>(idx, x, y, z) * f;
            gr += Real(S.image_kfac[2 * m]) * a;
            gi += Real(S.image_kfac[2 * m + 1]) * a;
          }
          if (sqrt(gr * gr + gi * gi) > tiny) {
            const Real wr = w_re[fb + q], wi = w_im[fb + q];
            acr += gr * wr - gi * wi;
            aci += gr * wi + gi * wr;
          }
        }
        continue;
      }
      Real fr[6] = {Real(0), Real(0), Real(0), Real(0), Real(0), Real(0)};
      Real fi[6] = {Real(0), Real(0), Real(0), Real(0), Real(0), Real(0)};
      for (int t = 0; t < im.count; t++) {
        const int m = im[t];
        const double* cp = S.image_pos + 3 * m;
        const Real x = Real(px - cp[0]), y = Real(py - cp[1]), z = Real(pz - cp[2]);
        const Real rd2 = x * x + y * y + z * z;
        if (!(rd2 < scut2)) continue;
        const Real rd = sqrt(rd2);
        if (!(rd < scut)) continue;
        const int i = int(rd * Real(S.inv_spacing));
        const Real h = rd - Real(i) * Real(S.spacing);
        const Real* cf = S.spline + ((size_t)cs.z + (size_t)i * cs.w) * 4 + 4 * kk;
        const Real f = spline_val(cf, h);
        Real a[6];
        int n;
        switch (sym) {
          case 0: a[0] = f; n = 1; break;
          case 1: a[0] = x * f; a[1] = y * f; a[2] = z * f; n = 3; break;
          case 2:
            a[0] = x * x * f; a[1] = y * y * f; a[2] = z * z * f; a[3] = x * y * f; a[4] = x * z * f; a[5] = y * z * f;
            n = 6;
            break;
          default:
            a[0] = (Real(2) * z * z - x * x - y * y) * f; a[1] = x * z * f; a[2] = y * z * f;
            a[3] = (x * x - y * y) * f; a[4] = x * y * f; n = 5;
            break;
        }
        const Real kc = Real(S.image_kfac[2 * m]), ks = Real(S.image_kfac[2 * m + 1]);
#pragma unroll
        for (int q = 0; q < 6; q++)
          if (q < n) { fr[q] += kc * a[q]; fi[q] += ks * a[q]; }
      }
      const int n = sym_nfunc(sym);
#pragma unroll
      for (int q = 0; q < 6; q++)
        if (q < n && sqrt(fr[q] * fr[q] + fi[q] * fi[q]) > tiny) {
          const Real wr = w_re[fb + q], wi = w_im[fb + q];
          acr += fr[q] * wr - fi[q] * wi;
          aci += fr[q] * wi + fi[q] * wr;
        }
    }
  }
  out_re = acr;
  out_im = aci;
}

// ---------------------------------------------------------------------------
// Jastrow pieces (tables from the parameter bank; sums in double)

// Two-body u(r) for a pair of given spins: value, f'/r, lap (precision T).
template <typename T, typename Real>
__device__ __forceinline__ void jas_pair_t(const DevSys<Real>& S, bool same, T r, double& u, double& fd, double& lap) {
  T uu = T(0), ff = T(0), ll = T(0);
  for (int k = 0; k < S.nee; k++) {
    const double c = same ? S.ee_like[k] : S.ee_unlike[k];
    if (c == 0.0) continue;
    T f, d, l;
    radial_lap<T>(S.ee[k], r, f, d, l);
    uu += T(c) * f; ff += T(c) * d; ll += T(c) * l;
  }
  u = double(uu); fd = double(ff); lap = double(ll);
}

// One-body sum over atoms for an electron at p: value, gradient, lap.
template <typename Real>
__device__ __forceinline__ void jas_onebody(const DevSys<Real>& S, double px, double py, double pz, double& u,
                                            double g[3], double& lap) {
  u = 0; g[0] = g[1] = g[2] = 0; lap = 0;
  for (int a = 0; a < S.natoms; a++) {
    const int t = S.atom_type[a];
    const double* ap = S.atom_pos[a];
    double dx = px - ap[0], dy = py - ap[1], dz = pz - ap[2];
    min_image(S, dx, dy, dz);
    double r = sqrt(dx * dx + dy * dy + dz * dz);
    for (int k = 0; k < S.ei_n[t]; k++) {
      double c = S.onebody[t][k];
      if (c == 0.0) continue;
      double f, d, l;
      radial_lap(S.ei[t][k], r, f, d, l);
      u += c * f; g[0] += c * d * dx; g[1] += c * d * dy; g[2] += c * d * dz; lap += c * l;
    }
  }
}

// Atoms whose e-e-n terms can be nonzero for an electron at p: the e-i
// radial functions vanish (value and derivatives) at and beyond their
// cutoff, so an atom farther than tb_rc (the largest cutoff its e-e-n terms
// use) from either electron of a pair contributes exactly zero.  Computed
// once per position; n < 0 means more than QWG_NEAR atoms are in range and
// the callers fall back to every atom.
constexpr int QWG_NEAR = 12;
struct NearSet {
  int n;
  int a[QWG_NEAR];
  double d[QWG_NEAR][3];  // p - atom, minimum image
  double r[QWG_NEAR];
};

template <typename Real>
__device__ __forceinline__ void near_atoms(const DevSys<Real>& S, const double p[3], NearSet& ns) {
  ns.n = 0;
  for (int a = 0; a < S.natoms; a++) {
    const int t = S.atom_type[a];
    if (!S.tb_n[t]) continue;
    double dx = p[0] - S.atom_pos[a][0], dy = p[1] - S.atom_pos[a][1], dz = p[2] - S.atom_pos[a][2];
    min_image(S, dx, dy, dz);
    const double r = sqrt(dx * dx + dy * dy + dz * dz);
    if (!(r < S.tb_rc[t])) continue;
    if (ns.n == QWG_NEAR) { ns.n = -1; return; }
    ns.a[ns.n] = a;
    ns.d[ns.n][0] = dx; ns.d[ns.n][1] = dy; ns.d[ns.n][2] = dz;
    ns.r[ns.n] = r;
    ns.n++;
  }
}

// e-e-n terms of the pair (i, j) at one atom of type t (Jastrow2_three.cpp:
// 138-404; THREEBODY_SPIN, Jastrow2_three_diffspin.cpp:233-330, picks the
// coefficient by the pair's spins): sum_terms c (a_k(i) a_l(j) + a_l(i) a_k(j))
// b_m(r_ij), with gradients/laps for both electrons.
template <typename Real>
__device__ __forceinline__ void tb_atom(const DevSys<Real>& S, int t, bool same, const double di[3], double ri,
                                        const double dj[3], double rj, const double dij[3], double rij, double& u,
                                        double gi[3], double& li, double gj[3], double& lj, bool need_derivs) {
  const int nt = S.tb_n[t];
  for (int n = 0; n < nt; n++) {
    const DTB& q0 = S.tb[t][n];
    struct { int k, l, m; double c; } q{q0.k, q0.l, q0.m, same ? q0.c : q0.cu};
    double aki, akdi, akli, akj, akdj, aklj, ali, aldi, alli, alj, aldj, allj, b, bd, bl;
    radial_lap(S.ei[t][q.k], ri, aki, akdi, akli);
    radial_lap(S.ei[t][q.k], rj, akj, akdj, aklj);
    radial_lap(S.ei[t][q.l], ri, ali, aldi, alli);
    radial_lap(S.ei[t][q.l], rj, alj, aldj, allj);
    radial_lap(S.ee[q.m], rij, b, bd, bl);
    double s = aki * alj + ali * akj;
    u += q.c * s * b;
    if (!need_derivs) continue;
    double gsi[3], gsj[3], gb[3];
    double dsi = 0, dsj = 0;
    for (int d = 0; d < 3; d++) {
      gsi[d] = akdi * di[d] * alj + aldi * di[d] * akj;
      gsj[d] = aki * aldj * dj[d] + ali * akdj * dj[d];
      gb[d] = bd * dij[d];
      dsi += gsi[d] * gb[d];
      dsj += gsj[d] * gb[d];
    }
    for (int d = 0; d < 3; d++) {
      gi[d] += q.c * (gsi[d] * b + s * gb[d]);
      gj[d] += q.c * (gsj[d] * b - s * gb[d]);
    }
    li += q.c * ((akli * alj + alli * akj) * b + s * bl + 2 * dsi);
    lj += q.c * ((aki * allj + ali * aklj) * b + s * bl - 2 * dsj);
  }
}

// Three-body (e-e-n) contribution of the pair (i, j) summed over the atoms
// (ns: the atoms in range of electron i, from near_atoms at pi; same: the
// two electrons have equal spin).
// pie: the position whose e-n basis values electron i uses (pi except for
// the stale-basis value path, DevSys::tb_stale_ei); ns was built at pie.
template <typename Real>
__device__ void jas_threebody_pair(const DevSys<Real>& S, const NearSet& ns, bool same, const double pi[3],
                                   const double pj[3], double& u, double gi[3], double& li, double gj[3], double& lj,
                                   bool need_derivs, const double* pie = nullptr) {
  u = 0; li = lj = 0;
  for (int d = 0; d < 3; d++) gi[d] = gj[d] = 0;
  if (ns.n == 0) return;
  if (!pie) pie = pi;
  double dij[3] = {pi[0] - pj[0], pi[1] - pj[1], pi[2] - pj[2]};
  min_image(S, dij[0], dij[1], dij[2]);
  const double rij = sqrt(dij[0] * dij[0] + dij[1] * dij[1] + dij[2] * dij[2]);
  const int cnt = ns.n < 0 ? S.natoms : ns.n;
  for (int q = 0; q < cnt; q++) {
    const int a = ns.n < 0 ? q : ns.a[q];
    const int t = S.atom_type[a];
    if (!S.tb_n[t]) continue;
    const double* ap = S.atom_pos[a];
    double di[3], ri;
    if (ns.n < 0) {
      di[0] = pie[0] - ap[0]; di[1] = pie[1] - ap[1]; di[2] = pie[2] - ap[2];
      min_image(S, di[0], di[1], di[2]);
      ri = sqrt(di[0] * di[0] + di[1] * di[1] + di[2] * di[2]);
    } else {
      di[0] = ns.d[q][0]; di[1] = ns.d[q][1]; di[2] = ns.d[q][2];
      ri = ns.r[q];
    }
    double dj[3] = {pj[0] - ap[0], pj[1] - ap[1], pj[2] - ap[2]};
    min_image(S, dj[0], dj[1], dj[2]);
    const double rj = sqrt(dj[0] * dj[0] + dj[1] * dj[1] + dj[2] * dj[2]);
    if (!(rj < S.tb_rc[t]) || !(ri < S.tb_rc[t])) continue;  // every term vanishes
    tb_atom(S, t, same, di, ri, dj, rj, dij, rij, u, gi, li, gj, lj, need_derivs);
  }
}

// e-e-n terms of the pair (e, j) before (old position) and after (new
// position) a move of e, in one pass over the atoms in range of either
// position: electron j's radials serve both positions, and each position's
// radials are taken once per atom and function.  dn / dq: new / old position
// minus r_j (minimum image), rn / rq their lengths.  Adds U_new - U_old to du,
// the new position's gradient and Laplacian terms to gi / li, and the change
// of electron j's to dgj / dlj (the sums of tb_atom over both near sets).
// Near sets that overflowed are not handled here (callers use
// jas_threebody_pair for them).
template <typename Real>
__device__ void tb_pair_move(const DevSys<Real>& S, const NearSet& nsn, const NearSet& nso, bool same,
                             const double pj[3], const double dn[3], double rn, const double dq[3], double rq,
                             double& du, double gi[3], double& li, double dgj[3], double& dlj) {
  int qn = 0, qo = 0;
  while (qn < nsn.n || qo < nso.n) {
    const int an = qn < nsn.n ? nsn.a[qn] : S.natoms, ao = qo < nso.n ? nso.a[qo] : S.natoms;
    const int a = min(an, ao);
    const bool hn = an == a, ho = ao == a;
    const int t = S.atom_type[a];
    const double* ap = S.atom_pos[a];
    double dj[3] = {pj[0] - ap[0], pj[1] - ap[1], pj[2] - ap[2]};
    min_image(S, dj[0], dj[1], dj[2]);
    const double rj = sqrt(dj[0] * dj[0] + dj[1] * dj[1] + dj[2] * dj[2]);
    if (rj < S.tb_rc[t]) {
      const int ne = S.ei_n[t];
      double fj[QWG_MAXEI], fdj[QWG_MAXEI], flj[QWG_MAXEI];
      for (int k = 0; k < ne; k++) radial_lap(S.ei[t][k], rj, fj[k], fdj[k], flj[k]);
      for (int side = 0; side < 2; side++) {
        if (side == 0 ? !hn : !ho) continue;
        const NearSet& ns = side == 0 ? nsn : nso;
        const int q = side == 0 ? qn : qo;
        const double* di = ns.d[q];
        const double ri = ns.r[q];
        const double* dij = side == 0 ? dn : dq;
        const double rij = side == 0 ? rn : rq;
        const double sg = side == 0 ? 1.0 : -1.0;
        double fi[QWG_MAXEI], fdi[QWG_MAXEI], fli[QWG_MAXEI];
        for (int k = 0; k < ne; k++) radial_lap(S.ei[t][k], ri, fi[k], fdi[k], fli[k]);
        for (int n = 0; n < S.tb_n[t]; n++) {
          const DTB& q0 = S.tb[t][n];
          const int k = q0.k, l = q0.l;
          const double c = same ? q0.c : q0.cu;
          double b, bd, bl;
          radial_lap(S.ee[q0.m], rij, b, bd, bl);
          const double sv = fi[k] * fj[l] + fi[l] * fj[k];
          du += sg * c * sv * b;
          double dsi = 0, dsj = 0, gsi[3], gsj[3], gb[3];
          for (int d = 0; d < 3; d++) {
            gsi[d] = fdi[k] * di[d] * fj[l] + fdi[l] * di[d] * fj[k];
            gsj[d] = fi[k] * fdj[l] * dj[d] + fi[l] * fdj[k] * dj[d];
            gb[d] = bd * dij[d];
            dsi += gsi[d] * gb[d];
            dsj += gsj[d] * gb[d];
          }
          if (side == 0) {
            for (int d = 0; d < 3; d++) gi[d] += c * (gsi[d] * b + sv * gb[d]);
            li += c * ((fli[k] * fj[l] + fli[l] * fj[k]) * b + sv * bl + 2 * dsi);
          }
          for (int d = 0; d < 3; d++) dgj[d] += sg * c * (gsj[d] * b - sv * gb[d]);
          dlj += sg * c * ((fi[k] * flj[l] + fi[l] * flj[k]) * b + sv * bl - 2 * dsj);
        }
      }
    }
    if (hn) qn++;
    if (ho) qo++;
  }
}

// Everything of the Jastrow exponent that depends on electron i placed at p
// (others at R): value U_i (one-body + all pairs with i), gradient, lap.
template <bool TB, typename Real>
__device__ void jas_electron(const DevSys<Real>& S, const double* R, int i, double px, double py, double pz,
                             double& u, double g[3], double& lap, bool need_derivs) {
  double ob, og[3], ol;
  jas_onebody(S, px, py, pz, ob, og, ol);
  u = ob; lap = ol;
  for (int d = 0; d < 3; d++) g[d] = og[d];
  const bool si = i < S.nup;
  const double pi[3] = {px, py, pz};
  NearSet ns;
  if constexpr (TB) near_atoms(S, pi, ns);
  for (int j = 0; j < S.nelec; j++) {
    if (j == i) continue;
    double dx = px - R[3 * j], dy = py - R[3 * j + 1], dz = pz - R[3 * j + 2];
    min_image(S, dx, dy, dz);
    const double r2 = dx * dx + dy * dy + dz * dz;
    if (!(r2 < S.ee_rc2)) continue;  // beyond every e-e cutoff: no pair term
    double r = sqrt(r2);
    double pu, pfd, pl;
    jas_pair_t<double>(S, si == (j < S.nup), r, pu, pfd, pl);
    u += pu; lap += pl;
    g[0] += pfd * dx; g[1] += pfd * dy; g[2] += pfd * dz;
    if constexpr (TB) {  // e-e-n terms compiled in only when the deck has them
      double tu, tgi[3], tli, tgj[3], tlj;
      jas_threebody_pair(S, ns, si == (j < S.nup), pi, R + 3 * j, tu, tgi, tli, tgj, tlj, need_derivs);
      u += tu; lap += tli;
      for (int d = 0; d < 3; d++) g[d] += tgi[d];
    }
  }
}

// Value-only version of jas_electron (the pseudopotential quadrature points),
// in the working precision T (float on the mixed path): differences of the
// FP64 positions are taken first, then everything runs in T.
template <typename T, bool TB, typename Real>
__device__ T jas_electron_val(const DevSys<Real>& S, const double* R, int i, double px, double py, double pz) {
  T u = T(0);
  for (int a = 0; a < S.natoms; a++) {
    const int t = S.atom_type[a];
    const double* ap = S.atom_pos[a];
    double ex = px - ap[0], ey = py - ap[1], ez = pz - ap[2];
    min_image(S, ex, ey, ez);
    const T dx = T(ex), dy = T(ey), dz = T(ez);
    const T r = sqrt(dx * dx + dy * dy + dz * dz);
    for (int k = 0; k < S.ei_n[t]; k++) {
      const double c = S.onebody[t][k];
      if (c != 0.0) u += T(c) * radial_val<T>(S.ei[t][k], r);
    }
  }
  const bool si = i < S.nup;
  const double pi[3] = {px, py, pz};
  const double* pie = S.tb_stale_ei ? R + 3 * i : pi;  // e-n position of the e-e-n terms
  NearSet ns;
  // e-e-n: the e-n values of electron i at its atoms in range, once per
  // point instead of once per pair (a near set that overflowed takes the
  // general pair routine)
  T av[TB ? QWG_NEAR : 1][QWG_MAXEI];
  if constexpr (TB) {
    near_atoms(S, pie, ns);
    for (int q = 0; q < ns.n; q++) {
      const int t = S.atom_type[ns.a[q]];
      for (int k = 0; k < S.ei_n[t]; k++) av[q][k] = radial_val<T>(S.ei[t][k], T(ns.r[q]));
    }
  }
  for (int j = 0; j < S.nelec; j++) {
    if (j == i) continue;
    double ex = px - R[3 * j], ey = py - R[3 * j + 1], ez = pz - R[3 * j + 2];
    min_image(S, ex, ey, ez);
    const T dx = T(ex), dy = T(ey), dz = T(ez);
    const T r2 = dx * dx + dy * dy + dz * dz;
    if (!(r2 < T(S.ee_rc2))) continue;  // beyond every e-e cutoff: no pair term
    const T r = sqrt(r2);
    const bool same = si == (j < S.nup);
    for (int k = 0; k < S.nee; k++) {
      const double c = same ? S.ee_like[k] : S.ee_unlike[k];
      if (c != 0.0) u += T(c) * radial_val<T>(S.ee[k], r);
    }
    if constexpr (TB) {
      if (ns.n < 0) {
        double tu, tgi[3], tli, tgj[3], tlj;
        jas_threebody_pair(S, ns, same, pi, R + 3 * j, tu, tgi, tli, tgj, tlj, false, pie);
        u += T(tu);
      } else {
        // sum over the atoms of c (a_k(i) a_l(j) + a_l(i) a_k(j)) b_m(r_ij)
        // (the terms of tb_atom, values only)
        for (int q = 0; q < ns.n; q++) {
          const int a = ns.a[q], t = S.atom_type[a];
          const double* ap = S.atom_pos[a];
          double jx = R[3 * j] - ap[0], jy = R[3 * j + 1] - ap[1], jz = R[3 * j + 2] - ap[2];
          min_image(S, jx, jy, jz);
          const T rj = T(sqrt(jx * jx + jy * jy + jz * jz));
          if (!(rj < T(S.tb_rc[t]))) continue;  // every term vanishes
          T aj[QWG_MAXEI];
          for (int k = 0; k < S.ei_n[t]; k++) aj[k] = radial_val<T>(S.ei[t][k], rj);
          for (int n = 0; n < S.tb_n[t]; n++) {
            const DTB& tq = S.tb[t][n];
            const T c = T(same ? tq.c : tq.cu);
            u += c * (av[q][tq.k] * aj[tq.l] + av[q][tq.l] * aj[tq.k]) * radial_val<T>(S.ee[tq.m], r);
          }
        }
      }
    }
  }
  return u;
}

// ---------------------------------------------------------------------------
// dense linear algebra in the warp

// Gauss-Jordan inversion with partial pivoting for any M (the matrix lives in
// HBM-resident scratch): lanes over columns; the pivot column is copied to
// fcol[M] before each elimination so that no lane reads a factor another lane
// is updating.  Same pivot rule, log|det| and sign as gj_inverse_warp.
template <typename Real>
__device__ void gj_inverse_warp_big(double* aug, double* fcol, int M, Real* invT, int invstride, double& logdet,
                                    double& sign, int lane) {
  const int W = 2 * M;
  for (int idx = lane; idx < M * M; idx += 32) {
    int i = idx / M, k = idx - i * M;
    aug[i * W + M + k] = (i == k) ? 1.0 : 0.0;
  }
  __syncwarp();
  double ld = 0.0, sg = 1.0;
  bool singular = false;
  for (int k = 0; k < M; k++) {
    double best = -1.0;
    int bi = k;
    for (int i = k + lane; i < M; i += 32) {
      double v = fabs(aug[i * W + k]);
      if (v > best) { best = v; bi = i; }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      double ob = __shfl_xor_sync(0xffffffffu, best, o);
      int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
    }
    if (!(best > 0.0)) { singular = true; break; }
    if (bi != k) {
      for (int c = lane; c < W; c += 32) {
        double t = aug[k * W + c];
        aug[k * W + c] = aug[bi * W + c];
        aug[bi * W + c] = t;
      }
      sg = -sg;
    }
    __syncwarp();
    const double piv = aug[k * W + k];
    ld += log(fabs(piv));
    if (piv < 0) sg = -sg;
    const double inv = 1.0 / piv;
    __syncwarp();
    for (int c = lane; c < W; c += 32) aug[k * W + c] *= inv;
    for (int i = lane; i < M; i += 32) fcol[i] = aug[i * W + k];
    __syncwarp();
    // columns k+1.. of the left half and the whole right half change; column k
    // becomes the unit vector
    for (int c = lane; c < W; c += 32) {
      if (c < k) continue;
      const double pk = aug[k * W + c];
      if (c == k) {
        for (int i = 0; i < M; i++)
          if (i != k) aug[i * W + c] = 0.0;
      } else {
        for (int i = 0; i < M; i++)
          if (i != k) aug[i * W + c] -= fcol[i] * pk;
      }
    }
    __syncwarp();
  }
  if (singular) {
    ld = -1e201;
    for (int idx = lane; idx < M * M; idx += 32) {
      int e = idx / M, i = idx - e * M;
      invT[e * invstride + i] = Real(0);
    }
  } else {
    for (int idx = lane; idx < M * M; idx += 32) {
      int e = idx / M, i = idx - e * M;
      invT[e * invstride + i] = Real(aug[i * W + M + e]);
    }
  }
  __syncwarp();
  logdet = ld;
  sign = sg;
}

// Gauss-Jordan inversion with partial pivoting of A (M x M, M <= 32, row-major,
// A[e][i] = phi_i(r_e)) held in aug[M][2M] (double).  Writes the transposed
// inverse invT[e][i] = (A^-1)[i][e] and returns log|det A| and its sign.
// Singular: logdet = -1e201 (the log of an exact zero determinant).
template <typename Real>
__device__ void gj_inverse_warp(double* aug, int M, Real* invT, int invstride, double& logdet, double& sign, int lane) {
  const int W = 2 * M;
  for (int idx = lane; idx < M * M; idx += 32) {
    int i = idx / M, k = idx - i * M;
    aug[i * W + M + k] = (i == k) ? 1.0 : 0.0;
  }
  __syncwarp();
  double ld = 0.0, sg = 1.0;
  bool singular = false;
  for (int k = 0; k < M; k++) {
    // pivot search over rows k..M-1 (lane i looks at row i)
    double best = -1.0;
    int bi = k;
    for (int i = k + lane; i < M; i += 32) {
      double v = fabs(aug[i * W + k]);
      if (v > best) { best = v; bi = i; }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      double ob = __shfl_xor_sync(0xffffffffu, best, o);
      int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
    }
    if (!(best > 0.0)) { singular = true; break; }
    if (bi != k) {
      for (int c = lane; c < W; c += 32) {
        double t = aug[k * W + c];
        aug[k * W + c] = aug[bi * W + c];
        aug[bi * W + c] = t;
      }
      sg = -sg;
    }
    __syncwarp();
    double piv = aug[k * W + k];
    ld += log(fabs(piv));
    if (piv < 0) sg = -sg;
    double inv = 1.0 / piv;
    __syncwarp();
    for (int c = lane; c < W; c += 32) aug[k * W + c] *= inv;
    __syncwarp();
    // factors of every row in column k (lane i holds row i), captured
    // before the update; lane c owns columns c and c + 32 (W <= 64)
    double fac = (lane < M) ? aug[lane * W + k] : 0.0;
    double pk0 = (lane < W) ? aug[k * W + lane] : 0.0;
    double pk1 = (lane + 32 < W) ? aug[k * W + lane + 32] : 0.0;
    __syncwarp();
    for (int i = 0; i < M; i++) {
      double f = __shfl_sync(0xffffffffu, fac, i);
      if (i == k) continue;
      if (lane < W) aug[i * W + lane] -= f * pk0;
      if (lane + 32 < W) aug[i * W + lane + 32] -= f * pk1;
    }
    __syncwarp();
  }
  if (singular) {
    ld = -1e201;
    for (int idx = lane; idx < M * M; idx += 32) {
      int e = idx / M, i = idx - e * M;
      invT[e * invstride + i] = Real(0);
    }
  } else {
    for (int idx = lane; idx < M * M; idx += 32) {
      int e = idx / M, i = idx - e * M;
      invT[e * invstride + i] = Real(aug[i * W + M + e]);
    }
  }
  __syncwarp();
  logdet = ld;
  sign = sg;
}

// Complex Gauss-Jordan inversion with partial pivoting on the modulus (the
// complex counterpart of gj_inverse_warp_big, TransposeInverseMatrix for
// dcomplex, MatrixAlgebrac.cpp:316-421): aug holds the real plane [M][2M],
// then the imaginary plane [M][2M], then the pivot column (real M, imaginary
// M).  Writes the transposed inverse (planar, imaginary plane at inv_im) and
// returns log|det A| and arg det A.
template <typename Real>
__device__ void gj_inverse_warp_cpx(double* aug, int M, Real* inv_re, Real* inv_im, int invstride, double& logdet,
                                    double& phase, int lane) {
  const int W = 2 * M;
  double* ar = aug;
  double* ai = aug + (size_t)M * W;
  double* fr = ai + (size_t)M * W;
  double* fi = fr + M;
  for (int idx = lane; idx < M * M; idx += 32) {
    int i = idx / M, k = idx - i * M;
    ar[i * W + M + k] = (i == k) ? 1.0 : 0.0;
    ai[i * W + M + k] = 0.0;
  }
  __syncwarp();
  double ld = 0.0, ph = 0.0;
  bool singular = false;
  for (int k = 0; k < M; k++) {
    double best = -1.0;
    int bi = k;
    for (int i = k + lane; i < M; i += 32) {
      const double v = hypot(ar[i * W + k], ai[i * W + k]);
      if (v > best) { best = v; bi = i; }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      double ob = __shfl_xor_sync(0xffffffffu, best, o);
      int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
    }
    if (!(best > 0.0)) { singular = true; break; }
    if (bi != k) {
      for (int c = lane; c < W; c += 32) {
        double t = ar[k * W + c]; ar[k * W + c] = ar[bi * W + c]; ar[bi * W + c] = t;
        t = ai[k * W + c]; ai[k * W + c] = ai[bi * W + c]; ai[bi * W + c] = t;
      }
      ph += CUDART_PI;
    }
    __syncwarp();
    const double pr = ar[k * W + k], pi = ai[k * W + k];
    const double m2 = pr * pr + pi * pi;
    ld += 0.5 * log(m2);
    ph += atan2(pi, pr);
    const double qr = pr / m2, qi = -pi / m2;  // 1 / pivot
    __syncwarp();
    for (int c = lane; c < W; c += 32) {
      const double xr = ar[k * W + c], xi = ai[k * W + c];
      ar[k * W + c] = xr * qr - xi * qi;
      ai[k * W + c] = xr * qi + xi * qr;
    }
    for (int i = lane; i < M; i += 32) { fr[i] = ar[i * W + k]; fi[i] = ai[i * W + k]; }
    __syncwarp();
    for (int c = lane; c < W; c += 32) {
      if (c < k) continue;
      const double pkr = ar[k * W + c], pki = ai[k * W + c];
      if (c == k) {
        for (int i = 0; i < M; i++)
          if (i != k) { ar[i * W + c] = 0.0; ai[i * W + c] = 0.0; }
      } else {
        for (int i = 0; i < M; i++)
          if (i != k) {
            ar[i * W + c] -= fr[i] * pkr - fi[i] * pki;
            ai[i * W + c] -= fr[i] * pki + fi[i] * pkr;
          }
      }
    }
    __syncwarp();
  }
  for (int idx = lane; idx < M * M; idx += 32) {
    int e = idx / M, i = idx - e * M;
    inv_re[e * invstride + i] = singular ? Real(0) : Real(ar[i * W + M + e]);
    inv_im[e * invstride + i] = singular ? Real(0) : Real(ai[i * W + M + e]);
  }
  __syncwarp();
  logdet = singular ? -1e201 : ld;
  phase = ph;
}

}  // namespace qwg
