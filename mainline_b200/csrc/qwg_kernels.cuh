// Walker kernels: full evaluation, single-electron ratio, VMC/DMC steps,
// branching and population gather.  See qwg_device.cuh for the execution
// model.  Reference semantics cited per routine (QWalk/mainline src/).
#pragma once
#include "qwg_device.cuh"
#include "qwg_tc.cuh"

namespace qwg {

// KM_STEPS runs whole steps (moves + local energy + weight) in one launch;
// KM_SWEEP and KM_ELOC split one step into its two phases (the electron
// moves; the local energy and weight), one launch each, with the same
// arithmetic and random streams, so the two schedules give identical walks.
// KM_TMOVE applies the T-moves the local-energy kernel selected.
// KM_ELOC_TM is KM_ELOC with the T-move selection compiled in.
enum KMode { KM_EVAL = 0, KM_RATIO = 1, KM_STEPS = 2, KM_SWEEP = 3, KM_ELOC = 4, KM_TMOVE = 5, KM_ELOC_TM = 6 };

struct EvalIO {
  const double* rot;     // [W][9] quadrature rotations (KM_EVAL) or nullptr
  const int* move_e;     // [W] (KM_RATIO)
  const double* move_r;  // [W][3]
  double* logpsi;        // [W]
  double* sign;          // [W]
  double* grad;          // [W][N][3] (KM_EVAL) or [W][3] (KM_RATIO)
  double* lap;           // [W][N] or [W]
  double* kinetic;       // [W]
  double* potential;     // [W]
  double* nonlocal;      // [W]
  double* energy;        // [W] local energy after the last step (KM_STEPS)
};

struct PPItem {
  int e, a;
  double r;
  double dx, dy, dz;     // electron - atom
  double vl[4];          // nonlocal channel radials (already scaled)
};

// MMAX > 0: at most MMAX orbitals per spin, state + scratch in shared
// memory.  MMAX == 0: any count up to 256 per spin, arrays strided by
// L.mstride and worked on in place in HBM.  MMAX == -1 (QWG_MM_CPX): the
// HBM-resident layout with complex orbitals (Slat_wf<dcomplex>): inverse,
// MO rows, basis rows and projected coefficients are planar complex arrays.
// PER: 0 molecule, 1 periodic cell, 2 either (decided at run time); the
// local-energy kernels are compiled per case, the others check at run time.
// XL: the F/G-shell and CUTOFF_MO code (HBM-resident kernels; the FP32 ones
// are also compiled without it for the decks that need none, as that code's
// register demand costs the move kernel ~5% in spills).
template <typename Real, int MMAX, bool TB, int PER, bool XL = (MMAX <= 0)>
struct Walker {
  const DevSys<Real>& S;
  const WLayout& L;
  unsigned char* base;   // persistent state
  unsigned char* sbase;  // scratch
  const Real* moc_s;     // [2][nbasis][mstride] MO coefficients (global, read through L1)
  int lane;
  // MO column of the proposal from the tensor-core GEMM (tc_phase 2):
  // tcD[(row0 + q) * tc_ldd + i] = component q of orbital i
  const float* tcD = nullptr;
  int tc_ldd = 0;
  unsigned long long* ph = nullptr;  // phase counters (profiling builds)
  static constexpr bool CPX = MMAX < 0;
  // F and G basis shells and CUTOFF_MO: compiled into the HBM-resident kernels only
  static constexpr bool HL = MMAX < 0 || (MMAX == 0 && XL);
  double cr_re = 0.0, cr_im = 0.0;  // complex determinant ratio of the last proposal (CPX)

  __device__ __forceinline__ int MS() const {
    if constexpr (MMAX > 0) return MMAX;
    else return L.mstride;
  }
  __device__ double* R() const { return (double*)(base + L.R); }
  __device__ Real* inv(int s) const {
    if constexpr (MMAX > 0) return (Real*)(base + L.inv) + (size_t)s * MS() * MS();
    else if constexpr (CPX) return (Real*)(base + L.inv) + (size_t)s * 2 * MS() * MS();  // + MS()^2: imaginary
    else return (Real*)(base + L.inv) + (size_t)s * L.nud * MS() * MS();
  }
  // ---- determinant expansions (HBM-resident kernels, S.ndet > 1)
  __device__ bool multi() const {
    if constexpr (MMAX != 0) return false;
    else return S.ndet > 1;
  }
  __device__ Real* inv_u(int s, int u) const { return (Real*)(base + L.inv) + ((size_t)s * L.nud + u) * MS() * MS(); }
  __device__ double* udl() const { return (double*)(base + L.udl); }
  __device__ double* mdt() const { return (double*)(base + L.mdt); }
  __device__ double* mdv() const { return (double*)(sbase + L.mdv); }
  __device__ double* mdr() const { return (double*)(sbase + L.mdr); }
  __device__ const int* cols(int s, int u) const { return S.ud_cols + ((size_t)s * QWG_MAXUD + u) * MS(); }
  // t_k = c_k sign_k exp(L_k - Lref) with L_k = log|D_up| + log|D_down|;
  // W = sum_k t_k (psi_D = W exp(Lref)); T[s][u] = sum of t_k over the
  // determinants whose spin-s factor is u.  mdt = [t_0..t_K-1, W, Lref, T[2][MAXUD]]
  __device__ void md_weights() {
    const double* ld = udl();
    double* t = mdt();
    const int K = S.ndet, nu = L.nud;
    double lref = -1e300;
    for (int k = 0; k < K; k++)
      lref = fmax(lref, ld[(0 * nu + S.det_ud[2 * k]) * 2] + ld[(1 * nu + S.det_ud[2 * k + 1]) * 2]);
    for (int k = lane; k < K; k += 32) {
      const int a = S.det_ud[2 * k], b = S.det_ud[2 * k + 1];
      const double lk = ld[(0 * nu + a) * 2] + ld[(1 * nu + b) * 2];
      t[k] = S.det_c[k] * ld[(0 * nu + a) * 2 + 1] * ld[(1 * nu + b) * 2 + 1] * exp(lk - lref);
    }
    __syncwarp();
    if (lane == 0) {
      double W = 0;
      double* T = t + QWG_MAXDET + 2;
      for (int q = 0; q < 2 * QWG_MAXUD; q++) T[q] = 0.0;
      for (int k = 0; k < K; k++) {
        W += t[k];
        T[S.det_ud[2 * k]] += t[k];
        T[QWG_MAXUD + S.det_ud[2 * k + 1]] += t[k];
      }
      t[QWG_MAXDET] = W;
      t[QWG_MAXDET + 1] = lref;
    }
    __syncwarp();
  }
  __device__ double md_logpsi_d(double& sign) const {
    const double W = mdt()[QWG_MAXDET];
    sign = W < 0 ? -1.0 : 1.0;
    return mdt()[QWG_MAXDET + 1] + log(fabs(W));
  }
  __device__ Real* mov() const { return (Real*)(base + L.mov); }
  __device__ double* gU() const { return (double*)(base + L.gU); }
  __device__ double* lU() const { return (double*)(base + L.lU); }
  __device__ WScal* sc() const { return (WScal*)(base + L.scal); }
  __device__ Real* bas() const { return (Real*)(sbase + L.bas); }
  __device__ Real* newcol() const { return (Real*)(sbase + L.newcol); }
  __device__ double* dG() const { return (double*)(sbase + L.dG); }
  __device__ double* Ue() const { return (double*)(sbase + L.Ue); }
  __device__ double* lu() const { return (double*)(sbase + L.lu); }
  __device__ PPItem* items() const { return (PPItem*)(sbase + L.items); }
  __device__ double* rot() const { return (double*)(sbase + L.rot); }
  __device__ Real* wproj() const { return (Real*)(sbase + L.wproj); }

  __device__ int spin(int e) const { return e < S.nup ? 0 : 1; }
  __device__ int eloc(int e) const { return e < S.nup ? e : e - S.nup; }
  __device__ const Real* mocs(int s) const { return moc_s + (size_t)s * S.nbasis * MS(); }
  __device__ const Real* mocs_im(int s) const { return S.moc_im + (size_t)s * S.nbasis * MS(); }
  // imaginary planes of the complex arrays (CPX)
  __device__ size_t mov_im_off() const { return (size_t)S.nelec * MS() * 4; }
  __device__ int newcol_im_off() const { return 5 * MS(); }
  __device__ int wproj_im_off() const { return L.wchunk * S.nbasis; }

  // Complex determinants (CPX): the recompute of both spins (Slat_wf<dcomplex>::
  // calcLap, Slat_wf.h:948-1016).
  __device__ void recompute_cpx() {
    double* Rp = R();
    Real* nc = newcol();
    double* aug = lu();
    WScal* w = sc();
    const int ms = MS();
    double phase = 0.0;
    for (int s = 0; s < 2; s++) {
      const int M = S.m[s];
      const int e0 = s == 0 ? 0 : S.nup;
      double* ar = aug;
      double* ai = aug + (size_t)2 * M * M;
      for (int el = 0; el < M; el++) {
        const int e = e0 + el;
        mo_lap_warp_cpx<Real>(S, mocs(s), mocs_im(s), Rp[3 * e], Rp[3 * e + 1], Rp[3 * e + 2], M, ms, bas(), nc, lane);
        for (int i = lane; i < M; i += 32) {
          ar[el * 2 * M + i] = double(nc[i * 5]);
          ai[el * 2 * M + i] = double(nc[newcol_im_off() + i * 5]);
          Real* mv = mov() + ((size_t)e * ms + i) * 4;
          Real* mw = mv + mov_im_off();
          for (int q = 0; q < 4; q++) { mv[q] = nc[i * 5 + 1 + q]; mw[q] = nc[newcol_im_off() + i * 5 + 1 + q]; }
        }
        __syncwarp();
      }
      double ld = 0.0, ph = 0.0;
      if (M > 0) gj_inverse_warp_cpx(aug, M, inv(s), inv(s) + (size_t)ms * ms, ms, ld, ph, lane);
      phase += ph;
      if (lane == 0) { w->logdet[s] = ld; w->sign[s] = 1.0; }
      __syncwarp();
    }
    if (lane == 0) w->phase = phase;
    __syncwarp();
  }

  // ---- full recompute: Slat_wf::calcLap (Slat_wf.h:948-1016) + the Jastrow
  // recomputation of every electron (Jastrow2_wf.cpp:988-1157).
  __device__ void recompute() {
    double* Rp = R();
    Real* nc = newcol();
    double* aug = lu();
    WScal* w = sc();
    if constexpr (CPX) recompute_cpx();
    for (int s = 0; s < 2 && multi(); s++) {
      // every orbital of the spin's union at every electron, then one
      // inversion per distinct spin-determinant (Slat_wf::calcLap for all
      // determinants, Slat_wf.h:948-1016)
      const int M = S.m[s], NU = S.nmo_u[s], ms = MS();
      const int e0 = s == 0 ? 0 : S.nup;
      double* vals = mdv();
      for (int el = 0; el < M; el++) {
        const int e = e0 + el;
        mo_lap_warp<Real, PER, HL>(S, mocs(s), Rp[3 * e], Rp[3 * e + 1], Rp[3 * e + 2], NU, bas(), nc, lane);
        for (int j = lane; j < NU; j += 32) {
          vals[(size_t)el * ms + j] = double(nc[j * 5]);
          Real* mv = mov() + ((size_t)e * ms + j) * 4;
          mv[0] = nc[j * 5 + 1]; mv[1] = nc[j * 5 + 2]; mv[2] = nc[j * 5 + 3]; mv[3] = nc[j * 5 + 4];
        }
        __syncwarp();
      }
      for (int u = 0; u < S.nud[s]; u++) {
        const int* cu = cols(s, u);
        for (int idx = lane; idx < M * M; idx += 32) {
          const int el = idx / M, i = idx - el * M;
          aug[el * 2 * M + i] = vals[(size_t)el * ms + cu[i]];
        }
        __syncwarp();
        double ld = 0.0, sg = 1.0;
        if (M > 0) gj_inverse_warp_big(aug, aug + 2 * M * M, M, inv_u(s, u), ms, ld, sg, lane);
        if (lane == 0) { udl()[((size_t)s * L.nud + u) * 2] = ld; udl()[((size_t)s * L.nud + u) * 2 + 1] = sg; }
        __syncwarp();
      }
      if (lane == 0) { w->logdet[s] = udl()[((size_t)s * L.nud) * 2]; w->sign[s] = udl()[((size_t)s * L.nud) * 2 + 1]; }
    }
    if (multi()) md_weights();
    for (int s = 0; s < 2 && !multi() && !CPX; s++) {
      const int M = S.m[s];
      const int e0 = s == 0 ? 0 : S.nup;
      for (int el = 0; el < M; el++) {
        const int e = e0 + el;
        mo_lap_warp<Real, PER, HL>(S, mocs(s), Rp[3 * e], Rp[3 * e + 1], Rp[3 * e + 2], M, bas(), nc, lane);
        for (int i = lane; i < M; i += 32) {
          aug[el * 2 * M + i] = double(nc[i * 5]);
          Real* mv = mov() + ((size_t)e * MS() + i) * 4;
          mv[0] = nc[i * 5 + 1]; mv[1] = nc[i * 5 + 2]; mv[2] = nc[i * 5 + 3]; mv[3] = nc[i * 5 + 4];
        }
        __syncwarp();
      }
      if (M > 0) {
        double ld, sg;
        if constexpr (MMAX > 0) gj_inverse_warp(aug, M, inv(s), MMAX, ld, sg, lane);
        else gj_inverse_warp_big(aug, aug + 2 * M * M, M, inv(s), MS(), ld, sg, lane);
        if (lane == 0) { w->logdet[s] = ld; w->sign[s] = sg; }
      } else if (lane == 0) {
        w->logdet[s] = 0.0; w->sign[s] = 1.0;
      }
      __syncwarp();
    }
    // Jastrow: every electron's gradient and Laplacian; U from the
    // one-body values and half the pair values.
    double usum = 0.0;
    for (int i = lane; i < S.nelec; i += 32) {
      double u, g[3], l, ob, og[3], ol;
      jas_electron<TB>(S, Rp, i, Rp[3 * i], Rp[3 * i + 1], Rp[3 * i + 2], u, g, l, true);
      jas_onebody(S, Rp[3 * i], Rp[3 * i + 1], Rp[3 * i + 2], ob, og, ol);
      gU()[3 * i] = g[0]; gU()[3 * i + 1] = g[1]; gU()[3 * i + 2] = g[2];
      lU()[i] = l;
      usum += 0.5 * (u + ob);
    }
    usum = warp_sum(usum);
    if (lane == 0) w->U = usum;
    __syncwarp();
  }

  // Slater gradient and Laplacian ratios of electron e at its position.
  __device__ void slater_gl(int e, double g[3], double& l) const {
    if (multi()) {
      // sum over distinct spin-determinants u of T[s][u] (grad D_u / D_u) / W
      const int s = spin(e), el = eloc(e), M = S.m[s], ms = MS();
      const double* T = mdt() + QWG_MAXDET + 2 + s * QWG_MAXUD;
      const double W = mdt()[QWG_MAXDET];
      const Real* mvb = mov() + (size_t)e * ms * 4;
      double b0 = 0, b1 = 0, b2 = 0, b3 = 0;
      for (int u = 0; u < S.nud[s]; u++) {
        const Real* iv = inv_u(s, u) + (size_t)el * ms;
        const int* cu = cols(s, u);
        double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
        for (int i = 0; i < M; i++) {
          const double c = iv[i];
          const Real* mv = mvb + 4 * cu[i];
          a0 += c * double(mv[0]); a1 += c * double(mv[1]); a2 += c * double(mv[2]); a3 += c * double(mv[3]);
        }
        b0 += T[u] * a0; b1 += T[u] * a1; b2 += T[u] * a2; b3 += T[u] * a3;
      }
      g[0] = b0 / W; g[1] = b1 / W; g[2] = b2 / W; l = b3 / W;
      return;
    }
    const int s = spin(e), el = eloc(e), M = S.m[s];
    const Real* iv = inv(s) + (size_t)el * MS();
    const Real* mv = mov() + (size_t)e * MS() * 4;
    if constexpr (CPX) {
      // real parts of grad D / D and lap D / D: the drift, and with the
      // Jastrow terms the kinetic energy -1/2 Re(lap psi / psi)
      // (System::calcKineticSeparated, System.cpp:105-140)
      const Real* ivi = iv + (size_t)MS() * MS();
      const Real* mvi = mv + mov_im_off();
      double b[4] = {0, 0, 0, 0};
      for (int i = 0; i < M; i++) {
        const double cr = iv[i], ci = ivi[i];
        for (int q = 0; q < 4; q++) b[q] += cr * double(mv[4 * i + q]) - ci * double(mvi[4 * i + q]);
      }
      g[0] = b[0]; g[1] = b[1]; g[2] = b[2]; l = b[3];
      return;
    }
    double a0 = 0, a1 = 0, a2 = 0, a3 = 0;  // FP64 accumulation of the short dots
    for (int i = 0; i < M; i++) {
      double c = iv[i];
      a0 += c * double(mv[4 * i]); a1 += c * double(mv[4 * i + 1]); a2 += c * double(mv[4 * i + 2]);
      a3 += c * double(mv[4 * i + 3]);
    }
    g[0] = a0; g[1] = a1; g[2] = a2; l = a3;
  }

  // ---- proposal of electron e at p: everything except the decision.
  // Fills the new MO column (newcol), the Jastrow deltas of the other
  // electrons (dG), and returns the determinant ratio, ln-ratio of the
  // Jastrow, new drift and lap of e.  (Slat_wf::updateLap + Jastrow2_wf::
  // updateLap + Slat_Jastrow::getLap for one electron.)
  __device__ void propose(int e, double px, double py, double pz, double& ratioD, double& dU, double gnew[3],
                          double& lapnew) {
    const int s = spin(e), el = eloc(e), M = S.m[s];
    const double* Rp = R();
    Real* nc = newcol();
    double r0 = 0, r1 = 0, r2 = 0, r3 = 0, r4 = 0;
    if (multi()) {
      // ratios of every distinct spin-determinant (kept in mdr for accept),
      // combined with the expansion weights
      mo_lap_warp<Real, PER, HL>(S, mocs(s), px, py, pz, S.nmo_u[s], bas(), nc, lane);
      double* rr = mdr();
      for (int u = lane; u < S.nud[s]; u += 32) {
        const Real* iv = inv_u(s, u) + (size_t)el * MS();
        const int* cu = cols(s, u);
        double a[5] = {0, 0, 0, 0, 0};
        for (int i = 0; i < M; i++) {
          const double c = iv[i];
          const Real* v = nc + 5 * cu[i];
          for (int q = 0; q < 5; q++) a[q] += c * double(v[q]);
        }
        for (int q = 0; q < 5; q++) rr[u * 5 + q] = a[q];
      }
      __syncwarp();
      const double* T = mdt() + QWG_MAXDET + 2 + s * QWG_MAXUD;
      const double W = mdt()[QWG_MAXDET];
      for (int u = 0; u < S.nud[s]; u++) {
        r0 += T[u] * rr[u * 5]; r1 += T[u] * rr[u * 5 + 1]; r2 += T[u] * rr[u * 5 + 2];
        r3 += T[u] * rr[u * 5 + 3]; r4 += T[u] * rr[u * 5 + 4];
      }
      r0 /= W; r1 /= W; r2 /= W; r3 /= W; r4 /= W;
    } else if constexpr (CPX) {
      // complex ratio R = sum_i invT[el][i] phi_i(p); |R| returned, R kept
      // for accept; drift and Laplacian from the real parts of the ratios
      mo_lap_warp_cpx<Real>(S, mocs(s), mocs_im(s), px, py, pz, M, MS(), bas(), nc, lane);
      const Real* iv = inv(s) + (size_t)el * MS();
      const Real* ivi = iv + (size_t)MS() * MS();
      const Real* nci = nc + newcol_im_off();
      double a[5] = {0, 0, 0, 0, 0}, b[5] = {0, 0, 0, 0, 0};
      for (int i = 0; i < M; i++) {
        const double cr = iv[i], ci = ivi[i];
        for (int q = 0; q < 5; q++) {
          const double xr = nc[i * 5 + q], xi = nci[i * 5 + q];
          a[q] += cr * xr - ci * xi;
          b[q] += cr * xi + ci * xr;
        }
      }
      cr_re = a[0]; cr_im = b[0];
      const double m2 = a[0] * a[0] + b[0] * b[0];
      r0 = sqrt(m2);
      // Re(x / R) = (Re x Re R + Im x Im R) / |R|^2, scaled by |R| for the
      // division below
      r1 = (a[1] * a[0] + b[1] * b[0]) / r0; r2 = (a[2] * a[0] + b[2] * b[0]) / r0;
      r3 = (a[3] * a[0] + b[3] * b[0]) / r0; r4 = (a[4] * a[0] + b[4] * b[0]) / r0;
    } else {
      QWG_PHASE_BEGIN(t_mo)
      bool from_gemm = false;
      if constexpr (MMAX == 0 && sizeof(Real) == 4) {
        if (tcD) {
          for (int idx = lane; idx < 5 * M; idx += 32) {
            const int i = idx / 5, q = idx - 5 * i;
            nc[idx] = Real(tcD[(size_t)q * tc_ldd + i]);
          }
          __syncwarp();
          from_gemm = true;
        }
      }
      if (!from_gemm) mo_lap_warp<Real, PER, HL>(S, mocs(s), px, py, pz, M, bas(), nc, lane);
      QWG_PHASE_END(t_mo, PH_MO, ph)
      const Real* iv = inv(s) + (size_t)el * MS();
      for (int i = 0; i < M; i++) {
        double c = iv[i];
        r0 += c * double(nc[i * 5]); r1 += c * double(nc[i * 5 + 1]); r2 += c * double(nc[i * 5 + 2]);
        r3 += c * double(nc[i * 5 + 3]); r4 += c * double(nc[i * 5 + 4]);
      }
    }
    QWG_PHASE_BEGIN(t_rest)
    ratioD = double(r0);
    double gD[3] = {double(r1) / ratioD, double(r2) / ratioD, double(r3) / ratioD};
    double lD = double(r4) / ratioD;
    // Jastrow: lanes over the other electrons
    const double ox = Rp[3 * e], oy = Rp[3 * e + 1], oz = Rp[3 * e + 2];
    const bool se = s == 0;
    constexpr bool has3 = TB;
    NearSet nsn, nso;  // atoms in e-e-n range of the new and the old position
    if constexpr (has3) {
      const double pn[3] = {px, py, pz}, po[3] = {ox, oy, oz};
      near_atoms(S, pn, nsn);
      near_atoms(S, po, nso);
    }
    double du = 0.0, ge[3] = {0, 0, 0}, le = 0.0;
    const bool halves = !has3 && S.nelec <= 16;
    if (halves) {
      // at most 16 electrons and no e-e-n terms: lanes 0-15 take the pairs
      // (e, j) at the proposed position, lanes 16-31 the same pairs at the
      // current one; each proposed-position lane collects its partner's terms
      const int j = lane & 15;
      const bool newp = lane < 16, live = j < S.nelec && j != e;
      double u1 = 0.0, f1 = 0.0, l1 = 0.0, dx = 0.0, dy = 0.0, dz = 0.0;
      if (live) {
        const double* pj = Rp + 3 * j;
        dx = (newp ? px : ox) - pj[0]; dy = (newp ? py : oy) - pj[1]; dz = (newp ? pz : oz) - pj[2];
        min_image(S, dx, dy, dz);
        const double d2 = dx * dx + dy * dy + dz * dz;
        if (d2 < S.ee_rc2) jas_pair_t<Real>(S, se == (j < S.nup), sqrt(Real(d2)), u1, f1, l1);
      }
      const double qgx = __shfl_xor_sync(0xffffffffu, f1 * dx, 16), qgy = __shfl_xor_sync(0xffffffffu, f1 * dy, 16),
                   qgz = __shfl_xor_sync(0xffffffffu, f1 * dz, 16), ql = __shfl_xor_sync(0xffffffffu, l1, 16);
      if (newp) {
        du += u1;
        ge[0] += f1 * dx; ge[1] += f1 * dy; ge[2] += f1 * dz;
        le += l1;
        if (live) {
          // gradient w.r.t. r_j of u(r_e - r_j) = -f'/r (r_e - r_j)
          double* dg = dG() + 4 * j;
          dg[0] = -f1 * dx + qgx; dg[1] = -f1 * dy + qgy; dg[2] = -f1 * dz + qgz; dg[3] = l1 - ql;
        }
      } else {
        du -= u1;
      }
    }
    for (int j = halves ? S.nelec : lane; j < S.nelec; j += 32) {
      double* dg = dG() + 4 * j;
      if (j == e) continue;
      const double* pj = Rp + 3 * j;
      const bool same = se == (j < S.nup);
      double nx = px - pj[0], ny = py - pj[1], nz = pz - pj[2];
      double qx = ox - pj[0], qy = oy - pj[1], qz = oz - pj[2];
      min_image(S, nx, ny, nz);
      min_image(S, qx, qy, qz);
      if (!(nx * nx + ny * ny + nz * nz < S.ee_rc2) && !(qx * qx + qy * qy + qz * qz < S.ee_rc2)) {
        dg[0] = dg[1] = dg[2] = dg[3] = 0.0;  // beyond every e-e cutoff before and after the move
        continue;
      }
      // pair functions in the working precision, sums in FP64
      const Real rn = sqrt(Real(nx * nx + ny * ny + nz * nz)), ro = sqrt(Real(qx * qx + qy * qy + qz * qz));
      double un, fn, ln, uo, fo, lo;
      jas_pair_t<Real>(S, same, rn, un, fn, ln);
      jas_pair_t<Real>(S, same, ro, uo, fo, lo);
      du += un - uo;
      ge[0] += fn * nx; ge[1] += fn * ny; ge[2] += fn * nz;
      le += ln;
      // gradient w.r.t. r_j of u(r_e - r_j) = -f'/r (r_e - r_j)
      double g0 = -fn * nx + fo * qx, g1 = -fn * ny + fo * qy, g2 = -fn * nz + fo * qz, l0 = ln - lo;
      if constexpr (has3) {
        if (nsn.n >= 0 && nso.n >= 0) {
          const double dn[3] = {nx, ny, nz}, dq[3] = {qx, qy, qz};
          const double rnd = sqrt(nx * nx + ny * ny + nz * nz), rqd = sqrt(qx * qx + qy * qy + qz * qz);
          double dgj[3] = {0, 0, 0}, dlj = 0;
          tb_pair_move(S, nsn, nso, same, pj, dn, rnd, dq, rqd, du, ge, le, dgj, dlj);
          g0 += dgj[0]; g1 += dgj[1]; g2 += dgj[2];
          l0 += dlj;
        } else {
          double pn[3] = {px, py, pz}, po[3] = {ox, oy, oz};
          double tu, tgi[3], tli, tgj[3], tlj, su, sgi[3], sli, sgj[3], slj;
          jas_threebody_pair(S, nsn, same, pn, pj, tu, tgi, tli, tgj, tlj, true);
          jas_threebody_pair(S, nso, same, po, pj, su, sgi, sli, sgj, slj, true);
          du += tu - su;
          ge[0] += tgi[0]; ge[1] += tgi[1]; ge[2] += tgi[2];
          le += tli;
          g0 += tgj[0] - sgj[0]; g1 += tgj[1] - sgj[1]; g2 += tgj[2] - sgj[2];
          l0 += tlj - slj;
        }
      }
      dg[0] = g0; dg[1] = g1; dg[2] = g2; dg[3] = l0;
    }
    // one-body terms: lanes over (atom, function) pairs
    for (int idx = lane; idx < S.natoms * QWG_MAXEI; idx += 32) {
      const int a = idx / QWG_MAXEI, k = idx - a * QWG_MAXEI;
      const int t = S.atom_type[a];
      if (k >= S.ei_n[t]) continue;
      const double c = S.onebody[t][k];
      if (c == 0.0) continue;
      const double* ap = S.atom_pos[a];
      double nx = px - ap[0], ny = py - ap[1], nz = pz - ap[2];
      double qx = ox - ap[0], qy = oy - ap[1], qz = oz - ap[2];
      min_image(S, nx, ny, nz);
      min_image(S, qx, qy, qz);
      double rn = sqrt(nx * nx + ny * ny + nz * nz), ro = sqrt(qx * qx + qy * qy + qz * qz);
      double fnv, fnd, fnl;
      radial_lap(S.ei[t][k], rn, fnv, fnd, fnl);
      du += c * (fnv - radial_val(S.ei[t][k], ro));
      ge[0] += c * fnd * nx; ge[1] += c * fnd * ny; ge[2] += c * fnd * nz;
      le += c * fnl;
    }
    dU = warp_sum(du);
    double gu[3] = {warp_sum(ge[0]), warp_sum(ge[1]), warp_sum(ge[2])};
    double lu_ = warp_sum(le);
    double dot = 0, gg = 0;
    for (int d = 0; d < 3; d++) {
      gnew[d] = gD[d] + gu[d];
      dot += gD[d] * gu[d];
      gg += gu[d] * gu[d];
    }
    lapnew = lD + lu_ + gg + 2 * dot;
    // stash the new Jastrow gradient/lap of e for an accept
    __syncwarp();
    if (lane == 0) { dG()[4 * e] = gu[0]; dG()[4 * e + 1] = gu[1]; dG()[4 * e + 2] = gu[2]; dG()[4 * e + 3] = lu_; }
    __syncwarp();
    QWG_PHASE_END(t_rest, PH_PROPOSE_REST, ph)
  }

  // ---- accept the proposal of electron e: Sherman-Morrison update of the
  // transposed inverse (InverseUpdateColumn, MatrixAlgebrac.cpp:766-838),
  // the stored MO row, position and Jastrow sums.
  __device__ void accept(int e, double px, double py, double pz, double ratioD, double dU) {
    const int s = spin(e), el = eloc(e), M = S.m[s];
    Real* iv = inv(s);
    Real* nc = newcol();
    // scratch: wk[k] = sum_i phi'_i invT[k][i], rowe[i] = invT[el][i]
    Real* wk = (Real*)lu();
    Real* rowe = wk + MS();
    const int ms = MS();
    if (multi()) {
      // Sherman-Morrison update of every distinct spin-determinant with its
      // own ratio (from propose), then the stored rows of every union orbital
      for (int u = 0; u < S.nud[s]; u++) {
        const double ru = mdr()[u * 5];
        Real* ivu = inv_u(s, u);
        const int* cu = cols(s, u);
        if (!(ru != 0.0) || !isfinite(ru)) {
          if (lane == 0) udl()[((size_t)s * L.nud + u) * 2] = -1e201;  // became singular
          __syncwarp();
          continue;
        }
        for (int k = lane; k < M; k += 32) {
          Real acc = 0;
          for (int i = 0; i < M; i++) acc += nc[cu[i] * 5] * ivu[(size_t)k * ms + i];
          wk[k] = acc;
          rowe[k] = ivu[(size_t)el * ms + k];
        }
        __syncwarp();
        const Real invr = Real(1.0 / ru);
        for (int idx = lane; idx < M * M; idx += 32) {
          int k = idx / M, i = idx - k * M;
          if (k == el) ivu[(size_t)k * ms + i] = rowe[i] * invr;
          else ivu[(size_t)k * ms + i] -= rowe[i] * wk[k] * invr;
        }
        __syncwarp();
        if (lane == 0) {
          double* d = udl() + ((size_t)s * L.nud + u) * 2;
          d[0] += log(fabs(ru));
          if (ru < 0) d[1] = -d[1];
        }
        __syncwarp();
      }
      for (int j = lane; j < S.nmo_u[s]; j += 32) {
        Real* mv = mov() + ((size_t)e * ms + j) * 4;
        mv[0] = nc[j * 5 + 1]; mv[1] = nc[j * 5 + 2]; mv[2] = nc[j * 5 + 3]; mv[3] = nc[j * 5 + 4];
      }
    }
    if constexpr (CPX) {
      // complex Sherman-Morrison update with R = cr_re + i cr_im
      Real* ivi = iv + (size_t)ms * ms;
      const Real* nci = nc + newcol_im_off();
      Real* wki = rowe + ms;
      Real* rowi = wki + ms;
      for (int k = lane; k < M; k += 32) {
        Real ar = 0, ai = 0;
        for (int i = 0; i < M; i++) {
          const Real xr = nc[i * 5], xi = nci[i * 5], vr = iv[(size_t)k * ms + i], vi = ivi[(size_t)k * ms + i];
          ar += xr * vr - xi * vi;
          ai += xr * vi + xi * vr;
        }
        wk[k] = ar; wki[k] = ai;
        rowe[k] = iv[(size_t)el * ms + k]; rowi[k] = ivi[(size_t)el * ms + k];
      }
      __syncwarp();
      const double m2 = cr_re * cr_re + cr_im * cr_im;
      const Real qr = Real(cr_re / m2), qi = Real(-cr_im / m2);  // 1 / R
      for (int idx = lane; idx < M * M; idx += 32) {
        int k = idx / M, i = idx - k * M;
        const Real ur = rowe[i] * qr - rowi[i] * qi, ui = rowe[i] * qi + rowi[i] * qr;  // row_el / R
        if (k == el) { iv[(size_t)k * ms + i] = ur; ivi[(size_t)k * ms + i] = ui; }
        else {
          iv[(size_t)k * ms + i] -= ur * wk[k] - ui * wki[k];
          ivi[(size_t)k * ms + i] -= ur * wki[k] + ui * wk[k];
        }
      }
      for (int i = lane; i < M; i += 32) {
        Real* mv = mov() + ((size_t)e * ms + i) * 4;
        Real* mw = mv + mov_im_off();
        for (int q = 0; q < 4; q++) { mv[q] = nc[i * 5 + 1 + q]; mw[q] = nci[i * 5 + 1 + q]; }
      }
    }
    for (int k = lane; k < M && !multi() && !CPX; k += 32) {
      Real acc = 0;
      for (int i = 0; i < M; i++) acc += nc[i * 5] * iv[(size_t)k * ms + i];
      wk[k] = acc;
      rowe[k] = iv[(size_t)el * ms + k];
    }
    __syncwarp();
    const Real invr = Real(1.0 / ratioD);
    for (int idx = lane; idx < M * M && !multi() && !CPX; idx += 32) {
      int k = idx / M, i = idx - k * M;
      if (k == el) iv[(size_t)k * ms + i] = rowe[i] * invr;
      else iv[(size_t)k * ms + i] -= rowe[i] * wk[k] * invr;
    }
    for (int i = lane; i < M && !multi() && !CPX; i += 32) {
      Real* mv = mov() + ((size_t)e * ms + i) * 4;
      mv[0] = nc[i * 5 + 1]; mv[1] = nc[i * 5 + 2]; mv[2] = nc[i * 5 + 3]; mv[3] = nc[i * 5 + 4];
    }
    for (int j = lane; j < S.nelec; j += 32) {
      const double* dg = dG() + 4 * j;
      if (j == e) {
        gU()[3 * j] = dg[0]; gU()[3 * j + 1] = dg[1]; gU()[3 * j + 2] = dg[2]; lU()[j] = dg[3];
      } else {
        gU()[3 * j] += dg[0]; gU()[3 * j + 1] += dg[1]; gU()[3 * j + 2] += dg[2]; lU()[j] += dg[3];
      }
    }
    if (lane == 0) {
      double* Rp = R();
      Rp[3 * e] = px; Rp[3 * e + 1] = py; Rp[3 * e + 2] = pz;
      WScal* w = sc();
      w->logdet[s] += log(fabs(ratioD));
      if (CPX) w->phase += atan2(cr_im, cr_re);
      else if (ratioD < 0) w->sign[s] = -w->sign[s];
      w->U += dU;
    }
    __syncwarp();
    if (multi()) md_weights();
  }

  __device__ void electron_grad(int e, double g[3], double& lap) const {
    double gD[3], lD;
    slater_gl(e, gD, lD);
    const double* gu = gU() + 3 * e;
    double dot = 0, gg = 0;
    for (int d = 0; d < 3; d++) {
      g[d] = gD[d] + gu[d];
      dot += gD[d] * gu[d];
      gg += gu[d] * gu[d];
    }
    lap = lD + lU()[e] + gg + 2 * dot;
  }

  // ---- local energy pieces
  __device__ double kinetic() const {
    double k = 0;
    for (int e = lane; e < S.nelec; e += 32) {
      double g[3], l;
      electron_grad(e, g, l);
      k += l;
    }
    return -0.5 * warp_sum(k);
  }

  // Periodic_system::ewaldElectron + the constant ion/self terms
  // (Periodic_system.cpp:586-973): real-space sums over the 27 images of the
  // minimum-image vectors, reciprocal sum over the kept G-vectors.
  __device__ double ewald() const {
    const double* Rp = R();
    const int N = S.nelec, A = S.natoms;
    double v = 0;
    for (int idx = lane; idx < N * A; idx += 32) {
      const int e = idx / A, a = idx - e * A;
      double dx = Rp[3 * e] - S.atom_pos[a][0], dy = Rp[3 * e + 1] - S.atom_pos[a][1], dz = Rp[3 * e + 2] - S.atom_pos[a][2];
      min_image(S, dx, dy, dz);
      double t = 0;
      for (int k = 0; k < 27; k++) {
        double x = dx + S.lattice_basis[k][0], y = dy + S.lattice_basis[k][1], z = dz + S.lattice_basis[k][2];
        double r = sqrt(x * x + y * y + z * z);
        t += erfc_poly(S.alpha * r) / r;
      }
      v -= S.atom_charge[a] * t;
    }
    for (int idx = lane; idx < N * N; idx += 32) {
      const int i = idx / N, j = idx - i * N;
      if (i >= j) continue;
      double dx = Rp[3 * i] - Rp[3 * j], dy = Rp[3 * i + 1] - Rp[3 * j + 1], dz = Rp[3 * i + 2] - Rp[3 * j + 2];
      min_image(S, dx, dy, dz);
      for (int k = 0; k < 27; k++) {
        double x = dx + S.lattice_basis[k][0], y = dy + S.lattice_basis[k][1], z = dz + S.lattice_basis[k][2];
        double r = sqrt(x * x + y * y + z * z);
        v += erfc_poly(S.alpha * r) / r;
      }
    }
    for (int g = lane; g < S.ng; g += 32) {
      const double* G = S.gvec + 3 * g;
      double ss = 0, cs = 0;
      for (int e = 0; e < N; e++) {
        double sn, cn;
        sincos(G[0] * Rp[3 * e] + G[1] * Rp[3 * e + 1] + G[2] * Rp[3 * e + 2], &sn, &cn);
        ss += sn; cs += cn;
      }
      const double w = S.gweight[g];
      v += 2.0 * (-(S.ion_cos[g] * cs + S.ion_sin[g] * ss) * w + (cs * cs + ss * ss) * w / 2);
    }
    return warp_sum(v) + S.ewald_const;
  }

  // Molecular_system::calcLoc (Molecular_system.cpp:209-287), no field.
  __device__ double coulomb() const {
    if (PER == 1 || (PER == 2 && S.periodic)) return ewald();
    const double* Rp = R();
    const int N = S.nelec, A = S.natoms;
    double v = 0;
    for (int idx = lane; idx < N * A; idx += 32) {
      int e = idx / A, a = idx - e * A;
      const double* ap = S.atom_pos[a];
      double dx = Rp[3 * e] - ap[0], dy = Rp[3 * e + 1] - ap[1], dz = Rp[3 * e + 2] - ap[2];
      v -= S.atom_charge[a] / sqrt(dx * dx + dy * dy + dz * dz);
    }
    for (int idx = lane; idx < N * N; idx += 32) {
      int i = idx / N, j = idx - i * N;
      if (i >= j) continue;
      double dx = Rp[3 * i] - Rp[3 * j], dy = Rp[3 * i + 1] - Rp[3 * j + 1], dz = Rp[3 * i + 2] - Rp[3 * j + 2];
      v += 1.0 / sqrt(dx * dx + dy * dy + dz * dz);
    }
    return warp_sum(v) + S.ion_ion;
  }

  // Radial v_l(r) of channel l for an electron of spin s (SPIN_DEP tables
  // per spin, Pseudopotential::getRadial, Pseudopotential.cpp:305-336).
  __device__ double pp_radial(int t, int s, int l, double r) const {
    const int* tf = s == 0 ? S.pp_term_first[t] : S.pp_term_first_dn[t];
    double v = 0;
    for (int n = tf[l]; n < tf[l + 1]; n++) {
      const double* q = S.pp_term[t][n];
      double ex = fmin(q[1] * r * r, 60.0);
      const double pw = q[0];
      const double rn = pw == 0.0 ? 1.0 : pw == -1.0 ? 1.0 / r : pw == 1.0 ? r : pw == -2.0 ? 1.0 / (r * r)
                      : pw == 2.0 ? r * r : pow(r, pw);
      v += q[2] * rn * exp(-ex);
    }
    return v;
  }

  // Semilocal pseudopotential (Pseudopotential::calcNonlocWithAllvariables,
  // Pseudopotential.cpp:596-815): local channel for every (e, atom) and the
  // Q-point quadrature of the nonlocal channels for the pairs selected
  // deterministically (r < cutoff) or stochastically (rand < strength, with
  // the nonlocal radials divided by the strength).  rot: 3x3 rows x,y,z.
  // T-moves: the quadrature terms v_xx of every point go to cand; with
  // tmoves == 2 every electron then moves to one of its points of negative
  // v_xx with probability tau |v_xx| / (1 + tau sum |v_xx|), with tmoves == 1
  // at most one electron of the walker moves, chosen over all such points
  // (Dmc_method::doTmove, Dmc_method.cpp:850-906; Pseudopotential.cpp:740-763).
  // The energy keeps every term.  Selected targets go to moves[N][4].
  template <bool TMV = false>
  __device__ double pseudo(const double* rotm, bool deterministic, uint64_t seed, uint32_t wid, uint64_t step,
                           int tmoves_ = 0, double tm_tau = 0.0, double* cand = nullptr, double* moves = nullptr) {
    const int tmoves = TMV ? tmoves_ : 0;  // T-move code only in the TMV instantiation
    const double* Rp = R();
    const int N = S.nelec, A = S.natoms;
    double vloc = 0;
    if (tmoves)
      for (int e = lane; e < N; e += 32) moves[4 * e + 3] = 0.0;
    double res_total = 1.0, res_x = 0, res_y = 0, res_z = 0;  // one-move-per-walker reservoir
    int res_e = -1;
    // per-electron Jastrow value at the current position
    QWG_PHASE_BEGIN(t_ue)
    for (int e = lane; e < N; e += 32)
      Ue()[e] = double(jas_electron_val<Real, TB>(S, Rp, e, Rp[3 * e], Rp[3 * e + 1], Rp[3 * e + 2]));
    __syncwarp();
    QWG_PHASE_END(t_ue, PH_PP_JASTROW, ph)
    double vnl = 0;
    // electrons in chunks of L.wchunk: the (electron, atom) items of the
    // chunk in electron-major order, the chunk's projected coefficients, then
    // lanes over the chunk's (item, quadrature point) pairs
    const int CH = L.wchunk;
    PPItem* it = items();
    Real* w = wproj();
    for (int e0 = 0; e0 < N; e0 += CH) {
      const int e1 = min(N, e0 + CH);
      QWG_PHASE_BEGIN(t_items)
      int nitems = 0;
      for (int base0 = e0 * A; base0 < e1 * A; base0 += 32) {
        const int idx = base0 + lane;
        bool take = false;
        PPItem item;
        if (idx < e1 * A) {
          const int e = idx / A, a = idx - e * A;
          const int t = S.atom_type[a];
          const int nch = S.pp_nchan[t];
          if (nch > 0) {
            const double* ap = S.atom_pos[a];
            item.e = e; item.a = a;
            item.dx = Rp[3 * e] - ap[0]; item.dy = Rp[3 * e + 1] - ap[1]; item.dz = Rp[3 * e + 2] - ap[2];
            min_image(S, item.dx, item.dy, item.dz);
            item.r = sqrt(item.dx * item.dx + item.dy * item.dy + item.dz * item.dz);
            const int sp = spin(e);
            vloc += pp_radial(t, sp, nch - 1, item.r) + (S.pp_addzeff[t] ? S.atom_charge[a] / item.r : 0.0);
            for (int l = 0; l < 4; l++) item.vl[l] = (l < nch - 1) ? pp_radial(t, sp, l, item.r) : 0.0;
            if (deterministic) {
              take = item.r < S.pp_cutoff[t];
            } else {
              double strength = 0;
              for (int l = 0; l < nch - 1; l++) strength += 10.0 * (2 * l + 1) * fabs(item.vl[l]);
              strength = fmin(1.0, strength);
              Rand4 rr = rand4(seed, wid, step, (uint32_t)idx, 7u);
              if (fabs(strength) > 0)
                for (int l = 0; l < nch - 1; l++) item.vl[l] /= strength;
              take = strength > rr.u[0];
            }
          }
        }
        unsigned m = __ballot_sync(0xffffffffu, take);
        int pos = nitems + __popc(m & ((1u << lane) - 1u));
        if (take) it[pos] = item;
        nitems += __popc(m);
      }
      __syncwarp();
      QWG_PHASE_END(t_items, PH_PP_ITEMS, ph)
      if (nitems == 0) continue;
      QWG_PHASE_BEGIN(t_proj)
      const int nproj = multi() ? L.nud : 1;  // projected-coefficient sets per electron
      for (int idx = lane; idx < (e1 - e0) * S.nbasis * nproj && multi(); idx += 32) {
        // one set per distinct spin-determinant u: w_f = sum_i C[f][col_u(i)] (A_u^-1)[i][e]
        const int u = idx / ((e1 - e0) * S.nbasis), r = idx - u * (e1 - e0) * S.nbasis;
        const int le = r / S.nbasis, f = r - le * S.nbasis;
        const int e = e0 + le, s = spin(e), el = eloc(e), M = S.m[s];
        if (u >= S.nud[s]) continue;
        const Real* cf = mocs(s) + (size_t)f * MS();
        const Real* iv = inv_u(s, u) + (size_t)el * MS();
        const int* cu = cols(s, u);
        Real acc = Real(0);
        for (int m = 0; m < M; m++) acc += cf[cu[m]] * iv[m];
        w[((size_t)u * CH + le) * S.nbasis + f] = acc;
      }
      for (int idx = lane; idx < (e1 - e0) * S.nbasis && CPX; idx += 32) {
        // complex w_f = sum_m C[f][m] invT[el][m]
        const int le = idx / S.nbasis, f = idx - le * S.nbasis;
        const int e = e0 + le, s = spin(e), el = eloc(e), M = S.m[s];
        const Real* cf = mocs(s) + (size_t)f * MS();
        const Real* cfi = mocs_im(s) + (size_t)f * MS();
        const Real* iv = inv(s) + (size_t)el * MS();
        const Real* ivi = iv + (size_t)MS() * MS();
        Real ar = Real(0), ai = Real(0);
        for (int m = 0; m < M; m++) {
          ar += cf[m] * iv[m] - cfi[m] * ivi[m];
          ai += cf[m] * ivi[m] + cfi[m] * iv[m];
        }
        w[le * S.nbasis + f] = ar;
        w[wproj_im_off() + le * S.nbasis + f] = ai;
      }
      for (int idx = lane; idx < (e1 - e0) * S.nbasis && !multi() && !CPX; idx += 32) {
        const int le = idx / S.nbasis, f = idx - le * S.nbasis;
        const int e = e0 + le, s = spin(e), el = eloc(e), M = S.m[s];
        const Real* cf = mocs(s) + (size_t)f * MS();
        const Real* iv = inv(s) + (size_t)el * MS();
        Real acc = Real(0);
        if constexpr (MMAX > 0) {
#pragma unroll
          for (int m = 0; m < MMAX; m++)
            if (m < M) acc += cf[m] * iv[m];
        } else {
          for (int m = 0; m < M; m++) acc += cf[m] * iv[m];
        }
        w[le * S.nbasis + f] = acc;
      }
      __syncwarp();
      QWG_PHASE_END(t_proj, PH_PP_PROJECT, ph)
      QWG_PHASE_BEGIN(t_pts)
      int total = 0;
      for (int k = 0; k < nitems; k++) total += S.pp_aip[S.atom_type[it[k].a]];
      int k = 0, qoff = 0;  // running item cursor for this lane's points
      for (int p = lane; p < total; p += 32) {
        while (p >= qoff + S.pp_aip[S.atom_type[it[k].a]]) { qoff += S.pp_aip[S.atom_type[it[k].a]]; k++; }
        const PPItem& I = it[k];
        const int q = p - qoff;
        const int ty = S.atom_type[I.a];
        const double* q0 = S.pp_quad[ty][q];
        double qx = q0[0] * rotm[0] + q0[1] * rotm[3] + q0[2] * rotm[6];
        double qy = q0[0] * rotm[1] + q0[1] * rotm[4] + q0[2] * rotm[7];
        double qz = q0[0] * rotm[2] + q0[1] * rotm[5] + q0[2] * rotm[8];
        // move relative to the nearest image of the atom, then into the cell
        double nx = Rp[3 * I.e] + qx * I.r - I.dx, ny = Rp[3 * I.e + 1] + qy * I.r - I.dy,
               nz = Rp[3 * I.e + 2] + qz * I.r - I.dz;
        const Real* wr = w + (I.e - e0) * S.nbasis;
        Real rd;
        if constexpr (CPX) {
          // the wrap's k-point phase pi k.n: the overall phase (sign for
          // integer k) of Periodic_sample::translateElectron enters the point
          // value (Pseudopotential.cpp:727-745): Re(R e^{-i pi k.n}) for complex
          // orbitals, R cos(pi k.n) for real orbitals at an integer k-point
          const double kd = wrap_pos_kphase(S, nx, ny, nz);
          Real pr, pi;
          basis_dot_lane_cpx(S, nx, ny, nz, wr, wr + wproj_im_off(), pr, pi);
          double sn, cs;
          sincos(kd, &sn, &cs);
          if (S.real_orb) rd = Real(double(pr) * (S.kint ? cs : 1.0));
          else rd = Real(double(pr) * cs + double(pi) * sn);
        } else {
          wrap_pos(S, nx, ny, nz);
          if (PER == 1 || (PER == 2 && S.periodic)) {
            rd = basis_dot_lane_periodic<Real, HL>(S, nx, ny, nz, wr);
          } else if (multi()) {
            // sum over distinct spin-determinants of T[s][u] R_u / W
            const int s = spin(I.e);
            Real ru[QWG_MAXUD];
            basis_dot_lane_multi(S, nx, ny, nz, wr, CH * S.nbasis, S.nud[s], ru);
            const double* T = mdt() + QWG_MAXDET + 2 + s * QWG_MAXUD;
            double acc = 0.0;
            for (int u = 0; u < S.nud[s]; u++) acc += T[u] * double(ru[u]);
            rd = Real(acc / mdt()[QWG_MAXDET]);
          } else {
            rd = basis_dot_lane<Real, HL>(S, nx, ny, nz, wr);
          }
        }
        QWG_PHASE_BEGIN(t_pj)
        const Real u = jas_electron_val<Real, TB>(S, Rp, I.e, nx, ny, nz);
        QWG_PHASE_END(t_pj, PH_PP_POINT_JAS, ph)
        double ratio = double(rd * exp(u - Real(Ue()[I.e]))) * S.pp_w[ty][q];
        // cos of the angle between the original and the quadrature direction
        const double* ap = S.atom_pos[I.a];
        double ndx = nx - ap[0], ndy = ny - ap[1], ndz = nz - ap[2];
        min_image(S, ndx, ndy, ndz);
        double nr = sqrt(ndx * ndx + ndy * ndy + ndz * ndz);
        double c = (ndx * I.dx + ndy * I.dy + ndz * I.dz) / (nr * I.r);
        double P[4] = {1.0, c, 0.5 * (3 * c * c - 1), 0.5 * (5 * c * c * c - 3 * c)};
        double ts = 0;
        for (int ll = 0; ll < 4; ll++) ts += (2 * ll + 1) * I.vl[ll] * P[ll];
        vnl += ts * ratio;
        if (tmoves) cand[p] = ts * ratio;
      }
      __syncwarp();
      QWG_PHASE_END(t_pts, PH_PP_POINTS, ph)
      if (tmoves) {
        // target of point p of this chunk (the same arithmetic as above)
        auto point_pos = [&](int p, double& x, double& y, double& z) {
          int kk = 0, qo = 0;
          while (p >= qo + S.pp_aip[S.atom_type[it[kk].a]]) { qo += S.pp_aip[S.atom_type[it[kk].a]]; kk++; }
          const PPItem& I = it[kk];
          const double* q0 = S.pp_quad[S.atom_type[I.a]][p - qo];
          const double qx = q0[0] * rotm[0] + q0[1] * rotm[3] + q0[2] * rotm[6];
          const double qy = q0[0] * rotm[1] + q0[1] * rotm[4] + q0[2] * rotm[7];
          const double qz = q0[0] * rotm[2] + q0[1] * rotm[5] + q0[2] * rotm[8];
          x = Rp[3 * I.e] + qx * I.r - I.dx; y = Rp[3 * I.e + 1] + qy * I.r - I.dy; z = Rp[3 * I.e + 2] + qz * I.r - I.dz;
          wrap_pos(S, x, y, z);
        };
        if (tmoves == 2) {
          // size-consistent: lanes over the chunk's electrons; the points of
          // one electron are contiguous (items are in electron order)
          for (int e = e0 + lane; e < e1; e += 32) {
            int pb = 0, k = 0;
            for (; k < nitems && it[k].e < e; k++) pb += S.pp_aip[S.atom_type[it[k].a]];
            int pe = pb;
            for (; k < nitems && it[k].e == e; k++) pe += S.pp_aip[S.atom_type[it[k].a]];
            if (pe == pb) continue;
            double sum = 1.0;
            for (int p = pb; p < pe; p++)
              if (cand[p] < 0) sum -= tm_tau * cand[p];
            const double x = rand4(seed, wid, step, (uint32_t)e, 8u).u[0] * sum;
            if (!(x > 1.0)) continue;
            double sel = 1.0;
            for (int p = pb; p < pe; p++) {
              if (!(cand[p] < 0)) continue;
              sel -= tm_tau * cand[p];
              if (x < sel) {
                point_pos(p, moves[4 * e], moves[4 * e + 1], moves[4 * e + 2]);
                moves[4 * e + 3] = 1.0;
                break;
              }
            }
          }
        } else {
          // one move per walker over all electrons: a weighted reservoir
          // across the chunks (same distribution as one draw over all terms)
          double tc = 0.0;
          for (int p = 0; p < total; p++)
            if (cand[p] < 0) tc -= tm_tau * cand[p];
          if (tc > 0) {
            const Rand4 r = rand4(seed, wid, step, 0x10000u + (uint32_t)e0, 9u);
            res_total += tc;
            if (r.u[1] * res_total < tc) {
              const double x = r.u[0] * tc;
              double sel = 0.0;
              for (int p = 0; p < total; p++) {
                if (!(cand[p] < 0)) continue;
                sel -= tm_tau * cand[p];
                if (x < sel || p == total - 1) {
                  int kk = 0, qo = 0;
                  while (p >= qo + S.pp_aip[S.atom_type[it[kk].a]]) { qo += S.pp_aip[S.atom_type[it[kk].a]]; kk++; }
                  res_e = it[kk].e;
                  point_pos(p, res_x, res_y, res_z);
                  break;
                }
              }
            }
          }
        }
        __syncwarp();
      }
    }
    if (tmoves == 1 && res_e >= 0 && lane == 0) {
      moves[4 * res_e] = res_x; moves[4 * res_e + 1] = res_y; moves[4 * res_e + 2] = res_z;
      moves[4 * res_e + 3] = 1.0;
    }
    __syncwarp();
    return warp_sum(vloc) + warp_sum(vnl);
  }
};

// Limited drift of Split_sampler (limDrift, drift_cyrus, Split_sample.cpp:40-88).
__device__ __forceinline__ void lim_drift(const double d[3], double tau, double out[3]) {
  double d2 = (d[0] * d[0] + d[1] * d[1] + d[2] * d[2]) * 0.25;
  double a = d2 > 1e-8 ? (sqrt(1.0 + 2.0 * tau * d2) - 1.0) / d2 : tau;
  out[0] = d[0] * a; out[1] = d[1] * a; out[2] = d[2] * a;
}

// Uniform random rotation from a random unit quaternion (Shoemake 1992).
__device__ __forceinline__ void random_rotation(const Rand4& r, double m[9]) {
  double s1 = sqrt(1.0 - r.u[0]), s2 = sqrt(r.u[0]);
  double a1, b1, a2, b2;
  sincospi(2.0 * r.u[1], &a1, &b1);
  sincospi(2.0 * r.u[2], &a2, &b2);
  double x = s1 * a1, y = s1 * b1, z = s2 * a2, w = s2 * b2;
  m[0] = 1 - 2 * (y * y + z * z); m[1] = 2 * (x * y + z * w);     m[2] = 2 * (x * z - y * w);
  m[3] = 2 * (x * y - z * w);     m[4] = 1 - 2 * (x * x + z * z); m[5] = 2 * (y * z + x * w);
  m[6] = 2 * (x * z + y * w);     m[7] = 2 * (y * z - x * w);     m[8] = 1 - 2 * (x * x + y * y);
}

// Resident 128-thread CTAs per SM the register budget of each kernel mode is
// sized for (the move and local-energy kernels are smaller than the fused one).
#ifndef QWG_MIN_BLOCKS
#define QWG_MIN_BLOCKS 4
#endif
#ifndef QWG_MIN_BLOCKS_SWEEP
#define QWG_MIN_BLOCKS_SWEEP 4
#endif
#ifndef QWG_MIN_BLOCKS_ELOC
#define QWG_MIN_BLOCKS_ELOC 4
#endif
template <int mode>
struct MinBlocks { static constexpr int value = QWG_MIN_BLOCKS; };
template <>
struct MinBlocks<KM_SWEEP> { static constexpr int value = QWG_MIN_BLOCKS_SWEEP; };
template <>
struct MinBlocks<KM_ELOC> { static constexpr int value = QWG_MIN_BLOCKS_ELOC; };
template <>
struct MinBlocks<KM_ELOC_TM> { static constexpr int value = QWG_MIN_BLOCKS_ELOC; };

// the parameter bank, layout, step parameters and I/O pointers travel as
// kernel parameters (at most 32764 bytes on sm_70 and later)
static_assert(sizeof(DevSys<double>) + sizeof(WLayout) + sizeof(StepParams) + sizeof(EvalIO) <= 32764,
              "walker kernel parameters exceed 32764 bytes");

template <typename Real, int MMAX, int mode, bool TB, int PER, bool XL = (MMAX <= 0)>
__global__ void __launch_bounds__(128, MinBlocks<mode>::value)
    k_walkers(const __grid_constant__ DevSys<Real> S, const __grid_constant__ WLayout L, StepParams P, EvalIO io) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int wpc = blockDim.x / 32;
  const int warp = threadIdx.x / 32, lane = threadIdx.x & 31;
  // MO coefficients are read through L1 (a few kB shared by every walker);
  // shared memory holds walker state only
  const Real* moc_s = S.moc;
  const size_t moc_bytes = 0;
  __shared__ double cta_acc[QWG_NACC];
  if (threadIdx.x < QWG_NACC) cta_acc[threadIdx.x] = 0.0;
  __syncthreads();

  const int wid = blockIdx.x * wpc + warp;
  constexpr bool HBM = MMAX <= 0;  // walker worked on in place in HBM
  constexpr bool CPXK = MMAX < 0;  // complex orbitals
  if (wid < P.nwalk) {
    unsigned char* gstate = P.state + (size_t)wid * L.state_bytes;
    constexpr bool SWEEP_ONLY = mode == KM_SWEEP || mode == KM_TMOVE;  // move-phase shared memory only
    unsigned char* wb = HBM ? gstate : smem + moc_bytes + (size_t)warp * (SWEEP_ONLY ? L.sweep_bytes : L.bytes);
    unsigned char* sb = HBM ? P.scratch + (size_t)wid * L.scratch_bytes : wb + L.state_bytes;
    Walker<Real, MMAX, TB, PER, XL> W{S, L, wb, sb, moc_s, lane};
    // tensor-core move schedule: this launch moves electron P.tc_e only
    W.ph = P.phases;
    QWG_PHASE_BEGIN(t_walker)
    const int tc_phase = (mode == KM_SWEEP && MMAX == 0 && sizeof(Real) == 4) ? P.tc_phase : 0;
    if (tc_phase == 2) {
      W.tcD = P.tc_D + (size_t)wid * 5 * P.tc_ldd;
      W.tc_ldd = P.tc_ldd;
    }
    const int N = S.nelec;
    double* Rp = W.R();
    const uint64_t step0 = P.dyn_step ? (uint64_t)P.etrial[DYN_STEP] : P.step0;
    int refresh = P.refresh;
    if (refresh == 2) {
      const uint64_t R = (uint64_t)P.refresh_every, m = step0 % R;
      refresh = (m == 0 || m + (uint64_t)P.nsteps > R) ? 1 : 0;
    }
    constexpr bool ELOCM = mode == KM_ELOC || mode == KM_ELOC_TM;  // local-energy phase
    if (ELOCM || mode == KM_TMOVE || (mode == KM_SWEEP && P.st > 0)) refresh = 0;  // a chunk's first sweep only
    if (tc_phase == 2 || (tc_phase == 1 && P.tc_e > 0)) refresh = 0;  // the sweep's first launch only
    constexpr bool STEPS = mode == KM_STEPS || mode == KM_SWEEP || ELOCM || mode == KM_TMOVE;
    if (!STEPS || refresh) {
      for (int i = lane; i < 3 * N; i += 32) Rp[i] = P.R[(size_t)wid * 3 * N + i];
      __syncwarp();
      if (S.periodic)
        for (int e = lane; e < N; e += 32) wrap_pos(S, Rp[3 * e], Rp[3 * e + 1], Rp[3 * e + 2]);
      double keep_e = 0, keep_w = 1;
      if (STEPS) { keep_e = ((WScal*)(gstate + L.scal))->eold; keep_w = ((WScal*)(gstate + L.scal))->weight; }
      __syncwarp();
      QWG_PHASE_BEGIN(t_ref)
      W.recompute();
      QWG_PHASE_END(t_ref, PH_REFRESH, P.phases)
      if (lane == 0 && STEPS) { W.sc()->eold = keep_e; W.sc()->weight = keep_w; }
      __syncwarp();
    } else if constexpr (!HBM) {
      // resident state: one coalesced copy HBM -> shared memory
      const int4* src = (const int4*)gstate;
      int4* dst = (int4*)wb;
      for (int i = lane; i < L.state_bytes / 16; i += 32) dst[i] = src[i];
      __syncwarp();
    }

    if constexpr (mode == KM_EVAL) {
      double rm[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
      if (io.rot)
        for (int k = 0; k < 9; k++) rm[k] = io.rot[(size_t)wid * 9 + k];
      for (int e = lane; e < N; e += 32) {
        double g[3], l;
        W.electron_grad(e, g, l);
        double* go = io.grad + ((size_t)wid * N + e) * 3;
        go[0] = g[0]; go[1] = g[1]; go[2] = g[2];
        io.lap[(size_t)wid * N + e] = l;
      }
      double kin = W.kinetic();
      double pot = W.coulomb();
      // P.tmoves here: T-move selection for qwg_tmove_select (no move is made)
      double nl = 0.0;
      if (S.has_pp) {
        if (P.tmoves)
          nl = W.template pseudo<true>(rm, true, P.seed, wid, 0, P.tmoves, P.tau, P.tm_cand + (size_t)wid * P.tm_cap,
                                       P.tm_moves + (size_t)wid * N * 4);
        else
          nl = W.pseudo(rm, true, 0, wid, 0);
      }
      if (lane == 0) {
        WScal* w = W.sc();
        if (W.multi()) {
          double sgn;
          io.logpsi[wid] = W.md_logpsi_d(sgn) + w->U;
          io.sign[wid] = sgn;
        } else {
          io.logpsi[wid] = w->logdet[0] + w->logdet[1] + w->U;
          // complex orbitals: arg psi; real orbitals on the complex kernels: the sign
          io.sign[wid] = !CPXK ? w->sign[0] * w->sign[1] : S.real_orb ? (cos(w->phase) < 0 ? -1.0 : 1.0) : w->phase;
        }
        io.kinetic[wid] = kin;
        io.potential[wid] = pot;
        io.nonlocal[wid] = nl;
      }
    } else if constexpr (mode == KM_RATIO) {
      const int e = io.move_e[wid];
      const double* rn = io.move_r + 3 * (size_t)wid;
      double mx = rn[0], my = rn[1], mz = rn[2];
      wrap_pos(S, mx, my, mz);
      double ratioD, dU, g[3], l;
      W.propose(e, mx, my, mz, ratioD, dU, g, l);
      if (lane == 0) {
        io.logpsi[wid] = log(fabs(ratioD)) + dU;
        // complex orbitals: the phase change; real ones: the sign of the ratio
        io.sign[wid] = CPXK && !S.real_orb ? atan2(W.cr_im, W.cr_re) : (CPXK ? W.cr_re : ratioD) < 0 ? -1.0 : 1.0;
        io.grad[3 * (size_t)wid] = g[0]; io.grad[3 * (size_t)wid + 1] = g[1]; io.grad[3 * (size_t)wid + 2] = g[2];
        io.lap[wid] = l;
      }
    } else if constexpr (mode == KM_TMOVE) {
      // the T-moves selected by the last local-energy pass: each chosen
      // electron moves to its quadrature point (Sample_point::translateElectron)
      const double* mv = P.tm_moves + (size_t)wid * N * 4;
      for (int e = 0; e < N; e++) {
        if (mv[4 * e + 3] == 0.0) continue;
        const double px = mv[4 * e], py = mv[4 * e + 1], pz = mv[4 * e + 2];
        double ratioD, dU, g[3], l;
        W.propose(e, px, py, pz, ratioD, dU, g, l);
        if (isfinite(ratioD) && ratioD != 0.0 && isfinite(dU)) W.accept(e, px, py, pz, ratioD, dU);
      }
      __syncwarp();
      for (int i = lane; i < 3 * N; i += 32) P.R[(size_t)wid * 3 * N + i] = Rp[i];
      if constexpr (!HBM) {
        int4* dst = (int4*)gstate;
        const int4* src = (const int4*)wb;
        for (int i = lane; i < L.state_bytes / 16; i += 32) dst[i] = src[i];
      }
    } else {
      // ---- VMC / DMC steps (KM_STEPS: P.nsteps steps; KM_SWEEP / KM_ELOC:
      // one phase of step P.st)
      const double sqt = sqrt(P.tau);
      double nacc = 0, natt = 0;
      double sw = 0, swe = 0, swk = 0, swv = 0, swnl = 0, swe2 = 0, nbad = 0, npts = 0;
      double u[10] = {0, 0, 0, 0, 0, 0, 0, 0, 0, 0};  // unweighted sums of E, E^2, T, T^2, V, V^2, NL, NL^2, w, w^2
      const double etr = P.dmc ? *P.etrial : 0.0;
      const double teff = P.dmc ? P.etrial[1] : 0.0;
      const int st0 = mode == KM_STEPS ? 0 : P.st, st1 = mode == KM_STEPS ? P.nsteps : P.st + 1;
      for (int st = st0; st < st1; st++) {
        const uint64_t step = step0 + st;
        if constexpr (!ELOCM) {
          const int e_lo = tc_phase ? P.tc_e : 0, e_hi = tc_phase ? P.tc_e + 1 : N;
          float pga[3] = {0.0f, 0.0f, 0.0f};  // lane k: deviates of electron e + k of the current 32
          double prb = 0.0;                   // and its acceptance number
          for (int e = e_lo; e < e_hi; e++) {
            // Split_sampler::split_driver depth 1 (Split_sample.cpp:380-478)
            if (((e - e_lo) & 31) == 0) {
              // the proposal deviates and acceptance numbers of the next 32
              // electrons, one electron per lane (the same counter-based
              // streams as drawing them electron by electron)
              const int ee = e + lane;
              if (ee < e_hi) {
                const Rand4 ra = rand4(P.seed, wid, step, ee, 1u);
                const Rand4 rb = rand4(P.seed, wid, step, ee, 2u);
                double g[4];
                box_muller(ra.u[0], ra.u[1], g[0], g[1]);
                box_muller(ra.u[2], ra.u[3], g[2], g[3]);
                pga[0] = float(g[0]); pga[1] = float(g[1]); pga[2] = float(g[2]);  // exact: FP32 deviates
                prb = rb.u[0];
              }
            }
            const int src = (e - e_lo) & 31;
            const double ga[3] = {double(__shfl_sync(0xffffffffu, pga[0], src)),
                                  double(__shfl_sync(0xffffffffu, pga[1], src)),
                                  double(__shfl_sync(0xffffffffu, pga[2], src))};
            const double rbu = __shfl_sync(0xffffffffu, prb, src);
            double g0[3], l0;
            W.electron_grad(e, g0, l0);
            double dv[3];
            lim_drift(g0, P.tau, dv);
            const double ox = Rp[3 * e], oy = Rp[3 * e + 1], oz = Rp[3 * e + 2];
            double nx = ox + ga[0] * sqt + dv[0];
            double ny = oy + ga[1] * sqt + dv[1];
            double nz = oz + ga[2] * sqt + dv[2];
            double wx = nx, wy = ny, wz = nz;  // the stored position is inside the cell
            double node = 1.0;  // sign of the continuous ratio across the wrap (complex kernels)
            if constexpr (CPXK) {
              const double kd = wrap_pos_kphase(S, wx, wy, wz);
              if (S.kint) node = cos(kd);  // overall sign of Periodic_sample::translateElectron
            } else {
              wrap_pos(S, wx, wy, wz);
            }
            if (tc_phase == 1) {
              // basis rows of the proposed position -> split-TF32 A rows of
              // this walker (rows wid * 5 + component)
              Real* b = W.bas();
              basis_lap_warp<Real, PER, (MMAX < 0 || (MMAX == 0 && XL))>(S, wx, wy, wz, b, lane);
              float* ah = P.tc_ahi + (size_t)wid * 5 * P.tc_kpad;
              float* al = P.tc_alo + (size_t)wid * 5 * P.tc_kpad;
              for (int idx = lane; idx < 5 * P.tc_kpad; idx += 32) {
                const int c = idx / P.tc_kpad, f = idx - c * P.tc_kpad;
                const float v = f < S.nbasis ? float(b[(size_t)f * 5 + c]) : 0.0f;
                float hi, lo;
                tc_split_tf32(v, hi, lo);
                ah[idx] = hi;
                al[idx] = lo;
              }
              continue;
            }
            double ratioD, dU, g1[3], l1;
            W.propose(e, wx, wy, wz, ratioD, dU, g1, l1);
            if constexpr (CPXK)
              if (S.real_orb && W.cr_re < 0) node = -node;
            // get_acceptance (Split_sample.cpp:302-373): psi ratio squared
            // times the ratio of drift-diffusion Green's functions
            double ratio = ratioD * exp(dU);
            double acc;
            if (P.dmc && (ratio < 0 || node < 0)) acc = 0;  // node restriction
            else {
              double bd[3];
              lim_drift(g1, P.tau, bd);
              double fw = 0, bw = 0;
              fw -= (nx - ox - dv[0]) * (nx - ox - dv[0]) + (ny - oy - dv[1]) * (ny - oy - dv[1]) +
                    (nz - oz - dv[2]) * (nz - oz - dv[2]);
              bw -= (ox - nx - bd[0]) * (ox - nx - bd[0]) + (oy - ny - bd[1]) * (oy - ny - bd[1]) +
                    (oz - nz - bd[2]) * (oz - nz - bd[2]);
              acc = fmin(1.0, ratio * ratio * exp((bw - fw) / (2.0 * P.tau)));
            }
            natt += 1;
            if (acc + rbu > 1.0) {
              QWG_PHASE_BEGIN(t_acc)
              W.accept(e, wx, wy, wz, ratioD, dU);
              QWG_PHASE_END(t_acc, PH_ACCEPT, P.phases)
              nacc += 1;
            } else if constexpr (mode == KM_STEPS) {
              if (!P.dmc && P.vmc_depth > 1) {
                // delayed rejection, second stage (Split_sampler::split_driver
                // depth 2, Split_sample.cpp:380-478): a new move from the same
                // point with timestep tau2 = tau / divider, accepted with
                // get_acceptance(0, 2) (Split_sample.cpp:302-373)
                const double tau2 = P.tau / P.vmc_divider;
                double dv2[3];
                lim_drift(g0, tau2, dv2);
                const Rand4 rc = rand4(P.seed, wid, step, e, 4u);
                const Rand4 rd = rand4(P.seed, wid, step, e, 5u);
                double gb[4];
                box_muller(rc.u[0], rc.u[1], gb[0], gb[1]);
                box_muller(rc.u[2], rc.u[3], gb[2], gb[3]);
                const double sq2 = sqrt(tau2);
                const double x2[3] = {ox + gb[0] * sq2 + dv2[0], oy + gb[1] * sq2 + dv2[1], oz + gb[2] * sq2 + dv2[2]};
                double vx = x2[0], vy = x2[1], vz = x2[2];
                if constexpr (CPXK) wrap_pos_kphase(S, vx, vy, vz);
                else wrap_pos(S, vx, vy, vz);
                double r2D, dU2, g2[3], l2;
                W.propose(e, vx, vy, vz, r2D, dU2, g2, l2);
                const double ratio2 = r2D * exp(dU2);  // psi(x2) / psi(x0)
                const double x1[3] = {nx, ny, nz}, x0[3] = {ox, oy, oz};
                // ln T(a -> b; t) = -|b - a - limdrift(drift_a, t)|^2 / (2 t)
                auto lnT = [&](const double* a, const double* ga, const double* b, double t) {
                  double d[3];
                  lim_drift(ga, t, d);
                  double q = 0;
                  for (int k = 0; k < 3; k++) q += (b[k] - a[k] - d[k]) * (b[k] - a[k] - d[k]);
                  return -q / (2.0 * t);
                };
                // a(2 -> 1): the reverse first stage from x2
                const double r21 = ratio / ratio2;
                const double a21 = fmin(1.0, r21 * r21 * exp(lnT(x1, g1, x2, P.tau) - lnT(x2, g2, x1, P.tau)));
                const double num = 1.0 - a21, den = 1.0 - acc;
                double acc2;
                if (fabs(den) < 1e-10) acc2 = fabs(num) < 1e-10 ? 0.0 : 1.0;
                else {
                  const double pt = lnT(x2, g2, x1, P.tau) - lnT(x0, g0, x1, P.tau) + lnT(x2, g2, x0, tau2) -
                                    lnT(x0, g0, x2, tau2);
                  acc2 = fmin(1.0, ratio2 * ratio2 * exp(pt) * num / den);
                }
                if (acc2 + rd.u[0] > 1.0) {
                  W.accept(e, vx, vy, vz, r2D, dU2);
                  nacc += 1;
                }
              }
            }
          }
        }
        if constexpr (mode != KM_SWEEP) {
          // gatherData (Properties_gather.cpp:40-74)
          Rand4 rr = rand4(P.seed, wid, step, 0xffffu, 3u);
          double rm[9];
          random_rotation(rr, rm);
          QWG_PHASE_BEGIN(t_kin)
          double kin = W.kinetic();
          QWG_PHASE_END(t_kin, PH_KINETIC, P.phases)
          QWG_PHASE_BEGIN(t_pot)
          double pot = W.coulomb();
          QWG_PHASE_END(t_pot, PH_POTENTIAL, P.phases)
          double nl = 0.0;
          if (S.has_pp) {
            if constexpr (mode == KM_ELOC_TM)
              nl = W.template pseudo<true>(rm, P.deterministic_pp != 0, P.seed, wid, step, P.tmoves, P.tau,
                                           P.tm_cand + (size_t)wid * P.tm_cap, P.tm_moves + (size_t)wid * N * 4);
            else
              nl = W.pseudo(rm, P.deterministic_pp != 0, P.seed, wid, step);
          }
          double el = kin + pot + nl;
          WScal* w = W.sc();
          double wt = 1.0;
          if (P.dmc) {
            // Dmc_method::getWeight (Dmc_method.cpp:801-824) + weight clamp
            double eold = w->eold;
            double teffac = teff / 2.0;
            double fbet = fmax(etr - el, etr - eold);
            if (fbet > P.branch_stop) teffac = 0;
            else if (fbet > P.branch_start)
              teffac = teffac * (1. - (fbet - P.branch_start) / (P.branch_stop - P.branch_start));
            wt = w->weight * exp(teffac * (etr * 2 - el - eold));
            if (wt > P.max_weight) wt = P.max_weight;
            if (!isfinite(el) || !isfinite(wt)) { nbad += 1; wt = 0.0; el = etr; }
            __syncwarp();
            if (lane == 0) { w->weight = wt; w->eold = el; }
            __syncwarp();
          } else {
            if (!isfinite(el)) { nbad += 1; el = 0.0; wt = 0.0; }
            if (lane == 0) w->eold = el;
          }
          sw += wt; swe += wt * el; swk += wt * kin; swv += wt * pot; swnl += wt * nl; swe2 += wt * el * el;
          u[0] += el; u[1] += el * el; u[2] += kin; u[3] += kin * kin; u[4] += pot; u[5] += pot * pot;
          u[6] += nl; u[7] += nl * nl; u[8] += wt; u[9] += wt * wt;
          npts += 1;
        }
      }
      QWG_PHASE_END(t_walker, PH_WALKER, P.phases)
      if (lane == 0) {
        if (!ELOCM) { atomicAdd(&cta_acc[6], nacc); atomicAdd(&cta_acc[7], natt); }
        if (mode != KM_SWEEP) {
          atomicAdd(&cta_acc[0], sw); atomicAdd(&cta_acc[1], swe); atomicAdd(&cta_acc[2], swk);
          atomicAdd(&cta_acc[3], swv); atomicAdd(&cta_acc[4], swnl); atomicAdd(&cta_acc[5], swe2);
          atomicAdd(&cta_acc[8], nbad);
          atomicAdd(&cta_acc[9], npts);
          for (int k = 0; k < 10; k++) atomicAdd(&cta_acc[10 + k], u[k]);
          if (io.energy) io.energy[wid] = W.sc()->eold;
        }
      }
      // write back: positions and the resident state after moves; only the
      // walker scalars after a local-energy pass
      __syncwarp();
      if (!ELOCM)
        for (int i = lane; i < 3 * N; i += 32) P.R[(size_t)wid * 3 * N + i] = Rp[i];
      if constexpr (!HBM) {
        int4* dst = (int4*)gstate;
        const int4* src = (const int4*)wb;
        if (ELOCM) {
          for (int i = lane; i < (int)sizeof(WScal) / 16; i += 32) ((int4*)(gstate + L.scal))[i] = ((const int4*)(wb + L.scal))[i];
        } else {
          for (int i = lane; i < L.state_bytes / 16; i += 32) dst[i] = src[i];
        }
      }
    }
  }
  if constexpr (mode == KM_STEPS || mode == KM_SWEEP || mode == KM_ELOC || mode == KM_ELOC_TM) {
    __syncthreads();
    if (threadIdx.x < QWG_NACC) atomicAdd(&((double*)P.acc)[threadIdx.x], cta_acc[threadIdx.x]);
  }
}

#ifndef QWG_WALKERS_ONLY  // population-control kernels live in the engine translation unit
// ---------------------------------------------------------------------------
// DMC population control on one CTA: E_T feedback (Dmc_method::updateEtrial,
// :780-797), constant-population split/kill pairing (match_walkers,
// :961-995), and the copy order of calcBranch (:1099-1107): survivors in
// walker order, each repeated by its branch count.
//
// dyn[0] = E_T, dyn[1] = teff, dyn[2] = sum of weights, dyn[3] = branched pairs
struct BranchParams {
  int nwalk, npow2;
  int nsteps;             // steps of the chunk just finished (advances the step counter)
  double feedback, timestep;
  uint64_t seed;
  const unsigned char* state;
  int state_bytes, scal_off;
  const BlockAcc* acc;    // running acceptance of this chunk
  double* dyn;
  int* src_of;            // [W] output mapping
  double* new_w;          // [W] weight of the slot after branching
  // sort keys and counts in global memory (large populations); null: in
  // dynamic shared memory
  double* gkey;           // [npow2]
  int* gidx;              // [npow2]
  int* gcnt;              // [nwalk]
  double* gnw;            // [nwalk]
};

__global__ void __launch_bounds__(1024) k_branch(BranchParams B) {
  extern __shared__ __align__(16) unsigned char sm[];
  double* key = B.gkey ? B.gkey : (double*)sm;                 // [npow2]
  int* idx = B.gkey ? B.gidx : (int*)(key + B.npow2);          // [npow2]
  int* cnt = B.gkey ? B.gcnt : idx + B.npow2;                  // [nwalk]
  double* nw = B.gkey ? B.gnw : (double*)(((uintptr_t)(cnt + B.nwalk) + 15) & ~(uintptr_t)15);  // [nwalk]
  __shared__ double red[32];
  const int t = threadIdx.x, nt = blockDim.x;
  double local = 0;
  for (int i = t; i < B.npow2; i += nt) {
    double w = 1e300;
    if (i < B.nwalk) {
      w = ((const WScal*)(B.state + (size_t)i * B.state_bytes + B.scal_off))->weight;
      local += w;
      cnt[i] = 1;
      nw[i] = w;
    }
    key[i] = w;
    idx[i] = i;
  }
  local = warp_sum(local);
  if ((t & 31) == 0) red[t >> 5] = local;
  __syncthreads();
  if (t < 32) {
    double v = (t < nt / 32) ? red[t] : 0.0;
    v = warp_sum(v);
    if (t == 0) {
      double acc_ratio = B.acc->attempted > 0 ? B.acc->accepted / B.acc->attempted : 1.0;
      B.dyn[DYN_TEFF] = B.timestep * acc_ratio;
      B.dyn[DYN_ETRIAL] = B.dyn[DYN_EREF] - B.feedback * log(v / double(B.nwalk));
      B.dyn[DYN_SUMW] = v;
    }
  }
  // bitonic sort ascending by weight (ties by index)
  for (int k = 2; k <= B.npow2; k <<= 1) {
    for (int j = k >> 1; j > 0; j >>= 1) {
      __syncthreads();
      for (int i = t; i < B.npow2; i += nt) {
        int ixj = i ^ j;
        if (ixj > i) {
          bool up = (i & k) == 0;
          double a = key[i], b = key[ixj];
          int ia = idx[i], ib = idx[ixj];
          bool gt = a > b || (a == b && ia > ib);
          if (gt == up) { key[i] = b; key[ixj] = a; idx[i] = ib; idx[ixj] = ia; }
        }
      }
    }
  }
  __syncthreads();
  // pairs k: the k-th largest (while >= 1.8) with the k-th smallest
  const int W = B.nwalk;
  int npair = 0;
  for (int k = t; k < W / 2; k += nt) {
    int big = W - 1 - k;
    if (big > 1 && key[big] >= 1.8 && k < big) {
      // all larger slots also qualify (sorted), so pair k is taken
      int wb = idx[big], ws = idx[k];
      double w1 = key[big], w2 = key[k];
      double weight1 = w1 / (w1 + w2);
      Rand4 r = rand4(B.seed, (uint32_t)k, (uint64_t)B.dyn[DYN_BRANCH], 0u, 5u);
      double merged = (w1 + w2) / 2.0;
      if (weight1 + r.u[0] >= 1.0) { cnt[wb] = 2; cnt[ws] = 0; nw[wb] = merged; }
      else { cnt[wb] = 0; cnt[ws] = 2; nw[ws] = merged; }
      npair++;
    }
  }
  __syncthreads();
  // exclusive prefix sum of counts in walker order (single pass per thread chunk)
  __shared__ int chunk_sum[1024];
  const int per = (W + nt - 1) / nt;
  int s0 = t * per, s1 = min(W, s0 + per), cs = 0;
  for (int i = s0; i < s1; i++) cs += cnt[i];
  chunk_sum[t] = cs;
  __syncthreads();
  if (t == 0) {
    int run = 0;
    for (int i = 0; i < nt; i++) { int v = chunk_sum[i]; chunk_sum[i] = run; run += v; }
  }
  __syncthreads();
  int off = chunk_sum[t];
  for (int i = s0; i < s1; i++) {
    for (int c = 0; c < cnt[i]; c++) {
      if (off < W) { B.src_of[off] = i; B.new_w[off] = nw[i]; }
      off++;
    }
  }
  if (npair) atomicAdd(&B.dyn[DYN_PAIRS], double(npair));
  __syncthreads();
  if (t == 0) {  // every thread has read the counters above
    B.dyn[DYN_STEP] += double(B.nsteps);
    B.dyn[DYN_BRANCH] += 1.0;
  }
}

// ---------------------------------------------------------------------------
// Population control for large populations (more walkers than the one-CTA
// kernel keeps in shared memory): the same E_T feedback, pairing and copy
// order as k_branch, with the sort of the weights done device-wide.
//   k_branch_prep    counts 1, new weights, 64-bit sort keys (the bits of a
//                    non-negative double order like the value) and walker
//                    indices; per-CTA weight sums
//   k_radix_hist / k_radix_scan / k_radix_scatter   one stable LSD pass of
//                    8 bits over (key, index) pairs: per-tile digit counts,
//                    their digit-major exclusive scan, and the scatter with
//                    in-tile ranks in element order (ties stay in index
//                    order, as the one-CTA sort breaks them); 8 passes
//   k_branch_pairs   pair k: the k-th heaviest (while >= 1.8) with the k-th
//                    lightest, the split/kill draw of k_branch
//   k_branch_finish  (one CTA) E_T feedback from the weight sum, exclusive
//                    prefix sum of the counts in walker order into the gather
//                    map, counters
constexpr int RADIX_TILE = 2048;  // elements per CTA (256 threads x 8)

struct BranchBig {
  unsigned long long* key[2];  // [W] double buffers of the sort
  int* idx[2];                 // [W]
  int* cnt;                    // [W]
  double* nw;                  // [W]
  int* hist;                   // [256][ntiles] digit counts, then their offsets
  double* psum;                // [prep CTAs] weight sums
  int* npair;                  // [pair CTAs] pairs
  int ntiles, nprep, npairblk;
};

__global__ void __launch_bounds__(256) k_branch_prep(BranchParams B, BranchBig G) {
  __shared__ double red[8];
  const int i = blockIdx.x * 256 + threadIdx.x;
  double w = 0.0;
  if (i < B.nwalk) {
    w = ((const WScal*)(B.state + (size_t)i * B.state_bytes + B.scal_off))->weight;
    G.cnt[i] = 1;
    G.nw[i] = w;
    G.key[0][i] = (unsigned long long)__double_as_longlong(w);
    G.idx[0][i] = i;
  }
  double v = warp_sum(w);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0;
    for (int k = 0; k < 8; k++) t += red[k];
    G.psum[blockIdx.x] = t;
  }
}

__global__ void __launch_bounds__(256) k_radix_hist(const unsigned long long* key, int n, int shift, int* hist,
                                                    int ntiles) {
  __shared__ int cnt[256];
  cnt[threadIdx.x] = 0;
  __syncthreads();
  const int base = blockIdx.x * RADIX_TILE;
  for (int j = 0; j < RADIX_TILE / 256; j++) {
    const int e = base + j * 256 + threadIdx.x;
    if (e < n) atomicAdd(&cnt[(int)((key[e] >> shift) & 255ull)], 1);
  }
  __syncthreads();
  hist[threadIdx.x * ntiles + blockIdx.x] = cnt[threadIdx.x];
}

// exclusive scan of hist[256 * ntiles] in place (digit-major), one CTA
__global__ void __launch_bounds__(1024) k_radix_scan(int* hist, int total) {
  __shared__ int part[1024];
  const int per = (total + 1023) / 1024;
  const int s0 = threadIdx.x * per, s1 = min(total, s0 + per);
  int run = 0;
  for (int i = s0; i < s1; i++) run += hist[i];
  part[threadIdx.x] = run;
  __syncthreads();
  for (int o = 1; o < 1024; o <<= 1) {  // inclusive Hillis-Steele scan of the chunk sums
    int v = threadIdx.x >= o ? part[threadIdx.x - o] : 0;
    __syncthreads();
    part[threadIdx.x] += v;
    __syncthreads();
  }
  int off = threadIdx.x ? part[threadIdx.x - 1] : 0;
  for (int i = s0; i < s1; i++) {
    const int v = hist[i];
    hist[i] = off;
    off += v;
  }
}

__global__ void __launch_bounds__(256) k_radix_scatter(const unsigned long long* kin, const int* iin,
                                                       unsigned long long* kout, int* iout, int n, int shift,
                                                       const int* off, int ntiles) {
  __shared__ int wcount[8][256];
  __shared__ int run[256];
  const int t = threadIdx.x, warp = t >> 5, lane = t & 31;
  run[t] = 0;
  const int base = blockIdx.x * RADIX_TILE;
  const unsigned lt = (1u << lane) - 1u;
  for (int j = 0; j < RADIX_TILE / 256; j++) {
    for (int k = t; k < 8 * 256; k += 256) (&wcount[0][0])[k] = 0;
    __syncthreads();
    const int e = base + j * 256 + t;
    const bool valid = e < n;
    unsigned long long key = 0;
    int d = 256;  // invalid lanes share a digit no valid lane has
    if (valid) {
      key = kin[e];
      d = (int)((key >> shift) & 255ull);
    }
    const unsigned m = __match_any_sync(0xffffffffu, d);
    const int lrank = __popc(m & lt);
    if (valid && lrank == 0) wcount[warp][d] = __popc(m);
    __syncthreads();
    if (valid) {
      int before = 0;
      for (int w = 0; w < warp; w++) before += wcount[w][d];
      const int pos = off[d * ntiles + blockIdx.x] + run[d] + before + lrank;
      kout[pos] = key;
      iout[pos] = iin[e];
    }
    __syncthreads();
    int sd = 0;
    for (int w = 0; w < 8; w++) sd += wcount[w][t];
    run[t] += sd;
    __syncthreads();
  }
}

__global__ void __launch_bounds__(256) k_branch_pairs(BranchParams B, BranchBig G, int sorted) {
  __shared__ int red[8];
  const unsigned long long* key = G.key[sorted];
  const int* idx = G.idx[sorted];
  const int W = B.nwalk;
  const int k = blockIdx.x * 256 + threadIdx.x;
  int paired = 0;
  if (k < W / 2) {
    const int big = W - 1 - k;
    const double w1 = __longlong_as_double((long long)key[big]);
    if (big > 1 && w1 >= 1.8 && k < big) {
      const int wb = idx[big], ws = idx[k];
      const double w2 = __longlong_as_double((long long)key[k]);
      const double weight1 = w1 / (w1 + w2);
      Rand4 r = rand4(B.seed, (uint32_t)k, (uint64_t)B.dyn[DYN_BRANCH], 0u, 5u);
      const double merged = (w1 + w2) / 2.0;
      if (weight1 + r.u[0] >= 1.0) { G.cnt[wb] = 2; G.cnt[ws] = 0; G.nw[wb] = merged; }
      else { G.cnt[wb] = 0; G.cnt[ws] = 2; G.nw[ws] = merged; }
      paired = 1;
    }
  }
  const int c = __reduce_add_sync(0xffffffffu, paired);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = c;
  __syncthreads();
  if (threadIdx.x == 0) {
    int t = 0;
    for (int w = 0; w < 8; w++) t += red[w];
    G.npair[blockIdx.x] = t;
  }
}

__global__ void __launch_bounds__(1024) k_branch_finish(BranchParams B, BranchBig G) {
  __shared__ int chunk_sum[1024];
  const int t = threadIdx.x, nt = blockDim.x, W = B.nwalk;
  if (t == 0) {
    double v = 0;
    for (int b = 0; b < G.nprep; b++) v += G.psum[b];
    double acc_ratio = B.acc->attempted > 0 ? B.acc->accepted / B.acc->attempted : 1.0;
    B.dyn[DYN_TEFF] = B.timestep * acc_ratio;
    B.dyn[DYN_ETRIAL] = B.dyn[DYN_EREF] - B.feedback * log(v / double(W));
    B.dyn[DYN_SUMW] = v;
    int np = 0;
    for (int b = 0; b < G.npairblk; b++) np += G.npair[b];
    if (np) B.dyn[DYN_PAIRS] += double(np);
  }
  const int per = (W + nt - 1) / nt;
  const int s0 = t * per, s1 = min(W, s0 + per);
  int cs = 0;
  for (int i = s0; i < s1; i++) cs += G.cnt[i];
  chunk_sum[t] = cs;
  __syncthreads();
  if (t == 0) {
    int run = 0;
    for (int i = 0; i < nt; i++) { const int v = chunk_sum[i]; chunk_sum[i] = run; run += v; }
  }
  __syncthreads();
  int off = chunk_sum[t];
  for (int i = s0; i < s1; i++)
    for (int c = 0; c < G.cnt[i]; c++) {
      if (off < W) { B.src_of[off] = i; B.new_w[off] = G.nw[i]; }
      off++;
    }
  __syncthreads();
  if (t == 0) {
    B.dyn[DYN_STEP] += double(B.nsteps);
    B.dyn[DYN_BRANCH] += 1.0;
  }
}

// Gather walkers into their new slots (positions + resident state).
__global__ void k_gather(int nwalk, int n3, int state_bytes, int scal_off, const int* src_of, const double* new_w,
                         const double* R, const unsigned char* state, double* R2, unsigned char* state2) {
  const int w = blockIdx.x;
  if (w >= nwalk) return;
  const int s = src_of[w];
  for (int i = threadIdx.x; i < n3; i += blockDim.x) R2[(size_t)w * n3 + i] = R[(size_t)s * n3 + i];
  const int4* src = (const int4*)(state + (size_t)s * state_bytes);
  int4* dst = (int4*)(state2 + (size_t)w * state_bytes);
  for (int i = threadIdx.x; i < state_bytes / 16; i += blockDim.x) dst[i] = src[i];
  __syncthreads();
  if (threadIdx.x == 0) ((WScal*)(state2 + (size_t)w * state_bytes + scal_off))->weight = new_w[w];
}

// End of a DMC block: block averages from the per-chunk accumulators, the
// block-energy history, E_ref = mean block energy (the first fifth of the
// blocks dropped as equilibration once there are more than five), and E_T
// (Dmc_method.cpp:475-530).  out[0..QWG_NACC-1]: the BlockAcc sums of the
// block; out[QWG_NACC] = E_T, out[QWG_NACC + 1] = E_ref.
__global__ void k_block_end(const BlockAcc* acc, int nchunk, double* dyn, double* hist, int hist_cap,
                            double feedback, int nwalk, double* out) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double t[QWG_NACC] = {0};
  for (int c = 0; c < nchunk; c++) {
    const double* a = (const double*)(acc + c);
    for (int k = 0; k < QWG_NACC; k++) t[k] += a[k];
  }
  const double eb = t[0] > 0 ? t[1] / t[0] : 0.0;
  const int nb = (int)dyn[DYN_NBLOCK];
  hist[nb % hist_cap] = eb;
  const int n = nb + 1;
  dyn[DYN_NBLOCK] = double(n);
  const int b0 = n > 5 ? n / 5 : 0;
  const int lo = max(b0, n - hist_cap);
  double se = 0;
  for (int b = lo; b < n; b++) se += hist[b % hist_cap];
  const double eref = se / double(n - lo);
  dyn[DYN_EREF] = eref;
  dyn[DYN_ETRIAL] = eref - feedback * log(dyn[DYN_SUMW] / double(nwalk));
  for (int k = 0; k < QWG_NACC; k++) out[k] = t[k];
  out[QWG_NACC] = dyn[DYN_ETRIAL];
  out[QWG_NACC + 1] = eref;
}

__global__ void k_init_weights(unsigned char* state, int nwalk, int state_bytes, int scal_off, const double* eloc) {
  int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= nwalk) return;
  WScal* s = (WScal*)(state + (size_t)w * state_bytes + scal_off);
  s->weight = 1.0;
  s->eold = eloc[w];
}

#endif  // QWG_WALKERS_ONLY

}  // namespace qwg
