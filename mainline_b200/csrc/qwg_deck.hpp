// Host side of the walker engine: QWalk input grammar and the flat tables the
// kernels consume.  Built once per context on the host, then uploaded.
#pragma once
#include <string>
#include <vector>
#include <stdexcept>

namespace qwg {

struct InputError : std::runtime_error {
  explicit InputError(const std::string& m) : std::runtime_error(m) {}
};

// Token list of a QWalk input file: '{' and '}' are words of their own, '#'
// starts a comment, INCLUDE <file> splices another file in place
// (program_utils/qmc_io.cpp:280-345).
std::vector<std::string> tokenize_file(const std::string& path);

// Level-0 section / value lookups (program_utils/qmc_io.cpp:168-230,
// qmc_io.h:62-124).  Keys compare case-insensitively.
bool find_section(const std::vector<std::string>& w, const std::string& name, size_t& pos,
                  std::vector<std::string>& out);
std::vector<std::vector<std::string>> all_sections(const std::vector<std::string>& w, const std::string& name);
bool has_section(const std::vector<std::string>& w, const std::string& name);
bool find_value(const std::vector<std::string>& w, const std::string& name, std::string& out);
bool has_keyword(const std::vector<std::string>& w, const std::string& name);

// Angular sets of Cubic_spline (basis_function/Cubic_spline_build.cpp:26-140,
// 660-790): F and G shells in Cartesian (10F, 15G), real-harmonic (7F, 9G) and
// CRYSTAL (7F_crystal) orders.
enum ShellSym {
  SYM_S = 0, SYM_P = 1, SYM_6D = 2, SYM_5D = 3, SYM_10F = 4, SYM_7F = 5, SYM_7F_CRYSTAL = 6, SYM_15G = 7, SYM_9G = 8
};
enum RadialKind { RAD_CUTOFF_CUSP = 0, RAD_POLYPADE = 1, RAD_PADE = 2 };

// One radial spline x Cartesian angular set attached to one center.
struct Shell {
  int center;      // atom index
  int spline;      // radial table index
  int sym;         // ShellSym
  int first;       // first basis function (global index)
  int nfunc;
  double cutoff;   // basis-object threshold: r >= cutoff gives zero
  double fcut;     // the spline's own cutoff (CUTOFF_MO evaluates a function only inside it)
  int obj;         // basis object (BASIS section) the spline belongs to
  int k;           // spline index inside its basis object
};

// A scalar Jastrow radial function (f, f'/r, lap).
struct Radial {
  int kind;        // RadialKind
  double rcut;
  double a, b;     // CUTOFF_CUSP: cusp, gamma ; POLYPADE: beta, unused
};

struct ThreeBodyTerm {
  int k, l, m;     // global e-n (per atom) function indices k,l and e-e index m
  double c;        // coefficient for electron pairs of equal spin
  double cu;       // coefficient for pairs of opposite spin (= c unless THREEBODY_SPIN)
};

struct PPAtom {
  int nchan = 0;                 // channels incl. the local one (last)
  int aip = 0;                   // quadrature points
  double cutoff = 0.0;           // nonlocal evaluation radius
  std::vector<int> term_first;   // [nchan+1] terms of each channel for spin-up electrons
  std::vector<int> term_first_dn;  // [nchan+1] for spin-down electrons (= term_first unless SPIN_DEP)
  bool add_zeff = false;         // ADD_ZEFF: the local channel also carries +Z_ion / r
  std::vector<double> term_n;    // r power (already n-2)
  std::vector<double> term_a;    // Gaussian exponent
  std::vector<double> term_c;    // coefficient
  std::vector<double> quad;      // [aip][3]
  std::vector<double> weight;    // [aip]
};

struct HostSystem {
  std::string deck_path;
  int nup = 0, ndn = 0, nelec = 0, natoms = 0;
  std::vector<std::string> labels;
  std::vector<double> atom_pos;      // [A][3]
  std::vector<double> atom_charge;   // [A]
  double ion_ion = 0.0;
  // basis
  std::vector<Shell> shells;
  int nbasis = 0;
  int nspline = 0, spline_npts = 0;
  double spline_spacing = 0.02;
  std::vector<double> spline_coef;   // [nspline][npts][4]
  std::vector<int> obj_first, obj_count;   // per basis object: its splines
  // molecular orbitals per spin: [nbasis][nmo_s], the union of the orbitals
  // the determinants of that spin occupy (one determinant: its occupied
  // orbitals in STATES order)
  int nmo[2] = {0, 0};
  std::vector<double> moc[2];
  // complex orbitals (CORBITALS, Slat_wf<dcomplex>): imaginary parts of moc,
  // same layout; real orbitals with a nonzero k-point also run on the complex
  // kernels (moc_im zero, real k-point factors)
  bool complex_orbitals = false;
  bool cutoff_mo = false;            // CUTOFF_MO evaluator (else BLAS_MO)
  std::vector<double> moc_im[2];
  double kpt[3] = {0, 0, 0};         // KPOINT (units of pi / lattice vector)
  // determinant expansion sum_k detwt[k] D_up(det_ud[k][0]) D_down(det_ud[k][1])
  // over the distinct spin-determinants; udet_cols[s][u] = the union columns
  // of spin-determinant u in STATES order (Slat_wf_data.cpp:34-303)
  int nel_s[2] = {0, 0};             // electrons per spin
  std::vector<double> detwt;         // [ndet]
  std::vector<int> det_ud;           // [ndet][2]
  std::vector<std::vector<int>> udet_cols[2];
  // Jastrow
  std::vector<Radial> ee;            // global e-e function list
  std::vector<double> ee_like, ee_unlike;  // two-body coefficients per ee function
  std::vector<Radial> ei;            // global e-n function list
  std::vector<int> ei_first, ei_count;     // per atom slice into ei
  std::vector<double> onebody;       // per ei function (already per atom slice)
  std::vector<int> tb_first, tb_count;     // per atom slice into tb
  std::vector<ThreeBodyTerm> tb;
  // THREEBODY_SPIN present and no plain THREEBODY group: the reference's
  // value-only Jastrow update leaves the moved electron's e-n basis values
  // stale for the e-e-n terms (see DevSys::tb_stale_ei)
  bool tb_stale_ei = false;
  // periodic cell (SYSTEM { PERIODIC }); molecules keep periodic == false and
  // one "image" per atom (the atom itself)
  bool periodic = false;
  double lat[9] = {0}, origin[3] = {0}, normvec[9] = {0}, corners[9] = {0};
  double smallest_height = 0, alpha = 0, volume = 0;
  std::vector<double> lattice_basis;   // [27][3] minimum-image search
  std::vector<double> image_pos;       // [nimage][3] image centers of all atoms
  std::vector<int> image_first, image_count;  // per atom slice of image_pos
  std::vector<int> image_shift;        // [nimage][3] lattice translation of each image center
  std::vector<double> gvec, gweight, ion_sin, ion_cos;  // Ewald G-vectors [G][3], [G]
  double ewald_const = 0;              // ion-ion Ewald + self/background terms
  // pseudopotential (per atom; nchan == 0 if none)
  std::vector<PPAtom> pp;
  bool has_pp = false;
  int max_aip = 0;
};

// Parse the deck and build every table (throws InputError).
HostSystem build_system(const std::string& deck_path);

}  // namespace qwg
