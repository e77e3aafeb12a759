// QWalk input grammar + table builder for the walker engine.
//
// Module semantics follow the reference (QWalk/mainline src/):
//   grammar            program_utils/qmc_io.cpp:168-345
//   AOSPLINE basis     basis_function/Cubic_spline_build.cpp:139-660 (GAMESS
//                      shells, GAMESSNORM, numerical renormalisation, optional
//                      smooth CUTOFF, clamped cubic spline on a 0.02 grid)
//   spline fit/cutoff  basis_function/Spline_fitter.cpp:153-293
//   MO coefficients    orbitals/MO_matrix.h:264-332 (ORB file), MO_matrix_blas.h:101-190
//   occupations        wavefunction/Slat_wf_data.cpp:34-303 (STATES, one determinant)
//   Jastrow groups     wavefunction/Jastrow2_wf.cpp:29-160, Jastrow2_one.cpp:25-100,
//                      Jastrow2_two.cpp:28-45/220-245, Jastrow2_three.cpp:29-100
//   radial functions   basis_function/Cutoff_cusp.cpp:26-60,
//                      Poly_pade_function.cpp:26-85
//   pseudopotential    system/Pseudopotential.cpp:874-1033, Rgaussian_function.cpp:24-100
//   quadrature         system/gesqua.cpp:32-120
#include "qwg_deck.hpp"

#include <algorithm>
#include <cctype>
#include <array>
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <map>
#include <sstream>

namespace qwg {

static bool ieq(const std::string& a, const std::string& b) {
  if (a.size() != b.size()) return false;
  for (size_t i = 0; i < a.size(); i++)
    if (std::toupper((unsigned char)a[i]) != std::toupper((unsigned char)b[i])) return false;
  return true;
}

static std::string dirname_of(const std::string& p) {
  size_t k = p.find_last_of('/');
  return k == std::string::npos ? std::string(".") : p.substr(0, k);
}

static bool file_exists(const std::string& p) {
  std::ifstream f(p);
  return bool(f);
}

std::vector<std::string> tokenize_file(const std::string& path) {
  std::ifstream in(path);
  if (!in) throw InputError("cannot open " + path);
  std::vector<std::string> raw;
  std::string line;
  while (std::getline(in, line)) {
    size_t hash = line.find('#');
    if (hash != std::string::npos) line.erase(hash);
    std::istringstream ss(line);
    std::string tok;
    while (ss >> tok) {
      std::string buf;
      for (char ch : tok) {
        if (ch == '{' || ch == '}') {
          if (!buf.empty()) raw.push_back(buf);
          raw.push_back(std::string(1, ch));
          buf.clear();
        } else {
          buf.push_back(ch);
        }
      }
      if (!buf.empty()) raw.push_back(buf);
    }
  }
  std::vector<std::string> out;
  for (size_t i = 0; i < raw.size(); i++) {
    if (ieq(raw[i], "INCLUDE")) {
      if (i + 1 >= raw.size()) throw InputError("INCLUDE without a file name in " + path);
      std::string inc = raw[i + 1];
      if (inc[0] != '/' && !file_exists(inc)) inc = dirname_of(path) + "/" + inc;
      std::vector<std::string> sub = tokenize_file(inc);
      out.insert(out.end(), sub.begin(), sub.end());
      i++;
    } else {
      out.push_back(raw[i]);
    }
  }
  return out;
}

bool find_section(const std::vector<std::string>& w, const std::string& name, size_t& pos,
                  std::vector<std::string>& out) {
  out.clear();
  int level = 0;
  for (; pos < w.size(); pos++) {
    if (w[pos] == "{") level++;
    else if (w[pos] == "}") level--;
    if (level < 0) { pos++; return false; }
    if (level == 0 && ieq(w[pos], name)) {
      if (pos + 1 >= w.size() || w[pos + 1] != "{")
        throw InputError("section " + name + " must be followed by {");
      pos += 2;
      int depth = 0;
      for (; pos < w.size(); pos++) {
        if (w[pos] == "{") depth++;
        if (w[pos] == "}") { if (depth == 0) break; depth--; }
        out.push_back(w[pos]);
      }
      if (pos >= w.size()) throw InputError("unterminated section " + name);
      pos++;
      return true;
    }
  }
  return false;
}

std::vector<std::vector<std::string>> all_sections(const std::vector<std::string>& w, const std::string& name) {
  std::vector<std::vector<std::string>> res;
  size_t pos = 0;
  std::vector<std::string> s;
  while (find_section(w, name, pos, s)) res.push_back(s);
  return res;
}

bool has_section(const std::vector<std::string>& w, const std::string& name) {
  size_t pos = 0;
  std::vector<std::string> s;
  return find_section(w, name, pos, s);
}

static std::vector<std::string> get_section(const std::vector<std::string>& w, const std::string& name) {
  size_t pos = 0;
  std::vector<std::string> s;
  if (!find_section(w, name, pos, s)) throw InputError("missing section " + name);
  return s;
}

bool find_value(const std::vector<std::string>& w, const std::string& name, std::string& out) {
  int level = 0;
  for (size_t i = 0; i < w.size(); i++) {
    if (w[i] == "{") level++;
    else if (w[i] == "}") level--;
    if (level < 0) return false;
    if (level == 0 && ieq(w[i], name)) {
      if (i + 1 >= w.size()) throw InputError("keyword " + name + " without a value");
      out = w[i + 1];
      return true;
    }
  }
  return false;
}

bool has_keyword(const std::vector<std::string>& w, const std::string& name) {
  int level = 0;
  for (auto& t : w) {
    if (t == "{") level++;
    else if (t == "}") level--;
    if (level == 0 && ieq(t, name)) return true;
  }
  return false;
}

// Every number of a deck or orbital file: a non-finite value (nan, inf)
// would reach the device tables and turn every walker non-finite, so it is
// refused at read time.
static double to_d(const std::string& s) {
  char* end = nullptr;
  double v = std::strtod(s.c_str(), &end);
  if (end == s.c_str()) throw InputError("expected a number, got '" + s + "'");
  if (!std::isfinite(v)) throw InputError("non-finite number '" + s + "' in the input");
  return v;
}
static int to_i(const std::string& s) {
  char* end = nullptr;
  long v = std::strtol(s.c_str(), &end, 10);
  if (end == s.c_str()) throw InputError("expected an integer, got '" + s + "'");
  return (int)v;
}
static double value_d(const std::vector<std::string>& w, const std::string& k, double def, bool required = false) {
  std::string s;
  if (find_value(w, k, s)) return to_d(s);
  if (required) throw InputError("missing keyword " + k);
  return def;
}

// ---------------------------------------------------------------------------
// cubic spline (clamped, uniform grid)

static void spline_fit(const std::vector<double>& x, const std::vector<double>& y, double yp1, double ypn,
                       double* coef /* [n][4] */) {
  const int n = (int)x.size();
  std::vector<double> y2(n), u(n);
  if (yp1 > 0.99e30) {
    y2[0] = 0; u[0] = 0;
  } else {
    y2[0] = -0.5;
    u[0] = (3.0 / (x[1] - x[0])) * ((y[1] - y[0]) / (x[1] - x[0]) - yp1);
  }
  for (int i = 1; i < n - 1; i++) {
    double sig = (x[i] - x[i - 1]) / (x[i + 1] - x[i - 1]);
    double p = sig * y2[i - 1] + 2.0;
    y2[i] = (sig - 1.0) / p;
    u[i] = (6.0 * ((y[i + 1] - y[i]) / (x[i + 1] - x[i]) - (y[i] - y[i - 1]) / (x[i] - x[i - 1])) /
                (x[i + 1] - x[i - 1]) - sig * u[i - 1]) / p;
  }
  double qn, un;
  if (ypn > 0.99e30) { qn = 0; un = 0; }
  else {
    qn = 0.5;
    un = (3.0 / (x[n - 1] - x[n - 2])) * (ypn - (y[n - 1] - y[n - 2]) / (x[n - 1] - x[n - 2]));
  }
  y2[n - 1] = (un - qn * u[n - 2]) / (qn * y2[n - 2] + 1.0);
  for (int k = n - 2; k >= 0; k--) y2[k] = y2[k] * y2[k + 1] + u[k];
  for (int i = 0; i < n - 1; i++) {
    double h = x[i + 1] - x[i];
    coef[4 * i + 0] = y[i];
    coef[4 * i + 1] = (y[i + 1] - y[i]) / h - h * (2.0 * y2[i] + y2[i + 1]) / 6.0;
    coef[4 * i + 2] = y2[i] / 2.0;
    coef[4 * i + 3] = (y2[i + 1] - y2[i]) / (6.0 * h);
  }
  coef[4 * (n - 1) + 0] = y[n - 1];
  coef[4 * (n - 1) + 1] = coef[4 * (n - 1) + 2] = coef[4 * (n - 1) + 3] = 0.0;
}

// Largest r (0.5 bohr steps down from the grid end) where |f| exceeds
// 1e-10 * min(max|f|, 1).
static double spline_cutoff(const double* c, int n, double spacing, double threshold) {
  double mx = 0;
  for (int i = 0; i < n; i++) mx = std::max(mx, std::fabs(c[4 * i]));
  mx = std::min(mx, 1.0);
  const double thr = 1e-10 * mx;
  const double inv = 1.0 / spacing;
  for (double x = threshold - 0.5; x >= 0; x -= 0.5) {
    int i = int(x * inv);
    double h = x - i * spacing;
    double t = c[4 * i] + h * (c[4 * i + 1] + h * (c[4 * i + 2] + h * c[4 * i + 3]));
    if (std::fabs(t) > thr) return x + 0.5;
  }
  return 0.0;
}

static int sym_of(const std::string& s) {
  if (ieq(s, "S")) return SYM_S;
  if (ieq(s, "P")) return SYM_P;
  if (ieq(s, "D") || ieq(s, "6D")) return SYM_6D;
  if (ieq(s, "5D")) return SYM_5D;
  if (ieq(s, "F") || ieq(s, "10F")) return SYM_10F;
  if (ieq(s, "7F")) return SYM_7F;
  if (ieq(s, "7F_crystal")) return SYM_7F_CRYSTAL;
  if (ieq(s, "G") || ieq(s, "15G")) return SYM_15G;
  if (ieq(s, "9G")) return SYM_9G;
  throw InputError("unsupported AOSPLINE shell symmetry " + s +
                   " (supported: S P 5D 6D 7F 10F 7F_crystal 9G 15G)");
}
static int sym_nfunc(int s) {
  static const int nf[9] = {1, 3, 6, 5, 10, 7, 7, 15, 9};
  return nf[s];
}
static int sym_l(int s) {
  static const int l[9] = {0, 1, 2, 2, 3, 3, 3, 4, 4};
  return l[s];
}

struct BasisObj {
  std::string label;
  std::vector<int> syms;
  std::vector<int> spline_ids;  // into HostSystem::spline table
  double threshold = 0;
  std::vector<double> cuts;     // per spline (Spline_fitter::findCutoff)
  int nfunc = 0;
};

static BasisObj read_aospline(const std::vector<std::string>& w, HostSystem& S,
                              std::vector<std::vector<double>>& tables) {
  BasisObj B;
  if (w.size() < 2) throw InputError("empty BASIS section");
  B.label = w[0];
  if (!ieq(w[1], "AOSPLINE")) throw InputError("BASIS type " + w[1] + " not supported (AOSPLINE only)");
  double spacing = 0.02;
  int n = 2500;
  std::string ntype = "GAMESSNORM", tmp;
  if (find_value(w, "NORMTYPE", tmp)) ntype = tmp;
  bool renorm = !has_keyword(w, "NORENORMALIZE");
  double reqcut = value_d(w, "CUTOFF", -1.0);
  if (find_value(w, "SPACING", tmp)) { spacing = to_d(tmp); n = int(50.0 / spacing); }
  if (has_keyword(w, "CUSP") || has_keyword(w, "ZERO_DERIVATIVE"))
    throw InputError("AOSPLINE CUSP/ZERO_DERIVATIVE options are not supported");
  if (S.nspline > 0 && std::fabs(spacing - S.spline_spacing) > 1e-12)
    throw InputError("all AOSPLINE bases must share one SPACING");
  S.spline_spacing = spacing;
  auto g = get_section(w, "GAMESS");
  std::vector<double> x(n), y(n);
  for (int j = 0; j < n; j++) x[j] = j * spacing;
  size_t p = 0;
  std::vector<std::vector<double>> coefs;
  while (p < g.size()) {
    int sym = sym_of(g[p]);
    if (p + 1 >= g.size()) throw InputError("truncated GAMESS section");
    int ng = to_i(g[p + 1]);
    if (ng <= 0 || p + 2 + 3 * (size_t)ng > g.size()) throw InputError("unexpected end of GAMESS section");
    std::fill(y.begin(), y.end(), 0.0);
    for (int i = 0; i < ng; i++) {
      double ex = to_d(g[p + 3 + 3 * i]);
      double cc = to_d(g[p + 4 + 3 * i]);
      double norm;
      if (ieq(ntype, "GAMESSNORM")) {
        double fac = std::sqrt(2.0 * ex / M_PI), feg = 4.0 * ex, feg2 = feg * feg;
        const double nl[5] = {std::sqrt(2.0 * feg * fac), std::sqrt(2.0 * feg2 * fac / 3.0),
                              std::sqrt(2.0 * feg * feg2 * fac / 15.0), std::sqrt(2.0 * feg2 * feg2 * fac / 105.0),
                              std::sqrt(2.0 * feg2 * feg2 * feg * fac / 945.0)};
        norm = nl[sym_l(sym)];
      } else if (ieq(ntype, "CRYSTAL")) {
        const double nl[5] = {1.0, 1.0 / std::sqrt(3.0), 1.0 / std::sqrt(5.0), 1.0 / std::sqrt(7.0), 1.0 / std::sqrt(9.0)};
        norm = nl[sym_l(sym)];
      } else if (ieq(ntype, "NONE")) {
        norm = 1.0;
      } else {
        throw InputError("NORMTYPE " + ntype + " not understood");
      }
      for (int j = 0; j < n; j++) y[j] += norm * cc * std::exp(-ex * x[j] * x[j]);
    }
    if (renorm) {
      int pw = sym_l(sym) + 1;
      double sum = 0;
      for (int j = 0; j < n; j++) sum += spacing * std::pow(x[j], 2 * pw) * y[j] * y[j];
      if (std::fabs(sum - 1) > 1e-5)
        for (int j = 0; j < n; j++) y[j] /= std::sqrt(sum);
    }
    if (reqcut > 0) {
      const double cutmax = reqcut - 1e-6, cutmin = cutmax - 1.2;
      for (int j = 0; j < n; j++) {
        if (x[j] > cutmin) {
          if (x[j] > cutmax) y[j] = 0;
          else {
            double zz = (x[j] - cutmin) / 1.2;
            y[j] *= (1 - zz * zz * zz * (6 * zz * zz - 15 * zz + 10));
          }
        }
      }
    }
    double yp1 = (y[1] - y[0]) / spacing, ypn = (y[n - 1] - y[n - 2]) / spacing;
    std::vector<double> c(4 * (size_t)n);
    spline_fit(x, y, yp1, ypn, c.data());
    coefs.push_back(std::move(c));
    B.syms.push_back(sym);
    p += 2 + 3 * ng;
  }
  double thr0 = x[n - 1];
  double thr = 0;
  for (auto& c : coefs) {
    B.cuts.push_back(spline_cutoff(c.data(), n, spacing, thr0));
    thr = std::max(thr, B.cuts.back());
  }
  B.threshold = thr;
  for (auto& c : coefs) {
    if (thr0 < thr) {  // pad with zeros out to the common threshold
      int extra = int((thr - thr0) / spacing) + 1;
      c.resize(c.size() + 4 * (size_t)extra, 0.0);
    }
    B.spline_ids.push_back((int)tables.size());
    tables.push_back(std::move(c));
  }
  S.nspline = (int)tables.size();
  for (int s : B.syms) B.nfunc += sym_nfunc(s);
  return B;
}

// ORB file: "mo basis center label" records until COEFFICIENTS, then the
// coefficient list; each (mo, center, basis) entry points at a label.
// Complex coefficients (CORBITALS) are written "(re,im)" (or a plain real);
// moc_im receives their imaginary parts when given.
static void read_orb(const std::string& path, int nmo, const std::vector<int>& nfunc_center,
                     std::vector<double>& moc /* [nbasis][nmo] */, std::vector<double>* moc_im = nullptr) {
  std::ifstream in(path);
  if (!in) throw InputError("cannot open ORBFILE " + path);
  int ncent = (int)nfunc_center.size();
  int maxb = 0;
  for (int v : nfunc_center) maxb = std::max(maxb, v);
  std::vector<long> cm((size_t)nmo * ncent * maxb, -1);
  std::string t;
  long maxlabel = 0;
  while (true) {
    if (!(in >> t)) throw InputError("ORBFILE " + path + ": no COEFFICIENTS");
    if (t == "COEFFICIENTS") break;
    int mo = to_i(t) - 1;
    std::string sb, sc, sl;
    in >> sb >> sc >> sl;
    int b = to_i(sb) - 1, c = to_i(sc) - 1;
    long l = to_i(sl) - 1;
    if (mo < nmo) {
      if (b < 0 || b >= maxb || c < 0 || c >= ncent) throw InputError("ORBFILE entry out of range");
      cm[((size_t)mo * ncent + c) * maxb + b] = l;
    }
    maxlabel = std::max(maxlabel, l + 1);
  }
  std::vector<double> coef(maxlabel), coef_im(maxlabel, 0.0);
  for (long i = 0; i < maxlabel; i++) {
    if (!(in >> t)) throw InputError("ORBFILE " + path + ": too few coefficients");
    if (!t.empty() && t[0] == '(') {
      if (!moc_im) throw InputError("ORBFILE " + path + ": complex coefficient in real ORBITALS");
      // "(re,im)" or "(re)"; a space may follow the comma
      while (t.back() != ')') {
        std::string more;
        if (!(in >> more)) throw InputError("ORBFILE " + path + ": unterminated complex coefficient");
        t += more;
      }
      const size_t comma = t.find(',');
      coef[i] = to_d(t.substr(1, (comma == std::string::npos ? t.size() - 1 : comma) - 1));
      if (comma != std::string::npos) coef_im[i] = to_d(t.substr(comma + 1, t.size() - comma - 2));
    } else {
      coef[i] = to_d(t);
    }
  }
  int nbasis = 0;
  for (int v : nfunc_center) nbasis += v;
  moc.assign((size_t)nbasis * nmo, 0.0);
  if (moc_im) moc_im->assign((size_t)nbasis * nmo, 0.0);
  int row = 0;
  for (int c = 0; c < ncent; c++)
    for (int f = 0; f < nfunc_center[c]; f++, row++)
      for (int mo = 0; mo < nmo; mo++) {
        long l = cm[((size_t)mo * ncent + c) * maxb + f];
        moc[(size_t)row * nmo + mo] = l >= 0 ? coef[l] : 0.0;
        if (moc_im) (*moc_im)[(size_t)row * nmo + mo] = l >= 0 ? coef_im[l] : 0.0;
      }
}

static std::vector<Radial> read_radial(const std::vector<std::string>& w) {
  if (w.size() < 2) throw InputError("empty Jastrow basis section");
  std::vector<Radial> out;
  if (ieq(w[1], "CUTOFF_CUSP")) {
    Radial r;
    r.kind = RAD_CUTOFF_CUSP;
    r.a = value_d(w, "CUSP", 0, true);
    r.b = value_d(w, "GAMMA", 0, true);
    r.rcut = value_d(w, "CUTOFF", 0, true);
    if (r.rcut < 0) throw InputError("CUTOFF_CUSP cutoff must be positive");
    out.push_back(r);
  } else if (ieq(w[1], "POLYPADE")) {
    double rcut = value_d(w, "RCUT", 0, true);
    double b0 = value_d(w, "BETA0", 0, true);
    int nf = (int)value_d(w, "NFUNC", 0, true);
    double b1 = std::log(b0 + 1.00001);
    for (int i = 0; i < nf; i++) {
      Radial r;
      r.kind = RAD_POLYPADE;
      r.rcut = rcut;
      r.a = i == 0 ? b0 : std::exp(b1 + 1.6 * i) - 1;
      r.b = 0;
      out.push_back(r);
    }
  } else if (ieq(w[1], "PADE")) {
    // Pade_function (basis_function/Pade_function.cpp:21-45, 128-184):
    // (a_i r / (1 + a_i r))^2 with a_i = ALPHA0 / 2^i, no cutoff
    const double a0 = value_d(w, "ALPHA0", 0, true);
    const int nf = (int)value_d(w, "NFUNC", 0, true);
    for (int i = 0; i < nf; i++) {
      Radial r;
      r.kind = RAD_PADE;
      r.rcut = 1e99;
      r.a = a0 / std::pow(2.0, i);
      r.b = 0;
      out.push_back(r);
    }
  } else {
    throw InputError("Jastrow basis type " + w[1] + " not supported (CUTOFF_CUSP, POLYPADE, PADE)");
  }
  return out;
}

static void gesqua(int& aip, std::vector<double>& q, std::vector<double>& wq) {
  if (aip < 4) throw InputError("AIP must be at least 4");
  q.clear(); wq.clear();
  if (aip < 6) {
    aip = 4;
    double s = 1.0 / std::sqrt(3.0);
    double p[4][3] = {{s, s, s}, {s, -s, -s}, {-s, s, -s}, {-s, -s, s}};
    for (auto& r : p) { q.insert(q.end(), r, r + 3); wq.push_back(0.25); }
  } else if (aip < 12) {
    aip = 6;
    double p[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    for (auto& r : p) { q.insert(q.end(), r, r + 3); wq.push_back(1.0 / 6.0); }
  } else if (aip < 18) {
    // icosahedron vertices: the poles and two staggered rings of five
    aip = 12;
    q.assign(36, 0.0);
    q[2] = 1.0; q[5] = -1.0;
    const double fi0 = M_PI / 5.0, c = 1.0 / std::sqrt(5.0), s = 2.0 / std::sqrt(5.0);
    for (int i = 0; i < 5; i++) {
      double rk2 = 2 * i;
      q[3 * (i + 2) + 0] = s * std::cos(rk2 * fi0);
      q[3 * (i + 2) + 1] = s * std::sin(rk2 * fi0);
      q[3 * (i + 2) + 2] = c;
      q[3 * (i + 7) + 0] = s * std::cos((rk2 + 1) * fi0);
      q[3 * (i + 7) + 1] = s * std::sin((rk2 + 1) * fi0);
      q[3 * (i + 7) + 2] = -c;
    }
    wq.assign(12, 1.0 / 12.0);
  } else if (aip < 32) {
    // 18: the octahedron's 6 vertices (weight 1/30) and 12 edge midpoints
    // (1/15); 26: those (40/840, 32/840) plus the cube's 8 vertices (27/840)
    // (Abramowitz & Stegun 25.4.62-63; gesqua.cpp:121-273 point order)
    aip = aip < 26 ? 18 : 26;
    const double pa[6][3] = {{1, 0, 0}, {-1, 0, 0}, {0, 1, 0}, {0, -1, 0}, {0, 0, 1}, {0, 0, -1}};
    for (auto& r : pa) q.insert(q.end(), r, r + 3);
    const double h = 1.0 / std::sqrt(2.0);
    const int pair[3][2] = {{0, 1}, {0, 2}, {2, 1}};  // (x,y), (x,z), (z,y): first axis varies fastest
    for (auto& ax : pair)
      for (int sb = 0; sb < 2; sb++)
        for (int sa = 0; sa < 2; sa++) {
          double r[3] = {0, 0, 0};
          r[ax[0]] = sa ? -h : h;
          r[ax[1]] = sb ? -h : h;
          q.insert(q.end(), r, r + 3);
        }
    if (aip == 26) {
      const double b = 1.0 / std::sqrt(3.0);
      for (int sx = 0; sx < 2; sx++)
        for (int sz = 0; sz < 2; sz++)
          for (int sy = 0; sy < 2; sy++) {
            const double r[3] = {sx ? -b : b, sy ? -b : b, sz ? -b : b};
            q.insert(q.end(), r, r + 3);
          }
      for (int i = 0; i < 26; i++) wq.push_back(i < 6 ? 40.0 / 840.0 : i < 18 ? 32.0 / 840.0 : 27.0 / 840.0);
    } else {
      for (int i = 0; i < 18; i++) wq.push_back(i < 6 ? 1.0 / 30.0 : 1.0 / 15.0);
    }
  } else if (aip == 32) {
    // the icosahedron's 12 vertices (weight 5/168) and the dodecahedron's 20
    // (27/840), as polar angles around z (gesqua.cpp:274-320 point order)
    q.assign(96, 0.0);
    q[2] = 1.0; q[5] = -1.0;
    const double t5 = std::sqrt(15.0 + 6.0 * std::sqrt(5.0));
    const double th1 = std::acos((2.0 + std::sqrt(5.0)) / t5), th2 = std::acos(1.0 / t5);
    auto put = [&](int idx, double th, double ph) {
      q[3 * idx] = std::sin(th) * std::cos(ph);
      q[3 * idx + 1] = std::sin(th) * std::sin(ph);
      q[3 * idx + 2] = std::cos(th);
    };
    for (int i = 0; i < 5; i++) {
      const double ev = 2 * i * M_PI / 5, od = (2 * i + 1) * M_PI / 5;
      put(i + 2, std::atan(2.0), ev);
      put(i + 7, M_PI - std::atan(2.0), od);
      put(i + 12, th1, od);
      put(i + 17, th2, od);
      put(i + 22, M_PI - th1, ev);
      put(i + 27, M_PI - th2, ev);
    }
    for (int i = 0; i < 32; i++) wq.push_back(i < 12 ? 5.0 / 168.0 : 27.0 / 840.0);
  } else {
    throw InputError("Bad number of AIP's: " + std::to_string(aip) + " (4, 6, 12, 18, 26 or 32)");
  }
}

static double pp_radial(const PPAtom& P, int spin, int l, double r) {
  const std::vector<int>& tf = spin == 0 ? P.term_first : P.term_first_dn;
  double v = 0;
  for (int t = tf[l]; t < tf[l + 1]; t++) {
    double ex = std::min(P.term_a[t] * r * r, 60.0);
    v += P.term_c[t] * std::pow(r, P.term_n[t]) * std::exp(-ex);
  }
  return v;
}

// ---------------------------------------------------------------------------
// periodic cell: Periodic_system::read (system/Periodic_system.cpp:106-413),
// enforcePbc (:521-570), find_centers (system/Pbc_enforcer.cpp:205-420),
// constEwald / ewaldIon (Periodic_system.cpp:620-749)

static void cross3(const double* a, const double* b, double* c) {
  c[0] = a[1] * b[2] - a[2] * b[1];
  c[1] = a[2] * b[0] - a[0] * b[2];
  c[2] = a[0] * b[1] - a[1] * b[0];
}
static double dot3(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }

static double erfc_poly(double x) {
  const double p = .3275911, a = .254829592, b = -.284496736, c = 1.421413741, d = -1.453152027, e = 1.061405429;
  double y = 1. / (1. + p * x);
  return y * (a + y * (b + y * (c + y * (d + y * e)))) * std::exp(-x * x);
}

static void wrap_host(const HostSystem& S, double* p) {
  for (int i = 0; i < 3; i++) {
    for (int it = 0; it < 1000; it++) {
      double too_short = 0, too_far = 0;
      for (int j = 0; j < 3; j++) {
        too_short += S.normvec[3 * i + j] * (p[j] - S.origin[j]);
        too_far += S.normvec[3 * i + j] * (p[j] - S.corners[3 * i + j]);
      }
      if (too_short < -1e-12) for (int j = 0; j < 3; j++) p[j] += S.lat[3 * i + j];
      else if (too_far > 1e-12) for (int j = 0; j < 3; j++) p[j] -= S.lat[3 * i + j];
      else break;
    }
  }
}

static void setup_cell(HostSystem& S, const std::vector<std::string>& sysw) {
  auto lv = get_section(sysw, "LATTICEVEC");
  if (lv.size() != 9) throw InputError("LATTICEVEC must have exactly 9 values");
  for (int i = 0; i < 9; i++) S.lat[i] = to_d(lv[i]);
  size_t pos = 0;
  std::vector<std::string> og;
  if (find_section(sysw, "ORIGIN", pos, og)) {
    if (og.size() < 3) throw InputError("ORIGIN section must have at least 3 elements");
    for (int i = 0; i < 3; i++) S.origin[i] = to_d(og[i]);
  }
  pos = 0;
  std::vector<std::string> kp;
  if (find_section(sysw, "KPOINT", pos, kp)) {
    if (kp.size() != 3) throw InputError("KPOINT must have 3 elements");
    for (int d = 0; d < 3; d++) S.kpt[d] = to_d(kp[d]);
  }
  const double divider = value_d(sysw, "CUTOFF_DIVIDER", 2.000001);
  const int gmax = (int)value_d(sysw, "EWALD_GMAX", 200);
  const double* a0 = S.lat;
  const double* a1 = S.lat + 3;
  const double* a2 = S.lat + 6;
  double cr[9];
  cross3(a1, a2, cr);
  cross3(a2, a0, cr + 3);
  cross3(a0, a1, cr + 6);
  double det = std::fabs(dot3(a0, cr));
  S.volume = det;
  double recip[9];
  for (int i = 0; i < 9; i++) recip[i] = cr[i] / det;
  for (int i = 0; i < 3; i++) {
    double d = dot3(cr + 3 * i, S.lat + 3 * i);
    for (int j = 0; j < 3; j++) S.normvec[3 * i + j] = d < 0 ? -cr[3 * i + j] : cr[3 * i + j];
    for (int j = 0; j < 3; j++) S.corners[3 * i + j] = S.origin[j] + S.lat[3 * i + j];
  }
  S.smallest_height = 1e99;
  for (int i = 0; i < 3; i++) {
    double h = std::fabs(dot3(cr + 3 * i, S.lat + 3 * i)) / std::sqrt(dot3(cr + 3 * i, cr + 3 * i));
    S.smallest_height = std::min(S.smallest_height, h);
  }
  S.alpha = 5.0 / S.smallest_height;
  for (int aa = -1; aa <= 1; aa++)
    for (int bb = -1; bb <= 1; bb++)
      for (int cc = -1; cc <= 1; cc++)
        for (int d = 0; d < 3; d++) S.lattice_basis.push_back(aa * a0[d] + bb * a1[d] + cc * a2[d]);
  // image centers within the cell enlarged by cutoff = min height / divider
  double hgt[3];
  {
    double c12[3], c02[3], c01[3];
    cross3(a1, a2, c12); cross3(a0, a2, c02); cross3(a0, a1, c01);
    hgt[0] = std::fabs(dot3(a0, c12)) / std::sqrt(dot3(c12, c12));
    hgt[1] = std::fabs(dot3(a1, c02)) / std::sqrt(dot3(c02, c02));
    hgt[2] = std::fabs(dot3(a2, c01)) / std::sqrt(dot3(c01, c01));
  }
  const double cutoff = std::min(std::min(hgt[0], hgt[1]), hgt[2]) / divider;
  double org[3] = {S.origin[0], S.origin[1], S.origin[2]}, piped[9];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      org[j] -= cutoff * S.lat[3 * i + j] / hgt[i];
      piped[3 * i + j] = S.lat[3 * i + j] * (1 + 2 * cutoff / hgt[i]);
    }
  double cm[3], diag[3];
  for (int i = 0; i < 3; i++) {
    cm[i] = S.origin[i];
    diag[i] = 0;
    for (int j = 0; j < 3; j++) { cm[i] += 0.5 * S.lat[3 * j + i]; diag[i] += S.lat[3 * j + i]; }
  }
  double radius = std::sqrt(dot3(diag, diag));
  for (int j = 0; j < 3; j++) {
    double d2[3];
    for (int i = 0; i < 3; i++) d2[i] = diag[i] - 2 * S.lat[3 * j + i];
    radius = std::max(radius, std::sqrt(dot3(d2, d2)));
  }
  radius = 0.5 * radius + cutoff;
  double pc[9];
  cross3(piped + 3, piped + 6, pc);
  cross3(piped + 6, piped, pc + 3);
  cross3(piped, piped + 3, pc + 6);
  for (int i = 0; i < 3; i++)
    if (dot3(pc + 3 * i, piped + 3 * i) < 0)
      for (int j = 0; j < 3; j++) pc[3 * i + j] = -pc[3 * i + j];
  std::vector<std::vector<double>> img(S.natoms);
  std::vector<std::vector<int>> shift(S.natoms);
  const int ns = 4;
  for (int ii = -ns; ii <= ns; ii++)
    for (int jj = -ns; jj <= ns; jj++)
      for (int kk = -ns; kk <= ns; kk++)
        for (int at = 0; at < S.natoms; at++) {
          double p[3];
          for (int i = 0; i < 3; i++) p[i] = S.atom_pos[3 * at + i] + a0[i] * ii + a1[i] * jj + a2[i] * kk;
          bool inside = true;
          for (int i = 0; i < 3 && inside; i++) {
            double sh = 0, fa = 0;
            for (int j = 0; j < 3; j++) {
              sh += pc[3 * i + j] * (p[j] - org[j]);
              fa += pc[3 * i + j] * (p[j] - (org[j] + piped[3 * i + j]));
            }
            if (sh < 0 || fa > 0) inside = false;
          }
          double dc[3] = {p[0] - cm[0], p[1] - cm[1], p[2] - cm[2]};
          if (inside && std::sqrt(dot3(dc, dc)) < radius) {
            img[at].insert(img[at].end(), p, p + 3);
            shift[at].insert(shift[at].end(), {ii, jj, kk});
          }
        }
  for (int at = 0; at < S.natoms; at++) {
    S.image_first.push_back((int)S.image_pos.size() / 3);
    S.image_count.push_back((int)img[at].size() / 3);
    S.image_pos.insert(S.image_pos.end(), img[at].begin(), img[at].end());
    S.image_shift.insert(S.image_shift.end(), shift[at].begin(), shift[at].end());
  }
  // the image centers come from the positions as given; the ions themselves
  // are then put inside the cell (same order as the reference's read)
  for (int a = 0; a < S.natoms; a++) wrap_host(S, &S.atom_pos[3 * a]);
  // G vectors: half space, weight 4 pi exp(-G^2/4 alpha^2)/(V G^2) > 1e-10
  for (int ig = 0; ig <= gmax; ig++)
    for (int jg = (ig == 0 ? 0 : -gmax); jg <= gmax; jg++)
      for (int kg = ((ig == 0 && jg == 0) ? 0 : -gmax); kg <= gmax; kg++) {
        double g[3];
        for (int i = 0; i < 3; i++) g[i] = 2 * M_PI * (ig * recip[i] + jg * recip[3 + i] + kg * recip[6 + i]);
        double g2 = dot3(g, g);
        if (g2 > 1e-8) {
          double w = 4.0 * M_PI * std::exp(-g2 / (4 * S.alpha * S.alpha)) / (S.volume * g2);
          if (w > 1e-10) { S.gvec.insert(S.gvec.end(), g, g + 3); S.gweight.push_back(w); }
        }
      }
  const int ng = (int)S.gweight.size();
  // constant terms
  const int N = S.nelec, na = S.natoms;
  double ionion = 0, ionelec = 0, q2 = 0;
  for (int i = 0; i < na; i++) {
    ionelec += S.atom_charge[i] * (-N);
    q2 += S.atom_charge[i] * S.atom_charge[i];
    for (int j = i + 1; j < na; j++) ionion += S.atom_charge[i] * S.atom_charge[j];
  }
  const double sq = -.5 * (2 * S.alpha / std::sqrt(M_PI) + M_PI / (S.volume * S.alpha * S.alpha));
  const double ij = -M_PI / (S.volume * S.alpha * S.alpha);
  const double self_ii = ionion * ij + q2 * sq;
  const double self_ei = ionelec * ij;
  const double self_ee = .5 * double(N) * (N - 1) * ij + N * sq;
  double real = 0;
  for (int i = 0; i < na; i++)
    for (int j = 0; j < i; j++)
      for (int kk = -2; kk <= 2; kk++)
        for (int jj = -2; jj <= 2; jj++)
          for (int ii = -2; ii <= 2; ii++) {
            double r2[3];
            for (int d = 0; d < 3; d++)
              r2[d] = S.atom_pos[3 * i + d] - S.atom_pos[3 * j + d] + kk * a0[d] + jj * a1[d] + ii * a2[d];
            double r = std::sqrt(dot3(r2, r2));
            real += S.atom_charge[i] * S.atom_charge[j] * erfc_poly(S.alpha * r) / r;
          }
  S.ion_sin.assign(ng, 0.0);
  S.ion_cos.assign(ng, 0.0);
  double eion = 0;
  for (int g = 0; g < ng; g++) {
    for (int a = 0; a < na; a++) {
      double dp = dot3(&S.atom_pos[3 * a], &S.gvec[3 * g]);
      S.ion_sin[g] += S.atom_charge[a] * std::sin(dp);
      S.ion_cos[g] += S.atom_charge[a] * std::cos(dp);
    }
    eion += S.gweight[g] * (S.ion_sin[g] * S.ion_sin[g] + S.ion_cos[g] * S.ion_cos[g]) / 2;
  }
  S.ewald_const = 2 * eion + real + self_ii + self_ee + self_ei;
}

HostSystem build_system(const std::string& deck_path) {
  HostSystem S;
  S.deck_path = deck_path;
  auto words = tokenize_file(deck_path);
  std::string base = dirname_of(deck_path);

  // ---- SYSTEM
  auto sysw = get_section(words, "SYSTEM");
  if (sysw.empty() || !(ieq(sysw[0], "MOLECULE") || ieq(sysw[0], "MOLECULAR") || ieq(sysw[0], "PERIODIC")))
    throw InputError("SYSTEM must be MOLECULE or PERIODIC");
  S.periodic = ieq(sysw[0], "PERIODIC");
  auto ns = get_section(sysw, "NSPIN");
  if (ns.size() != 2) throw InputError("NSPIN needs two numbers");
  S.nup = to_i(ns[0]);
  S.ndn = to_i(ns[1]);
  S.nelec = S.nup + S.ndn;
  for (auto& a : all_sections(sysw, "ATOM")) {
    if (a.size() < 2) throw InputError("bad ATOM section");
    S.labels.push_back(a[0]);
    S.atom_charge.push_back(to_d(a[1]));
    size_t k = 0;
    while (k < a.size() && !ieq(a[k], "COOR")) k++;
    if (k + 3 >= a.size()) throw InputError("ATOM needs COOR x y z");
    for (int d = 0; d < 3; d++) S.atom_pos.push_back(to_d(a[k + 1 + d]));
  }
  S.natoms = (int)S.labels.size();
  if (S.natoms == 0) throw InputError("no ATOM in SYSTEM");
  if (S.nelec <= 0 || S.nup < 0 || S.ndn < 0) throw InputError("bad NSPIN");
  if (S.periodic) {
    setup_cell(S, sysw);
  } else {
    for (int i = 0; i < S.natoms; i++)
      for (int j = 0; j < i; j++) {
        double d2 = 0;
        for (int d = 0; d < 3; d++) {
          double t = S.atom_pos[3 * i + d] - S.atom_pos[3 * j + d];
          d2 += t * t;
        }
        S.ion_ion += S.atom_charge[i] * S.atom_charge[j] / std::sqrt(d2);
      }
    S.image_pos = S.atom_pos;
    S.image_shift.assign((size_t)3 * S.natoms, 0);
    for (int a = 0; a < S.natoms; a++) { S.image_first.push_back(a); S.image_count.push_back(1); }
  }

  // ---- TRIALFUNC
  auto tf = get_section(words, "TRIALFUNC");
  std::vector<std::string> wf1, wf2;
  if (!tf.empty() && ieq(tf[0], "SLATER")) {
    wf1 = tf;  // a Slater wave function alone (Slat_wf_data, Wavefunction_data.cpp:32-59): U = 0
  } else {
    if (tf.empty() || !ieq(tf[0], "SLATER-JASTROW")) throw InputError("TRIALFUNC must be SLATER-JASTROW or SLATER");
    wf1 = get_section(tf, "WF1");
    wf2 = get_section(tf, "WF2");
    if (wf1.empty() || !ieq(wf1[0], "SLATER")) throw InputError("WF1 must be SLATER");
    if (wf2.empty() || !ieq(wf2[0], "JASTROW2")) throw InputError("WF2 must be JASTROW2");
  }

  // Slater: one or more determinants (DETWT weights, STATES per determinant)
  auto detwt = get_section(wf1, "DETWT");
  if (detwt.empty()) throw InputError("Need DETWT in SLATER section");
  if (detwt.size() > 64) throw InputError("more than 64 determinants: beyond this engine build");
  if (has_section(wf1, "CSF")) throw InputError("CSF expansions are not supported");
  // CORBITALS: complex orbitals (Slat_wf_data.cpp:130-147)
  S.complex_orbitals = has_section(wf1, "CORBITALS");
  if (S.complex_orbitals && has_section(wf1, "ORBITALS")) throw InputError("both ORBITALS and CORBITALS given");
  auto orbw = get_section(wf1, S.complex_orbitals ? "CORBITALS" : "ORBITALS");
  if (orbw.empty()) throw InputError("Need ORBITALS or CORBITALS section in SLATER wave function");
  if (!orbw.empty() && (ieq(orbw[0], "EINSPLINE_MO") || ieq(orbw[0], "BASFUNC_MO")))
    throw InputError("ORBITALS type " + orbw[0] + " not supported (BLAS_MO and CUTOFF_MO are)");
  // CUTOFF_MO (MO_matrix_cutoff, MO_matrix.cpp:33-49): per-function spline
  // cutoffs, no |value| <= 1e-8 skip of basis values, coefficients with
  // |c| <= 1e-12 dropped and MAGNIFY applied (MO_matrix_cutoff.h:141-247, 413-569)
  S.cutoff_mo = !orbw.empty() && ieq(orbw[0], "CUTOFF_MO");
  std::string tmp;
  if (!find_value(orbw, "NMO", tmp)) throw InputError("Need NMO in molecular orbital section");
  int nmo = to_i(tmp);
  std::vector<std::vector<double>> tables;
  std::vector<BasisObj> bases;
  for (auto& b : all_sections(orbw, "BASIS")) bases.push_back(read_aospline(b, S, tables));
  if (bases.empty()) throw InputError("Didn't find a BASIS section");
  {
    // A label may have several BASIS sections: the reference appends every
    // one to the label's centers (Center_set::assignBasis, Center_set.cpp:
    // 140-165).  They become one object (one spline row per interval) with the
    // splines in section order; the sections must share one cutoff.
    std::vector<BasisObj> merged;
    std::vector<std::vector<int>> ids;
    for (auto& B : bases) {
      size_t m = 0;
      while (m < merged.size() && merged[m].label != B.label) m++;
      if (m == merged.size()) {
        merged.push_back(B);
        ids.push_back(B.spline_ids);
        continue;
      }
      if (merged[m].threshold != B.threshold)
        throw InputError("several BASIS sections for " + B.label + " with different cutoffs are not supported");
      merged[m].syms.insert(merged[m].syms.end(), B.syms.begin(), B.syms.end());
      merged[m].cuts.insert(merged[m].cuts.end(), B.cuts.begin(), B.cuts.end());
      merged[m].nfunc += B.nfunc;
      ids[m].insert(ids[m].end(), B.spline_ids.begin(), B.spline_ids.end());
    }
    std::vector<std::vector<double>> reordered;
    for (size_t m = 0; m < merged.size(); m++) {
      merged[m].spline_ids.clear();
      for (int id : ids[m]) {
        merged[m].spline_ids.push_back((int)reordered.size());
        reordered.push_back(std::move(tables[id]));
      }
    }
    tables = std::move(reordered);
    bases = std::move(merged);
  }
  size_t cpos = 0;
  std::vector<std::string> cent;
  if (find_section(orbw, "CENTERS", cpos, cent) && !has_keyword(cent, "USEATOMS") && !has_keyword(cent, "USEGLOBAL"))
    throw InputError("CENTERS must be USEATOMS or USEGLOBAL");
  std::vector<int> nfunc_center(S.natoms, 0);
  int first = 0;
  for (auto& B : bases) {
    S.obj_first.push_back(B.spline_ids.empty() ? 0 : B.spline_ids[0]);
    S.obj_count.push_back((int)B.spline_ids.size());
  }
  for (int c = 0; c < S.natoms; c++) {
    for (size_t bi = 0; bi < bases.size(); bi++) {
      auto& B = bases[bi];
      if (B.label != S.labels[c]) continue;
      for (size_t k = 0; k < B.syms.size(); k++) {
        Shell sh;
        sh.center = c;
        sh.spline = B.spline_ids[k];
        sh.sym = B.syms[k];
        sh.first = first;
        sh.nfunc = sym_nfunc(B.syms[k]);
        sh.cutoff = B.threshold;
        sh.fcut = B.cuts[k];
        sh.obj = (int)bi;
        sh.k = (int)k;
        first += sh.nfunc;
        S.shells.push_back(sh);
      }
      nfunc_center[c] += B.nfunc;
    }
  }
  S.nbasis = first;
  // flatten spline tables (all share npts after padding to the longest)
  size_t maxlen = 0;
  for (auto& t : tables) maxlen = std::max(maxlen, t.size());
  S.spline_npts = (int)(maxlen / 4);
  S.spline_coef.assign(tables.size() * maxlen, 0.0);
  for (size_t i = 0; i < tables.size(); i++) std::copy(tables[i].begin(), tables[i].end(), S.spline_coef.begin() + i * maxlen);

  std::string orbfile;
  if (!find_value(orbw, "ORBFILE", orbfile)) throw InputError("Must specify ORBFILE for MO matrix");
  if (orbfile[0] != '/' && !file_exists(orbfile)) orbfile = base + "/" + orbfile;
  std::vector<double> moc_all, moc_all_im;
  read_orb(orbfile, nmo, nfunc_center, moc_all, S.complex_orbitals ? &moc_all_im : nullptr);
  if (S.cutoff_mo) {
    const double mag = value_d(orbw, "MAGNIFY", 1.0);
    for (size_t i = 0; i < moc_all.size(); i++) {
      const double im = moc_all_im.empty() ? 0.0 : moc_all_im[i];
      if (!(std::sqrt(moc_all[i] * moc_all[i] + im * im) > 1e-12)) {
        moc_all[i] = 0.0;
        if (!moc_all_im.empty()) moc_all_im[i] = 0.0;
      } else {
        moc_all[i] *= mag;
        if (!moc_all_im.empty()) moc_all_im[i] *= mag;
      }
    }
  }
  const bool kpt_nonzero = S.kpt[0] != 0.0 || S.kpt[1] != 0.0 || S.kpt[2] != 0.0;
  if ((S.complex_orbitals || kpt_nonzero) && detwt.size() > 1)
    throw InputError("determinant expansions need real orbitals at the Gamma point");
  auto states = get_section(wf1, "STATES");
  const int ndet = (int)detwt.size();
  if ((int)states.size() != ndet * S.nelec)
    throw InputError("STATES must list nup+ndown orbitals for every determinant");
  S.nel_s[0] = S.nup; S.nel_s[1] = S.ndn;
  S.detwt.resize(ndet);
  S.det_ud.assign((size_t)ndet * 2, 0);
  for (int s = 0; s < 2; s++) {
    const int ne = S.nel_s[s];
    std::vector<int> uni;                     // union of this spin's orbitals, first-use order
    std::vector<std::vector<int>> uorbs;      // distinct spin-determinants (MO lists)
    for (int k = 0; k < ndet; k++) {
      std::vector<int> orbs(ne);
      for (int i = 0; i < ne; i++) {
        int mo = to_i(states[(size_t)k * S.nelec + (s == 0 ? 0 : S.nup) + i]) - 1;
        if (mo < 0 || mo >= nmo) throw InputError("STATES entry beyond NMO");
        orbs[i] = mo;
        if (std::find(uni.begin(), uni.end(), mo) == uni.end()) uni.push_back(mo);
      }
      int u = (int)(std::find(uorbs.begin(), uorbs.end(), orbs) - uorbs.begin());
      if (u == (int)uorbs.size()) uorbs.push_back(orbs);
      S.det_ud[2 * k + s] = u;
    }
    if (uorbs.size() > 16) throw InputError("more than 16 distinct determinants of one spin: beyond this engine build");
    S.nmo[s] = (int)uni.size();
    S.moc[s].assign((size_t)S.nbasis * std::max(S.nmo[s], 1), 0.0);
    for (int j = 0; j < S.nmo[s]; j++)
      for (int f = 0; f < S.nbasis; f++) S.moc[s][(size_t)f * S.nmo[s] + j] = moc_all[(size_t)f * nmo + uni[j]];
    S.moc_im[s].assign(S.moc[s].size(), 0.0);
    if (S.complex_orbitals)
      for (int j = 0; j < S.nmo[s]; j++)
        for (int f = 0; f < S.nbasis; f++)
          S.moc_im[s][(size_t)f * S.nmo[s] + j] = moc_all_im[(size_t)f * nmo + uni[j]];
    S.udet_cols[s].clear();
    for (auto& o : uorbs) {
      std::vector<int> cols(ne);
      for (int i = 0; i < ne; i++) cols[i] = (int)(std::find(uni.begin(), uni.end(), o[i]) - uni.begin());
      S.udet_cols[s].push_back(cols);
    }
  }
  for (int k = 0; k < ndet; k++) S.detwt[k] = to_d(detwt[k]);
  {
    // Shells none of whose functions carries an orbital coefficient (e.g. a
    // BASIS section given twice with an ORB file for one copy) add exactly
    // zero to every orbital: they are left out of the evaluation.
    std::vector<Shell> kept;
    std::vector<int> rows;  // old basis row of every kept function
    for (const Shell& sh : S.shells) {
      bool used = false;
      for (int f = sh.first; f < sh.first + sh.nfunc && !used; f++)
        for (int s = 0; s < 2 && !used; s++)
          for (int j = 0; j < S.nmo[s] && !used; j++)
            used = S.moc[s][(size_t)f * S.nmo[s] + j] != 0.0 || S.moc_im[s][(size_t)f * S.nmo[s] + j] != 0.0;
      if (!used) continue;
      Shell k = sh;
      k.first = (int)rows.size();
      for (int f = sh.first; f < sh.first + sh.nfunc; f++) rows.push_back(f);
      kept.push_back(k);
    }
    if (kept.size() < S.shells.size() && !kept.empty()) {
      for (int s = 0; s < 2; s++) {
        const int nm = S.nmo[s];
        std::vector<double> re(rows.size() * std::max(nm, 1), 0.0), im(re.size(), 0.0);
        for (size_t r = 0; r < rows.size(); r++)
          for (int j = 0; j < nm; j++) {
            re[r * nm + j] = S.moc[s][(size_t)rows[r] * nm + j];
            im[r * nm + j] = S.moc_im[s][(size_t)rows[r] * nm + j];
          }
        S.moc[s] = std::move(re);
        S.moc_im[s] = std::move(im);
      }
      S.shells = std::move(kept);
      S.nbasis = (int)rows.size();
    }
  }

  // ---- Jastrow groups
  S.ei_first.assign(S.natoms, 0);
  S.ei_count.assign(S.natoms, 0);
  std::vector<std::vector<Radial>> ei_at(S.natoms);
  std::vector<std::vector<double>> ob_at(S.natoms);
  std::vector<std::vector<ThreeBodyTerm>> tb_at(S.natoms);
  static const int klm_default[12][3] = {{1, 1, 0}, {1, 0, 1}, {1, 1, 1}, {2, 2, 0}, {2, 0, 1}, {2, 0, 2},
                                         {2, 2, 2}, {3, 3, 0}, {3, 0, 2}, {3, 3, 2}, {1, 2, 2}, {2, 3, 2}};
  bool any3 = false, any3s = false;
  for (auto& g : all_sections(wf2, "GROUP")) {
    int ee0 = (int)S.ee.size();
    for (auto& b : all_sections(g, "EEBASIS")) {
      auto r = read_radial(b);
      S.ee.insert(S.ee.end(), r.begin(), r.end());
    }
    int nee_g = (int)S.ee.size() - ee0;
    S.ee_like.resize(S.ee.size(), 0.0);
    S.ee_unlike.resize(S.ee.size(), 0.0);
    // e-n functions of this group, per atom, in EIBASIS order
    std::vector<int> ei0(S.natoms);
    for (int a = 0; a < S.natoms; a++) ei0[a] = (int)ei_at[a].size();
    for (auto& b : all_sections(g, "EIBASIS")) {
      auto r = read_radial(b);
      bool found = false;
      for (int a = 0; a < S.natoms; a++)
        if (S.labels[a] == b[0]) { ei_at[a].insert(ei_at[a].end(), r.begin(), r.end()); found = true; }
      if (!found) throw InputError("Couldn't find center for basis label " + b[0]);
    }
    for (int a = 0; a < S.natoms; a++) ob_at[a].resize(ei_at[a].size(), 0.0);
    size_t pos = 0;
    std::vector<std::string> sec;
    if (find_section(g, "ONEBODY", pos, sec)) {
      for (auto& c : all_sections(sec, "COEFFICIENTS")) {
        bool found = false;
        for (int a = 0; a < S.natoms; a++) {
          if (S.labels[a] != c[0]) continue;
          found = true;
          int np = (int)c.size() - 1;
          if (np > (int)ei_at[a].size() - ei0[a]) throw InputError("ONEBODY has more coefficients than EIBASIS functions");
          for (int i = 0; i < np; i++) ob_at[a][ei0[a] + i] += to_d(c[i + 1]);
        }
        if (!found) throw InputError("Couldn't find a matching center for " + c[0]);
      }
    }
    bool has2 = false;
    pos = 0;
    if (find_section(g, "TWOBODY_SPIN", pos, sec)) {
      auto like = get_section(sec, "LIKE_COEFFICIENTS");
      auto unlike = get_section(sec, "UNLIKE_COEFFICIENTS");
      if (like.size() != unlike.size()) throw InputError("TWOBODY_SPIN like/unlike sizes differ");
      if ((int)like.size() > nee_g) throw InputError("Not enough EE basis functions for TWOBODY_SPIN");
      for (size_t p = 0; p < like.size(); p++) {
        S.ee_like[ee0 + p] += to_d(like[p]);
        S.ee_unlike[ee0 + p] += to_d(unlike[p]);
      }
      has2 = true;
    }
    pos = 0;
    if (find_section(g, "TWOBODY", pos, sec)) {
      if (has2) throw InputError("Can only have one of TWOBODY_SPIN or TWOBODY");
      auto c = get_section(sec, "COEFFICIENTS");
      if ((int)c.size() > nee_g) throw InputError("Not enough EE basis functions for TWOBODY");
      for (size_t p = 0; p < c.size(); p++) {
        S.ee_like[ee0 + p] += to_d(c[p]);
        S.ee_unlike[ee0 + p] += to_d(c[p]);
      }
    }
    // e-e-n terms: THREEBODY (Jastrow2_three.cpp) or THREEBODY_SPIN
    // (Jastrow2_three_diffspin.cpp:130-186: LIKE_COEFFICIENTS for pairs of
    // equal spin, UNLIKE_COEFFICIENTS for opposite spins); SM_TERMS replaces
    // the default (k, l, m) list
    std::vector<std::string> tb_sec, tbs_sec;
    pos = 0;
    const bool has3 = find_section(g, "THREEBODY", pos, tb_sec);
    pos = 0;
    const bool has3s = find_section(g, "THREEBODY_SPIN", pos, tbs_sec);
    if (has3 && has3s) throw InputError("Can only have one of THREEBODY_SPIN or THREEBODY");
    any3 = any3 || has3;
    any3s = any3s || has3s;
    if (has3 || has3s) {
      const std::vector<std::string>& ts = has3 ? tb_sec : tbs_sec;
      std::vector<std::array<int, 3>> klm;
      if (has_section(ts, "SM_TERMS")) {
        auto w = get_section(ts, "SM_TERMS");
        if (w.size() % 3 != 0) throw InputError("SM_TERMS must contain a multiple of 3 elements");
        for (size_t q = 0; q < w.size(); q += 3)
          klm.push_back({std::stoi(w[q]), std::stoi(w[q + 1]), std::stoi(w[q + 2])});
      } else {
        for (auto& t : klm_default) klm.push_back({t[0], t[1], t[2]});
      }
      const double scale = value_d(ts, "SCALE", 1.0);
      auto like = all_sections(ts, has3 ? "COEFFICIENTS" : "LIKE_COEFFICIENTS");
      auto unlike = has3 ? like : all_sections(ts, "UNLIKE_COEFFICIENTS");
      if (like.size() != unlike.size())
        throw InputError("Need same amount of LIKE_COEFFICIENTS and UNLIKE_COEFFICIENTS sections in three body");
      for (size_t sidx = 0; sidx < like.size(); sidx++) {
        const auto& c = like[sidx];
        const auto& cu = unlike[sidx];
        const int np = (int)c.size() - 1;
        if (cu.size() != c.size() || cu[0] != c[0])
          throw InputError("three-body spin coefficients: like and unlike sections differ for " + c[0]);
        if (np > (int)klm.size()) throw InputError("too many three-body parameters on " + c[0]);
        bool found = false;
        for (int a = 0; a < S.natoms; a++) {
          if (S.labels[a] != c[0]) continue;
          found = true;
          for (int i = 0; i < np; i++) {
            ThreeBodyTerm t;
            t.k = ei0[a] + klm[i][0];
            t.l = ei0[a] + klm[i][1];
            t.m = ee0 + klm[i][2];
            t.c = to_d(c[i + 1]) * scale;
            t.cu = to_d(cu[i + 1]) * scale;
            if (klm[i][0] < 0 || klm[i][1] < 0 || klm[i][2] < 0 ||
                klm[i][0] >= (int)ei_at[a].size() - ei0[a] || klm[i][1] >= (int)ei_at[a].size() - ei0[a] ||
                klm[i][2] >= nee_g)
              throw InputError("Threebody needs more basis functions");
            tb_at[a].push_back(t);
          }
        }
        if (!found) throw InputError("Couldn't find a matching center for " + c[0]);
      }
    }
  }
  S.tb_stale_ei = any3s && !any3;
  for (int a = 0; a < S.natoms; a++) {
    S.ei_first[a] = (int)S.ei.size();
    S.ei_count[a] = (int)ei_at[a].size();
    // three-body indices were per atom slice: rebase to the global list
    for (auto& t : tb_at[a]) { t.k += S.ei_first[a]; t.l += S.ei_first[a]; }
    S.ei.insert(S.ei.end(), ei_at[a].begin(), ei_at[a].end());
    S.onebody.insert(S.onebody.end(), ob_at[a].begin(), ob_at[a].end());
  }
  S.tb_first.assign(S.natoms, 0);
  S.tb_count.assign(S.natoms, 0);
  for (int a = 0; a < S.natoms; a++) {
    S.tb_first[a] = (int)S.tb.size();
    S.tb_count[a] = (int)tb_at[a].size();
    S.tb.insert(S.tb.end(), tb_at[a].begin(), tb_at[a].end());
  }

  // ---- PSEUDO
  S.pp.assign(S.natoms, PPAtom());
  for (auto& t : all_sections(words, "PSEUDO")) {
    PPAtom P;
    P.aip = (int)value_d(t, "AIP", 6);
    // RGAUSSIAN OLDQMC channels appended to P's term list; returns the
    // per-channel term offsets (Rgaussian_function.cpp:24-107)
    auto read_rgaussian = [&](const std::vector<std::string>& bw) {
      if (bw.size() < 2 || !ieq(bw[1], "RGAUSSIAN")) throw InputError("PSEUDO BASIS must be RGAUSSIAN");
      auto oq = get_section(bw, "OLDQMC");
      if (oq.size() < 2) throw InputError("badly formed OLDQMC section");
      size_t it = 1;
      const int nchan = to_i(oq[it++]);
      std::vector<int> nper(nchan);
      for (int l = 0; l < nchan; l++) nper[l] = to_i(oq[it++]);
      std::vector<int> first{(int)P.term_n.size()};
      for (int l = 0; l < nchan; l++) {
        for (int j = 0; j < nper[l]; j++) {
          if (it + 2 >= oq.size()) throw InputError("truncated OLDQMC section");
          P.term_n.push_back(to_d(oq[it]) - 2.0);
          P.term_a.push_back(to_d(oq[it + 1]));
          P.term_c.push_back(to_d(oq[it + 2]));
          it += 3;
        }
        first.push_back((int)P.term_n.size());
      }
      return first;
    };
    // SPIN_DEP: separate radial bases for spin-up and spin-down electrons
    // (Pseudopotential.cpp:912-933); ADD_ZEFF adds Z_ion / r to the local
    // channel (:309-316, 937-939)
    if (has_keyword(t, "SPIN_DEP")) {
      P.term_first = read_rgaussian(get_section(t, "BASIS_UP"));
      P.term_first_dn = read_rgaussian(get_section(t, "BASIS_DN"));
      if (P.term_first.size() != P.term_first_dn.size())
        throw InputError("SPIN_DEP: BASIS_UP and BASIS_DN have different channel counts");
    } else {
      P.term_first = read_rgaussian(get_section(t, "BASIS"));
      P.term_first_dn = P.term_first;
    }
    P.nchan = (int)P.term_first.size() - 1;
    P.add_zeff = has_keyword(t, "ADD_ZEFF");
    gesqua(P.aip, P.quad, P.weight);
    // evaluation radius: scan from 20 bohr down in 0.05 steps for the first
    // |v_l| > 1e-5 of each nonlocal channel for either spin (a channel never
    // above it keeps 20)
    std::vector<double> cutL(std::max(P.nchan - 1, 0), 20.0);
    std::vector<int> found(cutL.size(), 0);
    for (double r = 20.0; r > 0; r -= 0.05)
      for (int l = 0; l + 1 < P.nchan; l++)
        if ((std::fabs(pp_radial(P, 0, l, r)) > 1e-5 || std::fabs(pp_radial(P, 1, l, r)) > 1e-5) && !found[l]) {
          cutL[l] = r - 0.05;
          found[l] = 1;
        }
    P.cutoff = 0;
    for (double c : cutL) P.cutoff = std::max(P.cutoff, c);
    bool any = false;
    for (int a = 0; a < S.natoms; a++)
      if (S.labels[a] == t[0]) {
        if (S.pp[a].nchan) throw InputError("There are two PSEUDO sections for " + t[0]);
        S.pp[a] = P;
        any = true;
      }
    (void)any;
    S.has_pp = true;
    S.max_aip = std::max(S.max_aip, P.aip);
  }
  return S;
}

}  // namespace qwg
