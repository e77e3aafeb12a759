// QWalk walker-configuration files (include/qwg.h: qwg_write_configs,
// qwg_count_configs, qwg_read_configs), host only.  The text layout is the
// one write_configurations / read_configurations use with Config_save_point
// and Dmc_point (program_utils/qmc_io.h:371-470, system/Sample_point.cpp:
// 120-148, method/Dmc_method.cpp:1228-1267), so files move between the
// reference and the engine in both directions.
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>

#include "../../include/qwg.h"

namespace {

bool ieq(const std::string& a, const char* b) {
  size_t n = a.size();
  for (size_t i = 0; i < n; i++) {
    if (!b[i]) return false;
    char x = a[i], y = b[i];
    if (x >= 'A' && x <= 'Z') x = char(x - 'A' + 'a');
    if (y >= 'A' && y <= 'Z') y = char(y - 'A' + 'a');
    if (x != y) return false;
  }
  return b[n] == 0;
}

// Parses every walker; calls f(nelec, positions, weight, sign) for each.
// Returns QWG_OK or QWG_ERR_INPUT on a malformed file.
template <class F>
int parse(const char* path, F&& f) {
  std::ifstream is(path);
  if (!is) return QWG_ERR_INPUT;
  std::string w;
  std::vector<double> pos;
  while (is >> w) {
    if (!ieq(w, "walker")) continue;
    if (!(is >> w) || w != "{") return QWG_ERR_INPUT;
    while (is >> w && w != "nElec") {
    }
    int ne = 0, nd = 0;
    if (w != "nElec" || !(is >> ne) || !(is >> w) || w != "ndim" || !(is >> nd) || ne <= 0) return QWG_ERR_INPUT;
    pos.assign((size_t)ne * 3, 0.0);
    for (int e = 0; e < ne; e++)
      for (int d = 0; d < 3; d++)
        if (!(is >> pos[(size_t)e * 3 + d])) return QWG_ERR_INPUT;
    double weight = 1.0, sign = 1.0;
    if (!(is >> w)) return QWG_ERR_INPUT;
    if (ieq(w, "DMC")) {
      std::string k;
      if (!(is >> w) || w != "{" || !(is >> k >> weight) || !(is >> k >> sign) || !(is >> w) || w != "}")
        return QWG_ERR_INPUT;
      if (!(is >> w)) return QWG_ERR_INPUT;
    }
    if (w != "}") return QWG_ERR_INPUT;
    f(ne, pos, weight, sign);
  }
  return QWG_OK;
}

}  // namespace

extern "C" {

int qwg_write_configs(const char* path, const double* R, const double* weight, const double* sign, int nw,
                      int nelec) {
  if (!path || !R || nw <= 0 || nelec <= 0) return QWG_ERR_ARG;
  const std::string backup = std::string(path) + ".backup";
  std::rename(path, backup.c_str());  // as write_configurations: the previous file becomes the backup
  std::ofstream os(path);
  if (!os) return QWG_ERR_INPUT;
  os.precision(15);
  for (int w = 0; w < nw; w++) {
    os << " walker { \n";
    os << "nElec " << nelec << " ndim " << 3 << "\n";
    const double* p = R + (size_t)w * nelec * 3;
    for (int e = 0; e < nelec; e++) os << p[3 * e] << " " << p[3 * e + 1] << " " << p[3 * e + 2] << " \n";
    if (weight) {
      os << "DMC { \n";
      os << "weight " << weight[w] << "\n";
      os << "sign " << (sign ? sign[w] : 1.0) << "\n";
      os << "}\n";
    }
    os << " } \n";
  }
  return os ? QWG_OK : QWG_ERR_INPUT;
}

int qwg_count_configs(const char* path, int* nw, int* nelec) {
  if (!path || !nw) return QWG_ERR_ARG;
  int n = 0, ne = -1, bad = 0;
  int rc = parse(path, [&](int e, const std::vector<double>&, double, double) {
    if (ne >= 0 && e != ne) bad = 1;
    ne = e;
    n++;
  });
  if (rc != QWG_OK || bad) return QWG_ERR_INPUT;
  *nw = n;
  if (nelec) *nelec = ne < 0 ? 0 : ne;
  return QWG_OK;
}

int qwg_read_configs(const char* path, double* R, double* weight, double* sign, int maxw, int nelec, int* nw_read) {
  if (!path || !R || maxw <= 0 || nelec <= 0) return QWG_ERR_ARG;
  int n = 0, bad = 0;
  int rc = parse(path, [&](int e, const std::vector<double>& pos, double wt, double sg) {
    if (e != nelec) { bad = 1; return; }
    if (n >= maxw) return;
    for (size_t k = 0; k < pos.size(); k++) R[(size_t)n * nelec * 3 + k] = pos[k];
    if (weight) weight[n] = wt;
    if (sign) sign[n] = sg;
    n++;
  });
  if (rc != QWG_OK || bad) return QWG_ERR_INPUT;
  if (nw_read) *nw_read = n;
  return QWG_OK;
}

}  // extern "C"
