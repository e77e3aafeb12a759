// QWalk-format log output (include/qwg.h: qwg_log_header, qwg_log_block).
// Host-only; the field names, order and number format follow what the
// reference's Properties_block::restoreFromLog / gosling read back.
#include <cmath>
#include <cstdio>
#include <fstream>
#include <iomanip>
#include <string>

#include "../../include/qwg.h"

namespace {

void array_sec(std::ostream& os, const std::string& indent, const char* label, double v) {
  os << indent << label << " { " << v << "   } \n";
}

}  // namespace

extern "C" {

int qwg_log_header(const char* path, const char* method, const char* label, double timestep, int nconfig,
                   int nstep) {
  if (!path || !method || !label) return QWG_ERR_ARG;
  std::ofstream os(path, std::ios::app);
  if (!os) return QWG_ERR_INPUT;
  const std::string m = method;
  os << "#-------------------------------------------------\n";
  os << "#" << m << " run: timestep " << timestep;
  if (m == "VMC") os << " nconfig " << nconfig << " steps " << nstep;
  os << "\n";
  os << "#-------------------------------------------------\n\n\n";
  os << "init { \n";
  os << "   label " << label << "\n";
  os << "}\n";
  return os ? QWG_OK : QWG_ERR_INPUT;
}

int qwg_log_block(const char* path, const char* label, const qwg_block_stats* s) {
  if (!path || !label || !s) return QWG_ERR_ARG;
  std::ofstream os(path, std::ios::app);
  if (!os) return QWG_ERR_INPUT;
  os.precision(16);
  const std::string in = "   ";
  os << "block { \n";
  os << in << "label " << label << "\n";
  os << in << "totweight " << s->npoints << "\n";
  os << in << "nautocorr " << 0 << "\n";
  array_sec(os, in, "total_energy", s->energy);
  array_sec(os, in, "total_energyvar", s->var_energy);
  array_sec(os, in, "weight", s->weight);
  array_sec(os, in, "weightvar", s->var_weight);
  array_sec(os, in, "kinetic_energy", s->kinetic);
  array_sec(os, in, "kinetic_energyvar", s->var_kinetic);
  array_sec(os, in, "potential_energy", s->potential);
  array_sec(os, in, "potential_energyvar", s->var_potential);
  array_sec(os, in, "nonlocal_energy", s->nonlocal);
  array_sec(os, in, "nonlocal_energyvar", s->var_nonlocal);
  os << in << "autocorr_energy { } \n";
  os << "} \n\n";
  return os ? QWG_OK : QWG_ERR_INPUT;
}

}  // extern "C"
