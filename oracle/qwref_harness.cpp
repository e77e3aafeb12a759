// Per-configuration evaluation harness linked against the reference QWalk
// objects (built from the reference sources by oracle/Makefile).
//
// TEST INFRASTRUCTURE ONLY: this program writes the golden vectors that pin
// the oracle restatement and the CUDA engine.  Nothing in the product links
// or runs it.
//
// Usage: qwref_harness <deck> <inputs.bin> <outputs.bin>
//
// The deck is a QWalk input file (SYSTEM / PSEUDO / TRIALFUNC sections); its
// METHOD section, if any, is ignored.  Sections are parsed and modules built
// exactly as the reference driver does (program_utils/ooqmc.cpp:214-310 and
// method/Dmc_method.cpp:192-223).
//
// inputs.bin  (little endian):
//   int32 nconf, int32 nelec, int32 nmove
//   nconf x { f64 pos[nelec][3]; f64 rot[3][3] (rows x,y,z of the quadrature
//             rotation, Pseudopotential.cpp:830-864); nmove x { int32 e;
//             f64 newpos[3] } }
// outputs.bin:
//   int32 nconf, int32 nelec, int32 nmove
//   nconf x { f64 logpsi; f64 sign; f64 grad[nelec][3]; f64 lap[nelec];
//             f64 kinetic; f64 potential; f64 nonlocal;
//             nmove x { f64 dlogpsi; f64 signratio; f64 grad[3]; f64 lap } }
// where grad/lap are amp(0,1..3) and amp(0,4) - |phase(0,1..3)|^2 of
// Slat_Jastrow::getLap (wavefunction/Slat_Jastrow.cpp:313-357), i.e. the
// real parts of grad psi/psi and lap psi/psi (the phase terms vanish for real
// orbitals).  For complex orbitals (CORBITALS) "sign" is the phase of psi
// (phase(0,0), Wf_return.cpp:129-152) and "signratio" the phase difference
// of the move.  kinetic/potential/nonlocal are
// System::calcKinetic, System::calcLoc and the deterministic
// Pseudopotential::calcNonlocWithTest (system/Pseudopotential.cpp:412-424).

#include "Qmc_std.h"
#include "qmc_io.h"
#include "System.h"
#include "Wavefunction.h"
#include "Wavefunction_data.h"
#include "Pseudopotential.h"
#include "Sample_point.h"
#include <cstdio>
#include <cstdint>
#include <fstream>

static void die(const char* m) { fprintf(stderr, "qwref_harness: %s\n", m); exit(2); }

template <class T> static void rd(FILE* f, T* p, size_t n) {
  if (fread(p, sizeof(T), n, f) != n) die("short read");
}
template <class T> static void wr(FILE* f, const T* p, size_t n) {
  if (fwrite(p, sizeof(T), n, f) != n) die("short write");
}

int main(int argc, char** argv) {
  if (argc != 4) die("usage: qwref_harness deck inputs.bin outputs.bin");
  ifstream deck(argv[1]);
  if (!deck) die("cannot open deck");
  vector<string> words;
  parsefile(deck, words);

  vector<vector<string> > pseudotext;
  vector<string> sec, syssec, wftext;
  unsigned int pos = 0;
  while (readsection(words, pos, sec, "PSEUDO") != 0) pseudotext.push_back(sec);
  pos = 0;
  while (readsection(words, pos, sec, "TRIALFUNC") != 0) wftext.insert(wftext.end(), sec.begin(), sec.end());
  pos = 0;
  if (!readsection(words, pos, syssec, "SYSTEM")) die("no SYSTEM section");

  System* sys = NULL;
  allocate(syssec, sys);
  Pseudopotential* psp = NULL;
  sys->generatePseudo(pseudotext, psp);
  psp->setDeterministic(1);
  Wavefunction_data* wfdata = NULL;
  allocate(wftext, sys, wfdata);
  Wavefunction* wf = NULL;
  wfdata->generateWavefunction(wf);
  Sample_point* sample = NULL;
  sys->generateSample(sample);
  sample->attachObserver(wf);
  int nwf = wf->nfunc();

  FILE* fin = fopen(argv[2], "rb");
  if (!fin) die("cannot open inputs");
  int32_t hdr[3];
  rd(fin, hdr, 3);
  int nconf = hdr[0], nelec = hdr[1], nmove = hdr[2];
  if (nelec != sample->electronSize()) die("electron count mismatch");
  FILE* fout = fopen(argv[3], "wb");
  if (!fout) die("cannot open outputs");
  wr(fout, hdr, 3);

  Array1<doublevar> p(3), rx(3), ry(3), rz(3);
  vector<double> R(nelec * 3), out;
  Array1<doublevar> accept(max(psp->nTest(), 1));
  accept = 1.0;
  for (int c = 0; c < nconf; c++) {
    rd(fin, R.data(), nelec * 3);
    double rot[9];
    rd(fin, rot, 9);
    for (int d = 0; d < 3; d++) { rx(d) = rot[d]; ry(d) = rot[3 + d]; rz(d) = rot[6 + d]; }
    psp->rotateQuadrature(rx, ry, rz);

    for (int e = 0; e < nelec; e++) {
      for (int d = 0; d < 3; d++) p(d) = R[e * 3 + d];
      sample->setElectronPos(e, p);
    }
    wf->notify(all_electrons_move, 0);
    wf->updateLap(wfdata, sample);
    Wf_return val(nwf, 2);
    wf->getVal(wfdata, 0, val);
    out.clear();
    out.push_back(val.amp(0, 0));
    out.push_back(val.is_complex ? val.phase(0, 0) : double(val.sign(0)));
    vector<double> lapv(nelec);
    for (int e = 0; e < nelec; e++) {
      Wf_return lap(nwf, 5);
      wf->getLap(wfdata, e, lap);
      for (int d = 1; d < 4; d++) out.push_back(lap.amp(0, d));
      lapv[e] = lap.amp(0, 4);
      if (lap.is_complex)
        for (int d = 1; d < 4; d++) lapv[e] -= lap.phase(0, d) * lap.phase(0, d);
    }
    out.insert(out.end(), lapv.begin(), lapv.end());
    Array1<doublevar> kin(nwf), nonloc(nwf);
    sys->calcKinetic(wfdata, sample, wf, kin);
    doublevar pot = sys->calcLoc(sample);
    psp->calcNonlocWithTest(wfdata, sys, sample, wf, accept, nonloc);
    out.push_back(kin(0));
    out.push_back(pot);
    out.push_back(nonloc(0));

    for (int m = 0; m < nmove; m++) {
      int32_t e;
      double np[3];
      rd(fin, &e, 1);
      rd(fin, np, 3);
      if (e < 0 || e >= nelec) die("bad electron index in move");
      // fresh state for every move: the base configuration, full recompute
      for (int k = 0; k < nelec; k++) {
        for (int d = 0; d < 3; d++) p(d) = R[k * 3 + d];
        sample->setElectronPos(k, p);
      }
      wf->notify(all_electrons_move, 0);
      wf->updateLap(wfdata, sample);
      Wf_return v0(nwf, 2);
      wf->getVal(wfdata, 0, v0);
      for (int d = 0; d < 3; d++) p(d) = np[d];
      sample->setElectronPos(e, p);
      wf->updateLap(wfdata, sample);
      Wf_return v1(nwf, 2);
      wf->getVal(wfdata, 0, v1);
      Wf_return lap(nwf, 5);
      wf->getLap(wfdata, e, lap);
      out.push_back(v1.amp(0, 0) - v0.amp(0, 0));
      out.push_back(v1.is_complex ? v1.phase(0, 0) - v0.phase(0, 0) : double(v1.sign(0) * v0.sign(0)));
      for (int d = 1; d < 4; d++) out.push_back(lap.amp(0, d));
      double l4 = lap.amp(0, 4);
      if (lap.is_complex)
        for (int d = 1; d < 4; d++) l4 -= lap.phase(0, d) * lap.phase(0, d);
      out.push_back(l4);
    }
    wr(fout, out.data(), out.size());
  }
  fclose(fin);
  fclose(fout);
  return 0;
}
