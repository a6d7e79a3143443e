/* Stand-in for upstream GENESIS 1.3 v4's Diagnostic and FilterDiagnostics
 * (absent from the reference tree): the members DiagnosticCUDA reads
 * (src/Core/DiagnosticCUDA.cpp:381-412, filter_.beam.* and filter_.field.*).
 * val[2] holds the beam records, val[3 + i] those of field i.
 * Test infrastructure for the oracle/_ref build. */
#ifndef G4REF_UPSTREAM_DIAGNOSTIC_H_
#define G4REF_UPSTREAM_DIAGNOSTIC_H_
#include <map>
#include <string>
#include <vector>
struct FilterDiagnostics {
  struct {
    bool global = true, spatial = true, energy = true, current = true;
    bool auxiliar = true, twiss = true, exclharm = false;
    int harm = 1;
  } beam;
  struct {
    bool global = true, spatial = true, fft = true, intensity = true;
  } field;
};
class Diagnostic {
 public:
  std::vector<double> zout;
  std::vector<std::map<std::string, std::vector<double> > > val;
};
#endif
