/* Stand-in for upstream GENESIS 1.3 v4's EFieldSolver (space charge; absent
 * from the reference tree) with space charge switched off, the case the
 * oracle covers (src/Core/BeamSolverCUDA.cpp:525-562 takes the slice-eloss
 * branch).  Test infrastructure for the oracle/_ref build. */
#ifndef G4REF_UPSTREAM_EFIELDSOLVER_H_
#define G4REF_UPSTREAM_EFIELDSOLVER_H_
#include <vector>
#include "Particle.h"
class EFieldSolver {
 public:
  void init(double, int, int, int, double, bool) {}
  bool hasShortRange() { return false; }
  void shortRange(std::vector<Particle>*, double, double, int) {}
  double getEField(int) { return 0.0; }
  void allocateForOutput(unsigned long) {}
  double getSCField(int) { return 0.0; }
};
#endif
