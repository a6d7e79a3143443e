/* Stand-in for upstream GENESIS 1.3 v4's EFieldSolver (space charge; absent
 * from the reference tree).  By default space charge is off, the case the
 * reference's slice-loss branch covers (src/Core/BeamSolverCUDA.cpp:549-560).
 * g4ref_set_particle_ez hands it a per-particle field instead, so that the
 * reference's per-particle branch (:525-547) and its UseParticleEz kernels
 * run on given values: shortRange(beam, current, gammaz2, is) records the
 * slice, getEField(ip) returns field[off[is] + ip].  Test infrastructure for
 * the oracle/_ref build. */
#ifndef G4REF_UPSTREAM_EFIELDSOLVER_H_
#define G4REF_UPSTREAM_EFIELDSOLVER_H_
#include <vector>
#include "Particle.h"
namespace g4ref_sc {
inline const double* field = nullptr;  // per particle, slice-contiguous
inline const int* off = nullptr;       // slice offsets of the current call
}  // namespace g4ref_sc
class EFieldSolver {
 public:
  void init(double, int, int, int, double, bool) {}
  bool hasShortRange() { return g4ref_sc::field != nullptr; }
  void shortRange(std::vector<Particle>*, double, double, int is) { slice_ = is; }
  double getEField(int ip) { return g4ref_sc::field[g4ref_sc::off[slice_] + ip]; }
  void allocateForOutput(unsigned long) {}
  double getSCField(int) { return 0.0; }

 private:
  int slice_ = 0;
};
#endif
