/* Stand-in for upstream GENESIS 1.3 v4's CPU BeamSolver (absent from the
 * reference tree): the members include/Beam.h's inline functions name.
 * Test infrastructure for the oracle/_ref build. */
#ifndef G4REF_UPSTREAM_BEAMSOLVER_H_
#define G4REF_UPSTREAM_BEAMSOLVER_H_
class BeamSolver {
 public:
  void initEField(double, int, int, int, double, bool) {}
  void checkAllocation(unsigned long) {}
  double getSCField(int) { return 0.0; }
};
#endif
