/* Stand-in for upstream GENESIS 1.3 v4's Collective (wakes; absent from the
 * reference tree).  Test infrastructure for the oracle/_ref build. */
#ifndef G4REF_UPSTREAM_COLLECTIVE_H_
#define G4REF_UPSTREAM_COLLECTIVE_H_
class Collective {
 public:
  void initWake(unsigned int, unsigned int, double, double*, double*, double*,
                double*, double, double, bool) {}
  bool hasWakeDefined() { return false; }
};
#endif
