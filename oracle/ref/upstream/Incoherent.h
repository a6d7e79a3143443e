/* Stand-in for upstream GENESIS 1.3 v4's Incoherent (absent from the
 * reference tree).  Test infrastructure for the oracle/_ref build. */
#ifndef G4REF_UPSTREAM_INCOHERENT_H_
#define G4REF_UPSTREAM_INCOHERENT_H_
class Incoherent {
 public:
  void init(int, int, bool, bool) {}
};
#endif
