/* Stand-in for upstream GENESIS 1.3 v4's Sorting (absent from the reference
 * tree).  Test infrastructure for the oracle/_ref build. */
#ifndef G4REF_UPSTREAM_SORTING_H_
#define G4REF_UPSTREAM_SORTING_H_
class Sorting {};
#endif
