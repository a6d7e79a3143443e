/* Stand-in for upstream GENESIS 1.3 v4's Control (absent from the reference
 * tree): applyMarker as ControlCUDA::applyMarker forwards to it
 * (src/Core/ControlCUDA.cpp:131-146).  Test infrastructure for the
 * oracle/_ref build. */
#ifndef G4REF_UPSTREAM_CONTROL_H_
#define G4REF_UPSTREAM_CONTROL_H_
#include <vector>
class Beam;
class Field;
class Undulator;
class Control {
 public:
  bool applyMarker(Beam*, std::vector<Field*>*, Undulator*, bool&) { return false; }
};
#endif
