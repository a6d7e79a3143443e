// Undulator.h -- per-step lattice tables with the accessor API the reference's
// CUDA path calls on upstream GENESIS 1.3 v4's Undulator class (call sites:
// src/Core/BeamSolverCUDA.cpp:503,514-522,607,625-630;
// src/Core/FieldSolverADICUDA.cpp:697,707,722-729;
// src/Core/TrackBeamCUDA.cpp:163-167,261-262; src/Core/Gencore.cpp:172-174,229,247;
// src/Core/ControlCUDA.cpp:133).
#pragma once

#include <string>
#include <vector>

#include "g4b.h"

namespace g4h {

struct LatticeStep {
  g4b_step st{};
  double z = 0;         // position at the end of the step
  double slip = 0;      // slippage in units of lambda0
  int helical = 0;
  int marker = 0;       // bit0 dump beam, bit1 dump field, bit2 sort, bit3 stop
};

class Undulator {
 public:
  std::vector<LatticeStep> steps;
  double gamma0 = 0, lambda0 = 0;
  int output_step = 1;

  // iteration (Gencore main loop: `while (und->advance(rank))`)
  void reset() { istep_ = -1; }
  // position the iteration at step i (the next advance() goes to i + 1)
  void seek(int i) { istep_ = i; }
  bool advance(int /*rank*/ = 0) { return ++istep_ < (int)steps.size(); }
  int getStep() const { return istep_; }
  int nstep() const { return (int)steps.size(); }
  const g4b_step& current() const { return steps[istep_].st; }

  double steplength() const { return steps[istep_].st.delz; }
  bool inUndulator() const { return steps[istep_].st.in_undulator != 0; }
  double getaw() const { return steps[istep_].st.aw; }
  double getku() const { return steps[istep_].st.ku; }
  double getGammaRef() const { return gamma0; }
  double autophase() const { return steps[istep_].st.autophase; }
  bool isHelical() const { return steps[istep_].helical != 0; }
  double slippage() const { return steps[istep_].slip; }
  double getz() const { return istep_ < 0 ? 0.0 : steps[istep_].z; }
  // markers acting at the start of the current step: those placed after the
  // previous step (after the loop: those after the last step)
  int getMarker() const {
    const int k = istep_ < (int)steps.size() ? istep_ : (int)steps.size();
    return k <= 0 ? 0 : steps[k - 1].marker;
  }
  bool outstep() const { return ((istep_ + 1) % output_step) == 0 || istep_ + 1 == nstep(); }
  int outlength() const { return 1 + (nstep() + output_step - 1) / output_step; }
  double fc(int harm) const;
  double fc_at(int i, int harm) const;

 private:
  int istep_ = -1;
};

// Coupling factor aw * JJ_h (planar) or aw (helical, h = 1).
double coupling(double aw, int harm, bool helical);

// Parses the .lat subset and expands `beamline`; returns false with
// g4h::set_error on failure.
bool build_lattice(const std::string& text, const std::string& beamline, double delz,
                   double gamma0, double lambda0, Undulator& und);

}  // namespace g4h
