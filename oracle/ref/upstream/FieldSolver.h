/* Stand-in for upstream GENESIS 1.3 v4's FieldSolver base class (absent from
 * the reference tree): the three virtual members FieldSolverADICUDA and
 * FieldSolverFFTCUDA override (include/FieldSolverADICUDA.h:20-25).
 * Test infrastructure for the oracle/_ref build. */
#ifndef G4REF_UPSTREAM_FIELDSOLVER_H_
#define G4REF_UPSTREAM_FIELDSOLVER_H_
class Field;
class Beam;
class Undulator;
class FieldSolver {
 public:
  virtual ~FieldSolver() {}
  virtual void init(double, double, double, unsigned int) {}
  virtual void advance(double, Field*, Beam*, Undulator*) {}
  virtual void initSourceFilter(double, double, double, bool) {}
};
class FieldSolverADI : public FieldSolver {};
#endif
