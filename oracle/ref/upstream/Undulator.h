/* Stand-in for upstream GENESIS 1.3 v4's Undulator class (absent from the
 * reference tree), declaring only the members the reference's CUDA files
 * call.  Test infrastructure: it lets the reference's own sources compile
 * into oracle/_ref/ so that their outputs can pin the oracle.
 * Call sites: src/Core/BeamSolverCUDA.cpp:503,514-522,607,625-630,
 * src/Core/FieldSolverADICUDA.cpp:697,707,722-729,
 * src/Core/TrackBeamCUDA.cpp:163-167,261-262, src/Core/ControlCUDA.cpp:133. */
#ifndef G4REF_UPSTREAM_UNDULATOR_H_
#define G4REF_UPSTREAM_UNDULATOR_H_
#include <vector>

class Undulator {
 public:
  /* per-step tables, indexed by getStep() */
  std::vector<double> aw, ax, ay, ku, kx, ky, gradx, grady;
  std::vector<double> qf, qx, qy, cx, cy, chic_angle, chic_lb, chic_ld, chic_lt;
  std::vector<double> phasesh;
  std::vector<int> marker;
  std::vector<int> in_und;
  double gammaref = 0.0;
  double fc_by_harm[16] = {0};
  int istep = 0;

  int getStep() { return istep; }
  bool inUndulator() { return in_und[istep] != 0; }
  double fc(int harm) { return fc_by_harm[harm]; }
  double getaw() { return aw[istep]; }
  double getku() { return ku[istep]; }
  double getGammaRef() { return gammaref; }
  double autophase() { return phasesh[istep]; }
  int getMarker() { return marker[istep]; }
  void getUndulatorParameters(double* a, double* dx, double* dy, double* k,
                              double* fx, double* fy) {
    *a = aw[istep]; *dx = ax[istep]; *dy = ay[istep];
    *k = ku[istep]; *fx = kx[istep]; *fy = ky[istep];
  }
  void getQuadrupoleParameters(double* q, double* dx, double* dy) {
    *q = qf[istep]; *dx = qx[istep]; *dy = qy[istep];
  }
  void getCorrectorParameters(double* x, double* y) { *x = cx[istep]; *y = cy[istep]; }
  void getChicaneParameters(double* angle, double* lb, double* ld, double* lt) {
    *angle = chic_angle[istep]; *lb = chic_lb[istep]; *ld = chic_ld[istep]; *lt = chic_lt[istep];
  }
};
#endif
