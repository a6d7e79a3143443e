/* Stand-in for upstream GENESIS 1.3 v4's Particle (absent from the reference
 * tree).  Test infrastructure for the oracle/_ref build. */
#ifndef G4REF_UPSTREAM_PARTICLE_H_
#define G4REF_UPSTREAM_PARTICLE_H_
class Particle {
 public:
  double gamma, theta, x, y, px, py;
};
#endif
