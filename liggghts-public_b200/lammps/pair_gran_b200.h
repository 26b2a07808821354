/* pair_style gran/b200 -- pair_style gran (Hertz/history [rolling cdt]) whose
 * per-step force evaluation runs on the B200 under run_style verlet/b200.
 * Selected by "-sf b200" / "suffix b200" through Force::new_pair
 * (src/force.cpp:225-250).  The CPU implementation of the reference
 * (PairGranProxy, src/pair_gran_proxy.cpp) still serves Verlet::setup and
 * any non-b200 integrator; the accepted grammar is exactly the accelerated
 * model: model hertz tangential history [rolling_friction cdt] [surface
 * default] [cohesion off] [tangential_damping on|off]. */
#ifdef PAIR_CLASS

PairStyle(gran/b200,PairGranB200)

#else

#ifndef LMP_PAIR_GRAN_B200_H
#define LMP_PAIR_GRAN_B200_H

#include "pair_gran_proxy.h"

namespace LAMMPS_NS {

class PairGranB200 : public PairGranProxy {
 public:
  PairGranB200(class LAMMPS *);
  virtual void settings(int, char **);

  int rolling_cdt() const { return rolling_cdt_; }
  int tangential_damping() const { return tangential_damping_; }

 private:
  int rolling_cdt_, tangential_damping_;
};

}

#endif
#endif
