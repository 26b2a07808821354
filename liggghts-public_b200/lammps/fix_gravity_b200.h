/* fix gravity/b200 -- fix gravity (src/fix_gravity.cpp) applied on the device
 * under run_style verlet/b200 ("magnitude vector x y z" only: constant
 * magnitude and direction, the form the device path supports). */
#ifdef FIX_CLASS

FixStyle(gravity/b200,FixGravityB200)

#else

#ifndef LMP_FIX_GRAVITY_B200_H
#define LMP_FIX_GRAVITY_B200_H

#include "fix_gravity.h"

namespace LAMMPS_NS {

class FixGravityB200 : public FixGravity {
 public:
  FixGravityB200(class LAMMPS *, int, char **);
  double magnitude_value() const { return magnitude; }
  void direction(double *d) const { d[0] = xdir; d[1] = ydir; d[2] = zdir; }
};

}

#endif
#endif
