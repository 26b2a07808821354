/* fix nve/sphere/b200 -- fix nve/sphere (src/fix_nve_sphere.cpp:138-246)
 * integrated on the device under run_style verlet/b200; the plain form
 * (no "update dipole" / CAddRhoFluid) only.  Its CPU integration still
 * serves any non-b200 integrator. */
#ifdef FIX_CLASS

FixStyle(nve/sphere/b200,FixNVESphereB200)

#else

#ifndef LMP_FIX_NVE_SPHERE_B200_H
#define LMP_FIX_NVE_SPHERE_B200_H

#include <cstring>

#include "error.h"
#include "fix_nve_sphere.h"

namespace LAMMPS_NS {

class FixNVESphereB200 : public FixNVESphere {
 public:
  FixNVESphereB200(class LAMMPS *lmp, int narg, char **arg) : FixNVESphere(lmp, narg, arg)
  {
    if (narg > 3)
      error->all(FLERR, "fix nve/sphere/b200: keyword 'update' is outside the accelerated path");
  }
};

}

#endif
#endif
