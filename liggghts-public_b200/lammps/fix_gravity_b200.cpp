/* fix gravity/b200 -- see fix_gravity_b200.h */
#include "fix_gravity_b200.h"

#include <cstring>

#include "error.h"

using namespace LAMMPS_NS;

FixGravityB200::FixGravityB200(LAMMPS *lmp, int narg, char **arg) : FixGravity(lmp, narg, arg)
{
  // FixGravity's styles (src/fix_gravity.cpp:75-150): only a constant
  // magnitude with "vector" is the device's gravity
  if (narg != 8 || strcmp(arg[4], "vector") || strstr(arg[3], "v_") == arg[3] || strstr(arg[5], "v_") == arg[5] ||
      strstr(arg[6], "v_") == arg[6] || strstr(arg[7], "v_") == arg[7])
    error->all(FLERR, "fix gravity/b200: only 'fix ID group gravity <magnitude> vector <x> <y> <z>' with constants "
                      "is on the accelerated path");
}
