/* fix move/mesh/b200 -- see fix_move_mesh_b200.h */
#include "fix_move_mesh_b200.h"

#include <cstdlib>
#include <cstring>

#include "error.h"
#include "force.h"

using namespace LAMMPS_NS;

FixMoveMeshB200::FixMoveMeshB200(LAMMPS *lmp, int narg, char **arg)
  : FixMoveMesh(lmp, narg, arg), kind_(ROTATE), period_(0.)
{
  for (int k = 0; k < 3; k++) origin_[k] = axis_[k] = vel_[k] = 0.;
  // fix ID group move/mesh mesh <id> <mover> ... (the base constructor has
  // checked the grammar, src/fix_move_mesh.cpp:70-100)
  mesh_id_ = arg[4];
  const char *mv = arg[5];
  if (!strcmp(mv, "rotate") && narg >= 16) {
    kind_ = ROTATE;
    for (int k = 0; k < 3; k++) {
      origin_[k] = force->numeric(FLERR, arg[7 + k]);
      axis_[k] = force->numeric(FLERR, arg[11 + k]);
    }
    period_ = force->numeric(FLERR, arg[15]);
  } else if (!strcmp(mv, "linear") && narg >= 9) {
    kind_ = LINEAR;
    for (int k = 0; k < 3; k++) vel_[k] = force->numeric(FLERR, arg[6 + k]);
  } else {
    std::string msg = std::string("fix move/mesh/b200: mover '") + mv + "' is outside the accelerated path "
                      "(rotate origin x y z axis x y z period T, linear vx vy vz)";
    error->all(FLERR, msg.c_str());
  }
}
