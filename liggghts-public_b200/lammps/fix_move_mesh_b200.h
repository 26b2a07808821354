/* fix move/mesh/b200 -- fix move/mesh (src/fix_move_mesh.cpp) whose mesh
 * motion runs on the device under run_style verlet/b200; the "rotate origin
 * x y z axis x y z period T" (src/mesh_mover_rotation.cpp:66-96) and
 * "linear vx vy vz" (src/mesh_mover_linear.cpp:66-77) movers only. */
#ifdef FIX_CLASS

FixStyle(move/mesh/b200,FixMoveMeshB200)

#else

#ifndef LMP_FIX_MOVE_MESH_B200_H
#define LMP_FIX_MOVE_MESH_B200_H

#include <string>

#include "fix_move_mesh.h"

namespace LAMMPS_NS {

class FixMoveMeshB200 : public FixMoveMesh {
 public:
  enum Kind { ROTATE, LINEAR };
  FixMoveMeshB200(class LAMMPS *, int, char **);

  Kind kind() const { return kind_; }
  const std::string &mesh_id() const { return mesh_id_; }
  const double *origin() const { return origin_; }
  const double *axis() const { return axis_; }
  double period() const { return period_; }
  const double *velocity() const { return vel_; }

 private:
  Kind kind_;
  std::string mesh_id_;
  double origin_[3], axis_[3], period_, vel_[3];
};

}

#endif
#endif
