/* fix wall/gran/b200 -- fix wall/gran (src/fix_wall_gran.cpp) whose contact
 * forces run on the B200 under run_style verlet/b200; selected by "-sf b200"
 * through Modify::add_fix (src/modify.cpp:824-835).  Accepts the accelerated
 * grammar only: model hertz tangential history [rolling_friction cdt], then
 * "primitive type T {x,y,z}plane pos" or "primitive type T {x,y,z}cylinder
 * radius c1 c2" or "mesh n_meshes N meshes id ...", then
 * [tangential_damping on|off]; any other keyword is an error. */
#ifdef FIX_CLASS

FixStyle(wall/gran/b200,FixWallGranB200)

#else

#ifndef LMP_FIX_WALL_GRAN_B200_H
#define LMP_FIX_WALL_GRAN_B200_H

#include <string>
#include <vector>

#include "fix_wall_gran.h"

namespace LAMMPS_NS {

class FixWallGranB200 : public FixWallGran {
 public:
  enum Kind { PLANE, CYLINDER, MESH };
  FixWallGranB200(class LAMMPS *, int, char **);

  Kind kind() const { return kind_; }
  int dim() const { return dim_; }
  double param(int k) const { return param_[k]; }   // plane: pos; cylinder: radius c1 c2
  int wall_type() const { return atom_type_wall_; }
  int rolling_cdt() const { return rolling_cdt_; }
  int tangential_damping() const { return tangential_damping_; }
  // per-atom primitive-wall contact history (FixWallGran's property/atom), or NULL
  class FixPropertyAtom *primitive_history() const { return fix_history_primitive_; }

 private:
  Kind kind_;
  int dim_;
  double param_[3];
  int rolling_cdt_, tangential_damping_;
};

}

#endif
#endif
