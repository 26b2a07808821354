/* fix mesh/surface/b200 -- fix mesh/surface (src/fix_mesh_surface.cpp) whose
 * triangles become the device's mesh wall under run_style verlet/b200.
 * Accepts: file, type, verbose, scale, move, rotate, curvature,
 * curvature_tolerant (the import keywords that only shape the element list);
 * other keywords (temperature, surface velocities, heal, precision,
 * element_exclusion_list, ...) are outside the accelerated path. */
#ifdef FIX_CLASS

FixStyle(mesh/surface/b200,FixMeshSurfaceB200)

#else

#ifndef LMP_FIX_MESH_SURFACE_B200_H
#define LMP_FIX_MESH_SURFACE_B200_H

#include "fix_mesh_surface.h"

namespace LAMMPS_NS {

class FixMeshSurfaceB200 : public FixMeshSurface {
 public:
  FixMeshSurfaceB200(class LAMMPS *, int, char **);
  double curvature() const { return curvature_; }   // 0: the reference's default

 private:
  double curvature_;
};

}

#endif
#endif
