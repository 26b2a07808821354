/* fix mesh/surface/b200 -- see fix_mesh_surface_b200.h */
#include "fix_mesh_surface_b200.h"

#include <cstdlib>
#include <cstring>
#include <string>

#include "error.h"

using namespace LAMMPS_NS;

FixMeshSurfaceB200::FixMeshSurfaceB200(LAMMPS *lmp, int narg, char **arg)
  : FixMeshSurface(lmp, narg, arg), curvature_(0.)
{
  // FixMesh / FixMeshSurface have parsed the keywords (src/fix_mesh.cpp:
  // 105-280, src/fix_mesh_surface.cpp:110-215); count what each takes
  int i = 3;
  std::string bad;
  while (i < narg && bad.empty()) {
    const char *k = arg[i];
    if (!strcmp(k, "file") || !strcmp(k, "type") || !strcmp(k, "verbose") || !strcmp(k, "scale") ||
        !strcmp(k, "curvature_tolerant")) {
      i += 2;
    } else if (!strcmp(k, "curvature")) {
      if (i + 1 < narg) curvature_ = atof(arg[i + 1]);
      i += 2;
    } else if (!strcmp(k, "move")) {
      i += 4;
    } else if (!strcmp(k, "rotate")) {   // rotate axis ax ay az angle a
      i += 7;
    } else {
      bad = k;
    }
  }
  if (!bad.empty()) {
    std::string msg = "fix mesh/surface/b200: keyword '" + bad + "' is outside the accelerated path (file, type, "
                      "verbose, scale, move, rotate, curvature, curvature_tolerant)";
    error->all(FLERR, msg.c_str());
  }
}
