/* fix wall/gran/b200 -- see fix_wall_gran_b200.h */
#include "fix_wall_gran_b200.h"

#include <cstdlib>
#include <cstring>

#include "b200_args.h"
#include "error.h"

using namespace LAMMPS_NS;

FixWallGranB200::FixWallGranB200(LAMMPS *lmp, int narg, char **arg)
  : FixWallGran(lmp, narg, arg), kind_(PLANE), dim_(2), rolling_cdt_(0), tangential_damping_(1)
{
  param_[0] = param_[1] = param_[2] = 0.;
  // FixWallGran's constructor (src/fix_wall_gran.cpp:161-382) has checked the
  // grammar; here only the accelerated subset passes
  B200::ModelArgs m;
  int i = m.parse_pairs(narg, arg, 3);
  bool have_geom = false;
  while (i >= 0 && i < narg && m.bad.empty()) {
    if (!strcmp(arg[i], "primitive") && i + 3 < narg && !strcmp(arg[i + 1], "type")) {
      const char *w = arg[i + 3];
      const int d = w[0] - 'x';
      if (d < 0 || d > 2) { m.fail("primitive", w); break; }
      if (!strcmp(w + 1, "plane") && i + 4 < narg) {
        kind_ = PLANE;
        dim_ = d;
        param_[0] = atof(arg[i + 4]);
        i += 5;
      } else if (!strcmp(w + 1, "cylinder") && i + 6 < narg) {
        kind_ = CYLINDER;
        dim_ = d;
        for (int k = 0; k < 3; k++) param_[k] = atof(arg[i + 4 + k]);
        i += 7;
      } else {
        m.fail("primitive", w);
        break;
      }
      have_geom = true;
    } else if (!strcmp(arg[i], "mesh")) {
      kind_ = MESH;
      have_geom = true;
      i += 1;
    } else if (!strcmp(arg[i], "n_meshes") && i + 1 < narg) {
      const int nm = atoi(arg[i + 1]);
      i += 2;
      if (!strcmp(arg[i], "meshes")) i += 1 + nm;
    } else {
      const int used = m.parse_setting(narg, arg, i);
      if (!used) {
        m.fail(arg[i], i + 1 < narg ? arg[i + 1] : "");
        break;
      }
      i += used;
    }
  }
  if (m.bad.empty() && !have_geom) m.bad = "primitive or mesh (required)";
  if (!m.bad.empty()) {
    std::string msg = "fix wall/gran/b200: '" + m.bad + "' is outside the accelerated path (model hertz "
                      "tangential history [rolling_friction cdt]; primitive {x,y,z}plane / {x,y,z}cylinder or "
                      "mesh; tangential_damping on|off)";
    error->all(FLERR, msg.c_str());
  }
  rolling_cdt_ = m.rolling_cdt;
  tangential_damping_ = m.tangential_damping;
}
