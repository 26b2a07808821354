/* run_style verlet/b200 -- Verlet::run (src/verlet.cpp:264-388) with the
 * whole time step resident on one B200 (libgranb200, include/granb200.h).
 *
 * Selected by "-sf b200" / "suffix b200" through Update::create_integrate
 * (src/update.cpp:338-373), or by "run_style verlet/b200 [precision fp64|
 * split] [device N]".  setup() runs the reference's own Verlet::setup on the
 * CPU (so every fix and output sets itself up as usual), then builds the
 * device context from the LAMMPS state: atoms in local order, material
 * properties, the b200 fixes in definition order, and the pair, primitive
 * wall and mesh contact histories.  run(n) advances the device in chunks
 * that end at output steps; there the owned atoms come back to the host in
 * the device's order (the host's per-atom data of every fix permuted
 * alongside, as Atom::sort does), so thermo and dumps see the current state.
 * cleanup() also writes the contact histories back, so write_restart and a
 * following run continue where the device stopped.
 *
 * Only the accelerated path runs here: pair gran/b200, fix gravity/b200,
 * wall/gran/b200 (with mesh/surface/b200), move/mesh/b200, nve/sphere/b200,
 * all on group all, orthogonal box, newton off.  Any other fix is rejected
 * by init() through error->all; computes that read the neighbour list are
 * not refreshed during a run. */
#ifdef INTEGRATE_CLASS

IntegrateStyle(verlet/b200,VerletB200)

#else

#ifndef LMP_VERLET_B200_H
#define LMP_VERLET_B200_H

#include <vector>

#include "verlet.h"

struct gb2_ctx;

namespace LAMMPS_NS {

class VerletB200 : public Verlet {
 public:
  VerletB200(class LAMMPS *, int, char **);
  virtual ~VerletB200();
  virtual void init();
  virtual void setup();
  virtual void setup_minimal(int);
  virtual void run(int);
  void cleanup();

 private:
  gb2_ctx *ctx_;
  int precision_, device_;
  bool host_current_;
  // device fix index of each mesh wall (by its FixMeshSurface) and of each
  // primitive wall, for the history transfers
  std::vector<class FixWallGranB200 *> walls_;
  std::vector<int> wall_ifix_;                        // one per walls_ entry (primitive) or per mesh
  std::vector<class FixMeshSurface *> meshes_;
  std::vector<int> mesh_ifix_;

  void check(int rc, const char *what);
  void build_context();
  void download_atoms();
  void write_back_history();
};

}

#endif
#endif
