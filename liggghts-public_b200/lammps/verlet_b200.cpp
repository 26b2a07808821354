/* run_style verlet/b200 -- see verlet_b200.h */
#include "verlet_b200.h"

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "granb200.h"

#include "atom.h"
#include "atom_vec.h"
#include "domain.h"
#include "error.h"
#include "fix.h"
#include "fix_contact_history.h"
#include "fix_contact_history_mesh.h"
#include "fix_gravity_b200.h"
#include "fix_mesh_surface.h"
#include "fix_mesh_surface_b200.h"
#include "fix_move_mesh_b200.h"
#include "fix_nve_sphere_b200.h"
#include "fix_property_atom.h"
#include "fix_property_global.h"
#include "fix_wall_gran_b200.h"
#include "force.h"
#include "lmptype.h"
#include "modify.h"
#include "neighbor.h"
#include "output.h"
#include "pair_gran_b200.h"
#include "timer.h"
#include "tri_mesh.h"
#include "update.h"

using namespace LAMMPS_NS;

namespace {

// an integer in a double slot, as the reference's exchange buffers carry it
// (the ubuf unions of src/fix.h:302, src/atom_vec.h:164)
union IntSlot {
  double d;
  int64_t i;
  explicit IntSlot(int v) : i(v) {}
};

// Atom keeps the atom_modify sort bin size private (src/atom.h:319); the
// device needs it to bin atoms as Atom::sort does.  Read through an explicit
// instantiation with the member's address (such instantiations are exempt
// from access checking).
template <typename Tag, typename Tag::type M>
struct MemberOf {
  friend typename Tag::type member_ptr(Tag) { return M; }
};
struct AtomUserBinsize {
  typedef double Atom::*type;
  friend type member_ptr(AtomUserBinsize);
};
template struct MemberOf<AtomUserBinsize, &Atom::userbinsize>;

// write access to a mesh's nodes and centres (protected members of
// MultiNodeMesh, src/multi_node_mesh.h:214-224): the device moved the mesh,
// the host copy follows at download points
struct MeshAccess : public TriMesh {
  static double ***nodes(TriMesh *m) { return static_cast<MeshAccess *>(m)->node_.begin(); }
  static double **centers(TriMesh *m) { return static_cast<MeshAccess *>(m)->center_.begin(); }
};
}  // namespace

VerletB200::VerletB200(LAMMPS *lmp, int narg, char **arg)
  : Verlet(lmp, narg, arg), ctx_(NULL), precision_(GB2_PREC_FP64), device_(0), host_current_(true)
{
  for (int i = 0; i < narg; i++) {
    if (!strcmp(arg[i], "precision") && i + 1 < narg) {
      if (!strcmp(arg[i + 1], "fp64")) precision_ = GB2_PREC_FP64;
      else if (!strcmp(arg[i + 1], "split")) precision_ = GB2_PREC_SPLIT;
      else error->all(FLERR, "run_style verlet/b200: precision fp64 or split");
      i++;
    } else if (!strcmp(arg[i], "device") && i + 1 < narg) {
      device_ = atoi(arg[++i]);
    } else {
      error->all(FLERR, "run_style verlet/b200: keywords are precision fp64|split and device N");
    }
  }
}

VerletB200::~VerletB200()
{
  if (ctx_) gb2_destroy(ctx_);
}

void VerletB200::check(int rc, const char *what)
{
  if (rc >= 0) return;
  char buf[512] = "";
  if (ctx_) gb2_last_error(ctx_, buf, sizeof buf);
  static char msg[1024];
  snprintf(msg, sizeof msg, "run_style verlet/b200: %s failed (%d): %s", what, rc, buf);
  error->all(FLERR, msg);
}

/* Verlet::init, then the checks that the run is on the accelerated path */
void VerletB200::init()
{
  Verlet::init();
  if (!dynamic_cast<PairGranB200 *>(force->pair))
    error->all(FLERR, "run_style verlet/b200 needs pair_style gran/b200 (run with -sf b200 or suffix b200)");
  if (domain->triclinic) error->all(FLERR, "run_style verlet/b200: orthogonal boxes only");
  if (force->newton_pair) error->all(FLERR, "run_style verlet/b200: newton off is required");
  if (!atom->radius_flag || !atom->rmass_flag || !atom->omega_flag || !atom->torque_flag)
    error->all(FLERR, "run_style verlet/b200: atom style sphere (granular) is required");
  int nnve = 0;
  for (int i = 0; i < modify->nfix; i++) {
    Fix *f = modify->fix[i];
    const char *s = f->style;
    // a suffixed fix keeps the plain style name (Modify::add_fix passes the
    // unsuffixed arguments, src/modify.cpp:826-834), so classify by class
    const bool nve = dynamic_cast<FixNVESphereB200 *>(f) != NULL;
    const bool user = nve || dynamic_cast<FixGravityB200 *>(f) || dynamic_cast<FixWallGranB200 *>(f) ||
                      dynamic_cast<FixMeshSurfaceB200 *>(f) || dynamic_cast<FixMoveMeshB200 *>(f);
    // fixes the reference creates for the granular path itself, and global
    // material properties
    const bool internal = !strncmp(s, "property/", 9) || !strncmp(s, "contacthistory", 14) ||
                          !strcmp(s, "neighlist/mesh") || !strncmp(s, "contactproperty/atom", 20);
    static char msg[512];
    if (!user && !internal) {
      snprintf(msg, sizeof msg, "run_style verlet/b200: fix %s (style %s) is outside the accelerated path", f->id, s);
      error->all(FLERR, msg);
    }
    if (user && f->igroup != 0) {
      snprintf(msg, sizeof msg, "run_style verlet/b200: fix %s must act on group all", f->id);
      error->all(FLERR, msg);
    }
    if (nve) nnve++;
  }
  if (nnve != 1) error->all(FLERR, "run_style verlet/b200 needs exactly one fix nve/sphere/b200 on group all");
}

/* the reference's Verlet::setup on the CPU (every fix and output sets up as
   usual), then the device context from that state */
void VerletB200::setup()
{
  Verlet::setup();
  build_context();
  check(gb2_setup(ctx_), "gb2_setup");
  host_current_ = true;
}

void VerletB200::setup_minimal(int)
{
  error->all(FLERR, "run_style verlet/b200 does not run minimizations");
}

static FixPropertyGlobal *material(LAMMPS *lmp, const char *name, const char *kind, int n1, int n2)
{
  Fix *f = lmp->modify->find_fix_property(name, "property/global", kind, n1, n2, "run_style verlet/b200");
  return static_cast<FixPropertyGlobal *>(f);
}

void VerletB200::build_context()
{
  if (ctx_) gb2_destroy(ctx_);
  ctx_ = NULL;
  walls_.clear();
  wall_ifix_.clear();
  meshes_.clear();
  mesh_ifix_.clear();

  PairGranB200 *pg = dynamic_cast<PairGranB200 *>(force->pair);
  gb2_params p;
  memset(&p, 0, sizeof p);
  const int nt = atom->ntypes;
  p.ntypes = nt;
  p.dt = update->dt;
  p.skin = neighbor->skin;
  for (int d = 0; d < 3; d++) {
    p.boxlo[d] = domain->boxlo[d];
    p.boxhi[d] = domain->boxhi[d];
    p.periodic[d] = domain->periodicity[d];
  }
  p.neigh_every = neighbor->every;
  p.neigh_delay = neighbor->delay;
  p.neigh_check = neighbor->dist_check;
  p.sort_freq = atom->sortfreq;
  p.sort_binsize = atom->*member_ptr(AtomUserBinsize());
  p.rolling_cdt = pg->rolling_cdt();
  p.tangential_damping = pg->tangential_damping();
  p.precision = precision_;
  p.device = device_;
  const int rc = gb2_create(&p, &ctx_);
  if (rc) {
    ctx_ = NULL;
    error->all(FLERR, "run_style verlet/b200: no usable B200 (gb2_create failed)");
  }

  // material properties (fix property/global, src/global_properties.cpp:411-560)
  bool rolling = pg->rolling_cdt() != 0;
  for (int i = 0; i < modify->nfix; i++) {
    FixWallGranB200 *w = dynamic_cast<FixWallGranB200 *>(modify->fix[i]);
    if (w && w->rolling_cdt()) rolling = true;
  }
  std::vector<double> E(nt), nu(nt), e(nt * nt), mu(nt * nt), mur(nt * nt, 0.);
  FixPropertyGlobal *fE = material(lmp, "youngsModulus", "peratomtype", nt, 0);
  FixPropertyGlobal *fnu = material(lmp, "poissonsRatio", "peratomtype", nt, 0);
  FixPropertyGlobal *fe = material(lmp, "coefficientRestitution", "peratomtypepair", nt, nt);
  FixPropertyGlobal *fmu = material(lmp, "coefficientFriction", "peratomtypepair", nt, nt);
  FixPropertyGlobal *fmur = rolling ? material(lmp, "coefficientRollingFriction", "peratomtypepair", nt, nt) : NULL;
  for (int i = 0; i < nt; i++) {
    E[i] = fE->compute_vector(i);
    nu[i] = fnu->compute_vector(i);
    for (int j = 0; j < nt; j++) {
      e[i * nt + j] = fe->compute_array(i, j);
      mu[i * nt + j] = fmu->compute_array(i, j);
      if (fmur) mur[i * nt + j] = fmur->compute_array(i, j);
    }
  }
  check(gb2_set_materials(ctx_, E.data(), nu.data(), e.data(), mu.data(), mur.data()), "gb2_set_materials");

  // owned atoms in local order
  const int n = atom->nlocal;
  check(gb2_upload_atoms(ctx_, n, atom->x[0], atom->v[0], atom->omega[0], atom->radius, atom->rmass, atom->type,
                         atom->tag), "gb2_upload_atoms");
  check(gb2_set_timestep(ctx_, (long)update->ntimestep), "gb2_set_timestep");

  // post_force fixes in definition order; movers once their mesh exists
  for (int i = 0; i < modify->nfix; i++) {
    Fix *f = modify->fix[i];
    if (FixGravityB200 *g = dynamic_cast<FixGravityB200 *>(f)) {
      double dir[3];
      g->direction(dir);
      check(gb2_add_gravity(ctx_, g->magnitude_value(), dir), "gb2_add_gravity");
    } else if (FixWallGranB200 *w = dynamic_cast<FixWallGranB200 *>(f)) {
      if (w->tangential_damping() != pg->tangential_damping())
        error->all(FLERR, "run_style verlet/b200: tangential_damping must be the same for the pair style and walls");
      if (w->kind() == FixWallGranB200::PLANE) {
        const int k = gb2_add_wall_plane(ctx_, w->dim(), w->param(0), w->wall_type(), w->rolling_cdt());
        check(k, "gb2_add_wall_plane");
        walls_.push_back(w);
        wall_ifix_.push_back(k);
      } else if (w->kind() == FixWallGranB200::CYLINDER) {
        const int k = gb2_add_wall_cylinder(ctx_, w->dim(), w->param(0), w->param(1), w->param(2), w->wall_type(),
                                            w->rolling_cdt());
        check(k, "gb2_add_wall_cylinder");
        walls_.push_back(w);
        wall_ifix_.push_back(k);
      } else {
        for (int im = 0; im < w->n_meshes(); im++) {
          FixMeshSurface *fm = w->mesh_list()[im];
          TriMesh *mesh = fm->triMesh();
          const int ntri = mesh->sizeLocal();
          std::vector<double> nodes(9 * (size_t)(ntri > 0 ? ntri : 1));
          for (int t = 0; t < ntri; t++)
            for (int j = 0; j < 3; j++) mesh->node_slow(t, j, &nodes[9 * (size_t)t + 3 * j]);
          FixMeshSurfaceB200 *fb = dynamic_cast<FixMeshSurfaceB200 *>(fm);
          const int k = gb2_add_wall_mesh(ctx_, ntri, nodes.data(), fm->atomTypeWall(), fb ? fb->curvature() : 0.,
                                          w->rolling_cdt());
          check(k, "gb2_add_wall_mesh");
          meshes_.push_back(fm);
          mesh_ifix_.push_back(k);
        }
      }
    }
  }
  for (int i = 0; i < modify->nfix; i++) {
    FixMoveMeshB200 *mv = dynamic_cast<FixMoveMeshB200 *>(modify->fix[i]);
    if (!mv) continue;
    int k = -1;
    for (size_t m = 0; m < meshes_.size(); m++)
      if (mv->mesh_id() == meshes_[m]->id) k = mesh_ifix_[m];
    if (k < 0) error->all(FLERR, "run_style verlet/b200: fix move/mesh/b200 moves a mesh no wall/gran/b200 uses");
    if (mv->kind() == FixMoveMeshB200::ROTATE)
      check(gb2_add_move_mesh_rotate(ctx_, k, mv->origin(), mv->axis(), mv->period()), "gb2_add_move_mesh_rotate");
    else
      check(gb2_add_move_mesh_linear(ctx_, k, mv->velocity()), "gb2_add_move_mesh_linear");
  }

  // contact histories as they stand (FixContactHistory partner arrays,
  // primitive-wall property/atom, mesh contact slots)
  FixContactHistory *ch = pg->get_fix_history();
  if (ch) {
    if (ch->get_dnum() != 3) error->all(FLERR, "run_style verlet/b200: unexpected contact history size");
    std::vector<int> np(n), pt;
    std::vector<double> ph;
    for (int i = 0; i < n; i++) {
      np[i] = ch->n_partner(i);
      for (int k = 0; k < np[i]; k++) {
        pt.push_back(ch->partner(i, k));
        const double *h = ch->contacthistory(i, k);
        ph.insert(ph.end(), h, h + 3);
      }
    }
    pt.resize(pt.size() + 1);   // non-null buffers when no atom has a partner
    ph.resize(ph.size() + 3);
    check(gb2_upload_history(ctx_, n, np.data(), pt.data(), ph.data()), "gb2_upload_history");
  }
  for (size_t k = 0; k < walls_.size(); k++) {
    FixPropertyAtom *h = walls_[k]->primitive_history();
    if (!h || !h->array_atom) continue;
    std::vector<double> hist(3 * (size_t)n);
    for (int i = 0; i < n; i++)
      for (int c = 0; c < 3; c++) hist[3 * i + c] = h->array_atom[i][c];
    check(gb2_upload_wall_history(ctx_, wall_ifix_[k], n, hist.data()), "gb2_upload_wall_history");
  }
  for (size_t k = 0; k < meshes_.size(); k++) {
    FixContactHistoryMesh *cm = meshes_[k]->contactHistory();
    if (!cm) continue;
    std::vector<int> np(n, 0), tri;
    std::vector<double> hist;
    for (int i = 0; i < n; i++)
      for (int j = 0; j < cm->nneighs(i); j++) {
        const int t = cm->get_partner_idTri(i, j);
        if (t < 0) continue;
        np[i]++;
        tri.push_back(t);
        const double *h = cm->contacthistory(i, j);
        hist.insert(hist.end(), h, h + 3);
      }
    tri.resize(tri.size() + 1);
    hist.resize(hist.size() + 3);
    check(gb2_upload_mesh_history(ctx_, mesh_ifix_[k], n, np.data(), tri.data(), hist.data()),
          "gb2_upload_mesh_history");
  }
}

/* Verlet::run: the device advances in chunks that end at output steps */
void VerletB200::run(int n)
{
  const bigint last = update->ntimestep + n;
  while (update->ntimestep < last) {
    bigint stop = last;
    if (output->next > update->ntimestep && output->next < stop) stop = output->next;
    const int k = (int)(stop - update->ntimestep);
    timer->stamp();
    check(gb2_run(ctx_, k), "gb2_run");
    update->ntimestep += k;
    host_current_ = false;
    if (update->ntimestep == output->next) {
      download_atoms();
      write_back_history();
      timer->stamp(TIME_PAIR);
      output->write(update->ntimestep);
      timer->stamp(TIME_OUTPUT);
    }
  }
  check(gb2_sync(ctx_), "gb2_sync");
  timer->stamp(TIME_PAIR);
}

/* owned atoms back to the host in the device's order: the host's per-atom
   data (every fix's included, through AtomVec::copy) is permuted into that
   order with Atom::sort's in-place cycles (src/atom.cpp:1371-1394), then x,
   v, omega, f, torque are overwritten with the device's */
void VerletB200::download_atoms()
{
  const int n = atom->nlocal;
  std::vector<double> x(3 * (size_t)n), v(3 * (size_t)n), w(3 * (size_t)n), f(3 * (size_t)n), t(3 * (size_t)n);
  std::vector<int> tag(n);
  int m = 0;
  check(gb2_download_atoms(ctx_, n, &m, x.data(), v.data(), w.data(), f.data(), t.data(), tag.data()),
        "gb2_download_atoms");
  if (m != n) error->all(FLERR, "run_style verlet/b200: the device holds another number of atoms");
  std::vector<int> permute(n), current(n);
  for (int d = 0; d < n; d++) {
    const int h = atom->map(tag[d]);
    if (h < 0 || h >= n) error->all(FLERR, "run_style verlet/b200: atom tag not found on the host");
    permute[d] = h;
    current[d] = d;
  }
  atom->map_clear();
  if (n == atom->nmax) atom->avec->grow(0);
  for (int i = 0; i < n; i++) {
    if (current[i] == permute[i]) continue;
    atom->avec->copy(i, n, 0);
    int empty = i;
    while (permute[empty] != i) {
      atom->avec->copy(permute[empty], empty, 0);
      empty = current[empty] = permute[empty];
    }
    atom->avec->copy(n, empty, 0);
    current[empty] = permute[empty];
  }
  atom->nghost = 0;   // ghost images are rebuilt by the next setup
  atom->map_set();
  for (int i = 0; i < n; i++)
    for (int c = 0; c < 3; c++) {
      atom->x[i][c] = x[3 * i + c];
      atom->v[i][c] = v[3 * i + c];
      atom->omega[i][c] = w[3 * i + c];
      atom->f[i][c] = f[3 * i + c];
      atom->torque[i][c] = t[3 * i + c];
    }
  gb2_stats st;
  if (gb2_get_stats(ctx_, &st) == 0) neighbor->ncalls = st.nbuilds > 0 ? st.nbuilds - 1 : 0;
  // moving meshes: nodes, centres and node velocities ("v") as the device left them
  for (size_t k = 0; k < meshes_.size(); k++) {
    TriMesh *mesh = meshes_[k]->triMesh();
    if (!mesh->isMoving()) continue;
    const int ntri = mesh->sizeLocal();
    int nt = 0;
    std::vector<double> nodes(9 * (size_t)(ntri > 0 ? ntri : 1)), vel(9 * (size_t)(ntri > 0 ? ntri : 1));
    check(gb2_download_mesh_nodes(ctx_, mesh_ifix_[k], ntri, &nt, nodes.data(), vel.data()), "gb2_download_mesh_nodes");
    double ***nd = MeshAccess::nodes(mesh);
    double **ct = MeshAccess::centers(mesh);
    MultiVectorContainer<double, 3, 3> *vp = mesh->prop().getElementProperty<MultiVectorContainer<double, 3, 3> >("v");
    for (int t = 0; t < ntri && t < nt; t++) {
      double c[3] = {0., 0., 0.};
      for (int j = 0; j < 3; j++)
        for (int q = 0; q < 3; q++) {
          nd[t][j][q] = nodes[9 * (size_t)t + 3 * j + q];
          if (vp) (*vp)(t)[j][q] = vel[9 * (size_t)t + 3 * j + q];
          c[q] = nd[t][j][q] + c[q];
        }
      const double sinv = 1. / 3.0;   // MultiNodeMesh's centre: sum of nodes times 1/3
      for (int q = 0; q < 3; q++) ct[t][q] = sinv * c[q];
    }
  }
  host_current_ = true;
}

/* the device's contact histories into the reference's fixes, in the host
   order download_atoms left: FixContactHistory through pre_exchange (page
   reset, computeflag cleared so the next setup keeps the arrays) and
   unpack_exchange per atom (src/fix_contact_history.cpp:305-425, 529-548),
   primitive walls into their property/atom, mesh slots through
   FixContactHistoryMesh::unpack_exchange (src/fix_contact_history_mesh.cpp:
   573-607) */
void VerletB200::write_back_history()
{
  const int n = atom->nlocal;
  PairGranB200 *pg = dynamic_cast<PairGranB200 *>(force->pair);
  FixContactHistory *ch = pg ? pg->get_fix_history() : NULL;
  std::vector<double> buf;
  if (ch) {
    int na = 0, ntot = 0;
    check(gb2_download_history(ctx_, 0, 0, &na, &ntot, NULL, NULL, NULL, NULL), "gb2_download_history");
    std::vector<int> tg(n), np(n), pt(ntot > 0 ? ntot : 1);
    std::vector<double> ph(3 * (size_t)(ntot > 0 ? ntot : 1));
    check(gb2_download_history(ctx_, n, ntot, &na, &ntot, tg.data(), np.data(), pt.data(), ph.data()),
          "gb2_download_history");
    ch->pre_exchange();
    size_t off = 0;
    for (int i = 0; i < n; i++) {
      buf.assign(1, IntSlot(np[i]).d);
      for (int k = 0; k < np[i]; k++, off++) {
        buf.push_back(IntSlot(pt[off]).d);
        buf.insert(buf.end(), &ph[3 * off], &ph[3 * off] + 3);
      }
      ch->unpack_exchange(i, buf.data());
    }
  }
  for (size_t k = 0; k < walls_.size(); k++) {
    FixPropertyAtom *h = walls_[k]->primitive_history();
    if (!h || !h->array_atom) continue;
    std::vector<double> hist(3 * (size_t)n);
    check(gb2_download_wall_history(ctx_, wall_ifix_[k], n, hist.data()), "gb2_download_wall_history");
    for (int i = 0; i < n; i++)
      for (int c = 0; c < 3; c++) h->array_atom[i][c] = hist[3 * i + c];
  }
  for (size_t k = 0; k < meshes_.size(); k++) {
    FixContactHistoryMesh *cm = meshes_[k]->contactHistory();
    if (!cm) continue;
    int na = 0, ntot = 0;
    check(gb2_download_mesh_history(ctx_, mesh_ifix_[k], 0, 0, &na, &ntot, NULL, NULL, NULL, NULL),
          "gb2_download_mesh_history");
    std::vector<int> tg(n), np(n), tri(ntot > 0 ? ntot : 1);
    std::vector<double> hist(3 * (size_t)(ntot > 0 ? ntot : 1));
    check(gb2_download_mesh_history(ctx_, mesh_ifix_[k], n, ntot, &na, &ntot, tg.data(), np.data(), tri.data(),
                                    hist.data()), "gb2_download_mesh_history");
    size_t off = 0;
    for (int i = 0; i < n; i++) {
      buf.assign(1, IntSlot(np[i]).d);
      for (int q = 0; q < np[i]; q++, off++) {
        buf.push_back(IntSlot(tri[off]).d);
        buf.insert(buf.end(), &hist[3 * off], &hist[3 * off] + 3);
      }
      cm->unpack_exchange(i, buf.data());
    }
  }
}

/* the final state and histories back on the host, then Verlet::cleanup */
void VerletB200::cleanup()
{
  if (ctx_ && !host_current_) {
    download_atoms();
    write_back_history();
  }
  Verlet::cleanup();
}
