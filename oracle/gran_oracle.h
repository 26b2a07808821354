/*
 * gran_oracle.h -- CPU oracle for the LIGGGHTS granular hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * algorithm (LIGGGHTS-PUBLIC 3.8.0) used by tests/, by the smoke check and by
 * the CPU-baseline leg of bench.py as the checker.  The product path never
 * links, loads or calls it.
 *
 * Parity status: the reference cannot be compiled from a few of its own
 * source files (its contact-model headers include build-generated style
 * headers, src/contact_models.h:65-69, and the path needs the whole LAMMPS
 * core), so the oracle is NOT pinned against reference binaries
 * ("parity unpinned").  It is pinned instead against analytic known-answer
 * cases (tests/test_oracle_kat.py) and it restates, operation by operation,
 * the reference arithmetic cited at each function.
 *
 * Scope: one serial "rank" (no MPI), orthogonal box, periodic images as
 * ghost atoms exactly as Comm::borders creates them, Verlet::setup/run step
 * order, pair gran model hertz tangential history [rolling_friction cdt],
 * fix wall/gran primitive {x,y,z}plane and mesh, fix gravity, fix nve/sphere,
 * atom_modify sort.
 */
#ifndef GRAN_ORACLE_H
#define GRAN_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_sim orc_sim;

typedef struct {
    int ntypes;
    double dt;
    double skin;                 /* neighbor <skin> bin                       */
    double boxlo[3], boxhi[3];
    int periodic[3];
    int every, delay, check;     /* neigh_modify every/delay/check            */
    int sortfreq;                /* atom_modify sort <freq> <binsize>         */
    double sortbinsize;
    int rolling_cdt;             /* pair_style gran ... rolling_friction cdt  */
    int tangential_damping;      /* model option, default on                  */
    /* fix property/global: youngsModulus, poissonsRatio (peratomtype),
       coefficientRestitution, coefficientFriction, coefficientRollingFriction
       (peratomtypepair, row-major ntypes x ntypes)                           */
    const double *youngs, *poisson, *restitution, *friction, *rollfriction;
} orc_params;

/* post_force fix kinds, processed in the order they were added */
enum { ORC_FIX_GRAVITY = 1, ORC_FIX_WALL_PLANE = 2, ORC_FIX_WALL_MESH = 3, ORC_FIX_MOVE_MESH = 4 };

orc_sim *orc_create(const orc_params *p, int n,
                    const double *x, const double *v, const double *omega,
                    const double *radius, const double *rmass,
                    const int *type, const int *tag);
void orc_destroy(orc_sim *s);

/* fix ID all gravity <mag> vector dx dy dz */
int orc_add_gravity(orc_sim *s, double mag, double dx, double dy, double dz);
/* fix ID all wall/gran model hertz tangential history [rolling_friction cdt]
   primitive type <wtype> {x,y,z}plane <pos> ; dim = 0,1,2 */
int orc_add_wall_plane(orc_sim *s, int dim, double pos, int wall_type, int rolling_cdt);
/* fix ID all wall/gran ... primitive type <wtype> {x,y,z}cylinder <radius> <c1> <c2>
   (axis along dim through (c1, c2) in the other two coordinates, in cyclic order) */
int orc_add_wall_cylinder(orc_sim *s, int dim, double radius, double c1, double c2, int wall_type, int rolling_cdt);
/* fix mesh/surface (nodes as read from the STL: ntri x 3 x 3) + its own
   fix wall/gran ... mesh n_meshes 1 meshes <id>; returns fix index */
int orc_add_wall_mesh(orc_sim *s, int ntri, const double *nodes, int wall_type,
                      double curvature, int rolling_cdt);

/* fix move/mesh mesh <id> rotate origin ox oy oz axis ax ay az period T
   on the mesh of fix index ifix_mesh; returns fix index */
int orc_add_move_mesh_rotate(orc_sim *s, int ifix_mesh, double ox, double oy, double oz,
                             double ax, double ay, double az, double period);
/* fix move/mesh mesh <id> linear vx vy vz; returns fix index */
int orc_add_move_mesh_linear(orc_sim *s, int ifix_mesh, double vx, double vy, double vz);
/* current nodes (ntri x 3 x 3) and node velocities of a mesh fix; returns ntri */
int orc_get_mesh_nodes(orc_sim *s, int ifix, double *nodes, double *vnode);
/* element geometry, 29 doubles per triangle (centre, bounding radius, edge
   vectors, edge lengths, edge normals, surface normal, precision) */
int orc_get_mesh_geom(orc_sim *s, int ifix, double *geom);

/* Verlet::setup */
int orc_setup(orc_sim *s);
/* Verlet::run(n) */
int orc_run(orc_sim *s, int nsteps);

/* ---- state access (current local order) ---- */
int orc_nlocal(orc_sim *s);
int orc_nghost(orc_sim *s);
long orc_ntimestep(orc_sim *s);
int orc_nbuilds(orc_sim *s);
void orc_get_atoms(orc_sim *s, double *x, double *v, double *omega,
                   double *f, double *torque, int *tag);
/* half-list pairs: returns count; arrays may be NULL to query count */
int orc_get_pairs(orc_sim *s, int cap, int *tag_i, int *tag_j, int *flag, double *hist);
/* fix insert/pack over a region block + particledistribution/discrete of
   particletemplate/sphere templates with constant radius and density
   (src/fix_insert.cpp, src/fix_insert_pack.cpp,
   src/fix_particledistribution_discrete.cpp, src/fix_template_sphere.cpp).
   Field layout identical to the library's gb2_insert_pack. */
typedef struct {
    int seed;
    double region_lo[3], region_hi[3];
    double volumefraction_region;
    int particles_in_region;
    double mass_in_region;
    int insert_every, start, maxattempt, overlapcheck, all_in, exact_number, vel_style;
    double vel[3], vel_fluct[3], omega[3];
    int ntry_mc, check_dist_from_subdomain_border;
    int dist_seed, dist_mass_based, ntemplates;
    int tmpl_type[8];
    double tmpl_radius[8], tmpl_density[8], tmpl_weight[8];
    int max_atoms;
    int tmpl_radius_style[8];   /* 0 constant, 1 uniform(radius, radius2), 2 gaussian(radius, radius2) */
    double tmpl_radius2[8];
    int tmpl_seed[8];
    int region_style;             /* 0 block, 1 cylinder */
    int cyl_axis;
    double cyl_c1, cyl_c2, cyl_radius, cyl_lo, cyl_hi;
} orc_insert_pack;
int orc_add_insert_pack(orc_sim *s, const orc_insert_pack *p);
int orc_insert_stats(orc_sim *s, long *ninserted, double *massinserted, long *next_step);
int orc_park_after(int seed, int n);
void orc_get_radius_mass(orc_sim *s, double *radius, double *rmass);
int orc_add_mesh_wear(orc_sim *s, int ifix, const double *k_finnie);
int orc_get_mesh_wear(orc_sim *s, int ifix, double *wear);
/* mesh contact history in the restart layout (sorts the slots first, as write_restart does) */
int orc_get_mesh_history(orc_sim *s, int ifix, int cap, int *npartner, int *tri, double *hist);
int orc_upload_mesh_hist(orc_sim *s, int ifix, int n, const int *npartner, const int *tri, const double *hist);
/* compute pair/gran/local: rows of the columns keys selects (bit b of keys:
   pos, vel, id, force, force_normal, force_tangential, torque, torque_normal,
   torque_tangential, history, contactArea, delta, contactPoint) */
int orc_pair_gran_local(orc_sim *s, unsigned keys, int cap, double *rows);
/* fix mesh/surface/stress: per-element force and totals of the last step */
int orc_add_mesh_stress(orc_sim *s, int ifix, double px, double py, double pz);
int orc_get_mesh_stress(orc_sim *s, int ifix, double *tri_f, double *tot6);
int orc_get_mesh_sigma(orc_sim *s, int ifix, double *sigma_n, double *sigma_t);
/* restart: contact history in FixContactHistory's partner layout */
int orc_upload_history(orc_sim *s, int n, const int *npartner, const int *ptag, const double *hist);
int orc_get_history(orc_sim *s, int *npartner, int *ptag, double *hist);
int orc_upload_wall_hist(orc_sim *s, int ifix, int n, const double *hist);
/* compute contact/atom (skin 0) per owned atom, atom order */
int orc_contact_atom(orc_sim *s, double *out);
/* per-atom primitive-wall shear history of fix index ifix (3 per atom) */
int orc_get_wall_hist(orc_sim *s, int ifix, double *hist);
/* mesh contacts of fix ifix: (tag, tri id, hist[3]) for every occupied slot */
int orc_get_mesh_contacts(orc_sim *s, int ifix, int cap, int *tag, int *tri, double *hist);
/* mesh topology of fix ifix: per triangle edge_active[3], corner_active[3],
   obtuse index; returns ntri after duplicate removal */
int orc_get_mesh_topology(orc_sim *s, int ifix, unsigned char *edge_active,
                          unsigned char *corner_active, int *obtuse);
/* per-atom candidate triangle count of a mesh fix (fix_nneighs) */
int orc_get_mesh_nneighs(orc_sim *s, int ifix, int *nneighs);

/* stand-alone pair kernel for known-answer tests: one i-j contact computed
   exactly like Granular<...>::compute_force for a single pair */
void orc_pair_force(const orc_params *p, const double xi[3], const double xj[3],
                    const double vi[3], const double vj[3],
                    const double wi[3], const double wj[3],
                    double ri, double rj, double mi, double mj, int ti, int tj,
                    double shear[3], int shearupdate,
                    double fi[3], double ti_out[3], double fj[3], double tj_out[3]);

const char *orc_error(orc_sim *s);

#ifdef __cplusplus
}
#endif
#endif
