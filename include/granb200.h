/*
 * granb200.h -- C ABI of the B200 granular hot-path engine (libgranb200.so).
 *
 * One context = one LIGGGHTS "run" state on one GPU: particles (owned +
 * periodic ghost images), the granular half neighbor list with contact
 * history, wall fixes and the Velocity-Verlet sphere integrator.  The whole
 * time step stays on the device; the host only uploads the initial state and
 * downloads state on request.
 *
 * The entry points replace the following reference interfaces
 * (LIGGGHTS-PUBLIC 3.8.0, paths relative to the project root):
 *   gb2_create / gb2_set_materials  <- pair_style gran ... settings and the
 *       material matrices of MODEL_PARAMS::createYeff/Geff/BetaEff/
 *       CoeffFrict/CoeffRollFrict (src/pair_gran_proxy.cpp:63,
 *       src/global_properties.cpp:411-560)
 *   gb2_upload_atoms               <- read_data Atoms/Velocities into
 *       Atom::x,v,omega,radius,rmass,type,tag (src/atom_vec_sphere.cpp:1055)
 *   gb2_add_gravity                <- FixGravity (src/fix_gravity.cpp:301)
 *   gb2_add_wall_plane             <- FixWallGran primitive {x,y,z}plane
 *       (src/fix_wall_gran.cpp:1024)
 *   gb2_add_wall_mesh              <- FixMeshSurface + FixWallGran mesh
 *       (src/fix_mesh.cpp:343, src/fix_wall_gran.cpp:845)
 *   gb2_setup                      <- Verlet::setup (src/verlet.cpp:134)
 *   gb2_run                        <- Verlet::run (src/verlet.cpp:264): per
 *       step FixNVESphere::initial_integrate, Neighbor::decide, the rebuild
 *       (FixContactHistory::pre_exchange, Domain::pbc, Atom::sort,
 *       Comm::borders, Neighbor::granular_bin_no_newton) or
 *       Comm::forward_comm, PairGran::compute, post_force fixes and
 *       FixNVESphere::final_integrate
 *   gb2_download_atoms             <- lammps_gather_atoms (src/library.cpp)
 *   gb2_download_pairs             <- NeighList firstneigh/firstdouble of the
 *       granular history list (src/neigh_gran.cpp:485)
 *   gb2_download_wall_history      <- fix wall/gran property/atom history
 *   gb2_download_mesh_contacts     <- FixContactHistoryMesh partner_/
 *       contacthistory_ (src/fix_contact_history_mesh.cpp)
 *
 * Every call returns 0 on success or a negative GB2_ERR_* code; the message
 * is available from gb2_last_error.  The ABI is single-host-thread per
 * context; different contexts are independent.
 */
#ifndef GRANB200_H
#define GRANB200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GB2_OK               0
#define GB2_ERR_ARG         -1   /* bad argument / unsupported keyword      */
#define GB2_ERR_CUDA        -2   /* CUDA runtime error                      */
#define GB2_ERR_CAPACITY    -3   /* capacity could not be grown             */
#define GB2_ERR_LOST        -4   /* atom left a non-periodic box            */
#define GB2_ERR_STATE       -5   /* call out of order (e.g. run before setup) */
#define GB2_ERR_UNSUPPORTED -6   /* option outside the accelerated path     */

#define GB2_PREC_FP64   0        /* IEEE FP64 throughout, FMA contraction off */
#define GB2_PREC_SPLIT  1        /* FP32 contact arithmetic on FP64-differenced
                                    positions, FP64 integration              */

typedef struct gb2_ctx gb2_ctx;

typedef struct {
    int ntypes;                  /* atom types 1..ntypes                    */
    double dt;                   /* timestep                                */
    double skin;                 /* neighbor <skin> bin                     */
    double boxlo[3], boxhi[3];   /* orthogonal box                          */
    int periodic[3];             /* boundary p (1) or f (0) per dimension   */
    int neigh_every;             /* neigh_modify every  (default 1)         */
    int neigh_delay;             /* neigh_modify delay  (0 recommended)     */
    int neigh_check;             /* neigh_modify check yes/no               */
    int sort_freq;               /* atom_modify sort <freq> (default 1000)  */
    double sort_binsize;         /* atom_modify sort ... <binsize> (0: auto)*/
    int rolling_cdt;             /* pair_style gran ... rolling_friction cdt*/
    int tangential_damping;      /* model option tangential_damping on/off  */
    int precision;               /* GB2_PREC_FP64 or GB2_PREC_SPLIT          */
    int device;                  /* CUDA device ordinal                     */
} gb2_params;

typedef struct {
    long ntimestep;              /* update->ntimestep                       */
    int nlocal, nghost;
    int nbuilds;                 /* neighbor list builds so far             */
    long npairs;                 /* half-list pairs at the last build       */
    long ntouch;                 /* pairs with a set contact flag           */
    int maxneigh, maxpartner;    /* current per-atom capacities             */
    double time_pair, time_neigh, time_other;   /* device ms, cumulative    */
    long kernel_launches;        /* kernels launched by this context so far */
    /* per-kernel device time (ms, cumulative) while profiling is on */
    double t_integrate, t_pair_tail, t_pair_main, t_forward, t_rebuild;
    long n_pair_main;            /* pair-pass launches timed                */
    long nsteps_rebuild;         /* steps that rebuilt the neighbour list   */
    int maxrev, maxmesh;         /* reverse-entry and mesh-slot capacities  */
    long ngrow;                  /* capacity growths (device reallocations) */
    long n_rebuild_timed;        /* rebuilds timed into t_rebuild (all, while profiling) */
} gb2_stats;

/* contact census of the current state (device reduction): half-list entries,
   touching pairs (rsq < (ri+rj)^2), reverse entries, primitive-wall and mesh
   contacts within reach, mesh candidate slots */
typedef struct {
    long nlist, ntouch, nrev, nwall_list, nwall_touch, nmesh_cand, nmesh_touch;
} gb2_contact_census;

/* context lifecycle.  A context's small page-locked host words (flags and
   counts it reads back from the device) are a 256-byte slot of a pinned
   arena the library shares between contexts: the first context of a process
   locks a 64 KiB block (256 slots; more blocks as more contexts are live at
   once), and those pages stay locked until the process exits. */
int gb2_create(const gb2_params *p, gb2_ctx **out);
int gb2_destroy(gb2_ctx *ctx);

/* fix property/global youngsModulus/poissonsRatio (per type, ntypes values)
   and coefficientRestitution/coefficientFriction/coefficientRollingFriction
   (per type pair, row-major ntypes x ntypes; rollfriction may be NULL when
   rolling friction is off). */
int gb2_set_materials(gb2_ctx *ctx, const double *youngs, const double *poisson,
                      const double *restitution, const double *friction,
                      const double *rollfriction);

/* owned atoms, host arrays: x,v,omega [n][3], radius,rmass [n], type,tag [n].
   Arrays in page-locked memory (gb2_host_alloc) are copied to the device
   directly; others go through the context's pinned staging buffer. */
int gb2_upload_atoms(gb2_ctx *ctx, int n, const double *x, const double *v,
                     const double *omega, const double *radius, const double *rmass,
                     const int *type, const int *tag);

/* post_force fixes, applied in the order they are added */
int gb2_add_gravity(gb2_ctx *ctx, double magnitude, const double dir[3]);
int gb2_add_wall_plane(gb2_ctx *ctx, int dim, double pos, int wall_type, int rolling_cdt);
/* fix ID all wall/gran ... primitive type <wall_type> {x,y,z}cylinder <radius> <c1> <c2>
   (FixWallGran::post_force_primitive with Cylinder<dim>,
   src/primitive_wall_definitions.h:157-206): axis along dim through (c1, c2)
   in the coordinates (dim+1)%3, (dim+2)%3; contact inside and outside the
   shell.  Returns the fix index or a negative error. */
int gb2_add_wall_cylinder(gb2_ctx *ctx, int dim, double radius, double c1, double c2, int wall_type,
                          int rolling_cdt);
/* ntri triangles as read from an STL file, nodes[ntri][3][3]; curvature <= 0
   selects the default 1 - 1e-5.  Returns the fix index (>= 0) or an error. */
int gb2_add_wall_mesh(gb2_ctx *ctx, int ntri, const double *nodes, int wall_type,
                      double curvature, int rolling_cdt);

/* fix ID all move/mesh mesh <mesh-id> rotate origin ox oy oz axis ax ay az period T
   (src/fix_move_mesh.cpp:221 FixMoveMesh::initial_integrate,
    src/mesh_mover_rotation.cpp:66-138 MeshMoverRotate) on the mesh wall of
   fix index ifix_mesh.  Each step rotates the mesh by 2*pi/T*dt about the
   axis through origin, sets the node velocities omega x (node - origin) that
   the wall contact interpolates at the contact point, and forces a neighbour
   rebuild on the step after any node has moved more than skin/2 since the last
   one (src/fix_mesh.cpp:564-588).  Call before gb2_setup; one mover per mesh. */
int gb2_add_move_mesh_rotate(gb2_ctx *ctx, int ifix_mesh, const double origin[3], const double axis[3],
                             double period);
/* fix ID all move/mesh mesh <mesh-id> linear vx vy vz
   (src/mesh_mover_linear.cpp:66-112 MeshMoverLinear): each step shifts the
   mesh by v dt, sets the node velocities to v and forces the rebuild after
   skin/2 as for the rotation.  Call before gb2_setup; one mover per mesh. */
int gb2_add_move_mesh_linear(gb2_ctx *ctx, int ifix_mesh, const double vel[3]);
/* fix insert/pack (src/fix_insert_pack.cpp with src/fix_insert.cpp) over a
 * region block or cylinder, fed by fix particledistribution/discrete
 * (src/fix_particledistribution_discrete.cpp) of fix particletemplate/sphere
 * templates with constant radius and density (src/fix_template_sphere.cpp).
 * Every insertion step (start, then every insert_every steps; insert_every 0
 * = once) forces a neighbour rebuild; the particles already in the region
 * are counted and the particles near it gathered on the device, the
 * reference's Park-Miller draws (src/random_park.cpp) pick positions and
 * velocities on the host, accepted particles are appended to the device
 * arrays with tags beyond the largest tag.  Call after gb2_upload_atoms and
 * before gb2_setup; max_atoms reserves device room for the owned atoms
 * (initial + inserted: an insertion beyond it returns GB2_ERR_CAPACITY).
 * Out of scope here: other region styles, density distributions other than
 * constant, multisphere templates, orientation, set_property. */
#define GB2_INSERT_MAX_TEMPLATES 8
typedef struct {
    int seed;                        /* prime > 10000 (Random::Random, src/random.cpp:55-95) */
    double region_lo[3], region_hi[3];   /* region block, units box */
    /* exactly one target (FixInsertPack::calc_insertion_properties) */
    double volumefraction_region;
    int particles_in_region;
    double mass_in_region;
    int insert_every;                /* >= 0; 0 = once */
    int start;                       /* first insertion step; 0 = the step after the current one */
    int maxattempt;                  /* default 50 */
    int overlapcheck;                /* default 1 */
    int all_in;                      /* default 0 */
    int exact_number;                /* random_distribute exact (1, default) or uncorrelated (0) */
    int vel_style;                   /* 0 constant, 1 uniform, 2 gaussian */
    double vel[3], vel_fluct[3], omega[3];
    int ntry_mc;                     /* region volume Monte Carlo samples, default 100000 */
    int check_dist_from_subdomain_border;   /* default 1 */
    int dist_seed;                   /* particledistribution/discrete seed, prime > 10000 */
    int dist_mass_based;             /* 1: weights are mass fractions; 0: numberbased */
    int ntemplates;
    int tmpl_type[GB2_INSERT_MAX_TEMPLATES];
    double tmpl_radius[GB2_INSERT_MAX_TEMPLATES], tmpl_density[GB2_INSERT_MAX_TEMPLATES];
    double tmpl_weight[GB2_INSERT_MAX_TEMPLATES];
    int max_atoms;
    /* radius distribution of each template (ProbabilityDistribution,
     * src/probability_distribution.h): 0 constant tmpl_radius; 1 uniform
     * between tmpl_radius and tmpl_radius2; 2 gaussian, mean tmpl_radius and
     * sigma tmpl_radius2, cut at +-3 sigma; drawn from the template's own
     * generator (tmpl_seed, prime > 10000) */
    int tmpl_radius_style[GB2_INSERT_MAX_TEMPLATES];
    double tmpl_radius2[GB2_INSERT_MAX_TEMPLATES];
    int tmpl_seed[GB2_INSERT_MAX_TEMPLATES];
    /* region style: 0 block (region_lo/hi), 1 cylinder (RegCylinder,
     * src/region_cylinder.cpp:213-470): axis 0/1/2, centre (c1, c2) in the
     * other two coordinates in x, y, z order, radius, extent lo..hi along the
     * axis; region_lo/hi are then ignored */
    int region_style;
    int cyl_axis;
    double cyl_c1, cyl_c2, cyl_radius, cyl_lo, cyl_hi;
} gb2_insert_pack;
int gb2_add_insert_pack(gb2_ctx *ctx, const gb2_insert_pack *p);
/* fix insert/stream (src/fix_insert_stream.cpp with src/fix_insert.cpp):
 * particles appear in the volume swept by a planar insertion face (a fix
 * mesh/surface, given here as its triangles) extruded against the insertion
 * velocity's normal component v_n, move with v_n regardless of forces (their
 * force and torque read as zero) until they reach the face, and are released
 * there with the insertion velocity and omega.  Insertion steps: start, then
 * every insert_every steps (or the steps v_n takes to cross extrude_length);
 * each inserts int(rate * insert_every * dt + uniform) particles until the
 * total (nparticles or mass; ninsert_inf for no limit) is reached.  The
 * distribution and template fields mean what they mean for insert/pack.
 * One insertion fix (pack or stream) per context; before gb2_setup. */
typedef struct {
    int seed;
    int nface;                       /* insertion face triangles */
    const double *face_nodes;        /* [nface][3][3], planar */
    double nparticles;               /* total count, or 0 with mass */
    double mass;                     /* total mass, or 0 with nparticles */
    int ninsert_inf;                 /* 1: nparticles / mass INF */
    double particlerate, massrate;   /* exactly one > 0 */
    int insert_every;                /* -1: from extrude_length */
    double extrude_length;           /* 0: from insert_every (and duration) */
    int duration;                    /* 0: insert_every */
    int start;                       /* first insertion step; 0 = the step after the current one */
    int maxattempt, overlapcheck, exact_number;
    int vel_style;                   /* 0 constant, 1 uniform, 2 gaussian */
    double vel[3], vel_fluct[3], omega[3];
    int ntry_mc;                     /* insertion-fraction Monte Carlo samples, default 100000 */
    int dist_seed, dist_mass_based, ntemplates;
    int tmpl_type[GB2_INSERT_MAX_TEMPLATES];
    double tmpl_radius[GB2_INSERT_MAX_TEMPLATES], tmpl_density[GB2_INSERT_MAX_TEMPLATES];
    double tmpl_weight[GB2_INSERT_MAX_TEMPLATES];
    int tmpl_radius_style[GB2_INSERT_MAX_TEMPLATES];
    double tmpl_radius2[GB2_INSERT_MAX_TEMPLATES];
    int tmpl_seed[GB2_INSERT_MAX_TEMPLATES];
    int max_atoms;
} gb2_insert_stream;
int gb2_add_insert_stream(gb2_ctx *ctx, const gb2_insert_stream *p);
/* inserted count and mass so far, and the next insertion step (-1 / 0: none) */
int gb2_insert_stats(gb2_ctx *ctx, int ifix, long *ninserted, double *massinserted, long *next_step);
/* current mesh nodes [ntri][3][3] and node velocities (zero for a static mesh)
   of mesh fix ifix; *ntri = element count, nothing written when cap < ntri */
int gb2_download_mesh_nodes(gb2_ctx *ctx, int ifix, int cap, int *ntri, double *nodes, double *vnode);

/* Verlet::setup and Verlet::run(nsteps) */
/* update->ntimestep at the start of the run (default 0): sets the step the
   atom-sort schedule counts from (Atom::sort's nextsort, src/atom.cpp:1315);
   call before gb2_setup */
int gb2_set_timestep(gb2_ctx *ctx, long ntimestep);
int gb2_setup(gb2_ctx *ctx);
int gb2_run(gb2_ctx *ctx, int nsteps);
/* block until all device work of this context has finished */
int gb2_sync(gb2_ctx *ctx);

/* downloads (current owned-atom order; any pointer may be NULL); arrays in
   page-locked memory are written by the device directly */
int gb2_download_atoms(gb2_ctx *ctx, int cap, int *n, double *x, double *v, double *omega,
                       double *f, double *torque, int *tag);
/* page-locked host memory for the atom arrays of gb2_upload_atoms and
   gb2_download_atoms, so their copies run at full bus speed without the
   staging copy (LAMMPS' own Atom arrays are ordinary heap memory,
   src/memory.cpp; this has no reference counterpart).  gb2_host_free
   releases what gb2_host_alloc returned. */
int gb2_host_alloc(size_t bytes, void **ptr);
int gb2_host_free(void *ptr);
/* half-list pairs (tag_i, tag_j, contact flag, shear history[3]); returns
   the pair count in *n, writes at most cap entries */
int gb2_download_pairs(gb2_ctx *ctx, int cap, int *n, int *tag_i, int *tag_j, int *flag, double *hist);
/* per-atom shear history of primitive-wall fix ifix, [nlocal][3] */
/* compute pair/gran/local with keywords id force torque history
 * (src/compute_pair_gran_local.cpp, via PairGran::compute_pgl
 * src/pair_gran.cpp:676: the pair loop with shearupdate 0 on the current
 * state): one row of 12 doubles per touching pair in list order -- tag_i,
 * tag_j, periodic (1 for a pair through a periodic boundary, kept once, when
 * tag_i > tag_j), force on i[3], torque on i[3], shear history[3].  *nrows is
 * always set; rows are written when cap >= *nrows. */
int gb2_pair_gran_local(gb2_ctx *ctx, int cap, int *nrows, double *rows);
/* compute pair/gran/local with any of its per-pair keywords
 * (src/compute_pair_gran_local.cpp:96-110, columns in the order of add_pair,
 * :445-606): keys is an OR of GB2_PGL_*; *ncols (when not NULL) receives the
 * row width (pos 6, vel 6, id 3, force / force_normal / force_tangential /
 * torque / torque_normal / torque_tangential 3 each, history 3, contactArea 1,
 * delta 1, contactPoint 3).  pos is remapped into the periodic box as
 * Domain::remap does.  GB2_PGL_DEFAULT is the keyword set the reference uses
 * when the command names none.  heatFlux and ms_id need models outside this
 * library and are refused (GB2_ERR_ARG), as are unknown bits and keys == 0. */
#define GB2_PGL_POS               0x0001u
#define GB2_PGL_VEL               0x0002u
#define GB2_PGL_ID                0x0004u
#define GB2_PGL_FORCE             0x0008u
#define GB2_PGL_FORCE_NORMAL      0x0010u
#define GB2_PGL_FORCE_TANGENTIAL  0x0020u
#define GB2_PGL_TORQUE            0x0040u
#define GB2_PGL_TORQUE_NORMAL     0x0080u
#define GB2_PGL_TORQUE_TANGENTIAL 0x0100u
#define GB2_PGL_HISTORY           0x0200u
#define GB2_PGL_CONTACT_AREA      0x0400u
#define GB2_PGL_DELTA             0x0800u
#define GB2_PGL_CONTACT_POINT     0x1000u
#define GB2_PGL_ALL               0x1fffu
#define GB2_PGL_DEFAULT (GB2_PGL_POS | GB2_PGL_VEL | GB2_PGL_ID | GB2_PGL_FORCE | GB2_PGL_TORQUE | \
                         GB2_PGL_HISTORY | GB2_PGL_CONTACT_AREA)
int gb2_pair_gran_local_keys(gb2_ctx *ctx, unsigned keys, int cap, int *nrows, int *ncols, double *rows);
/* fix mesh/surface/stress on mesh wall fix ifix (before setup): the force of
 * every wall contact, negated, is added to its triangle and to the mesh's
 * f_total / torque_total about p_ref each step (MeshModuleStress::
 * add_particle_contribution, src/mesh_module_stress.cpp:276-304; zeroed per
 * step as FixMesh::pre_force / MeshModuleStress::pre_force do).  Sums are
 * device atomics: equal to the reference to rounding, not bit for bit. */
int gb2_add_mesh_stress(gb2_ctx *ctx, int ifix, const double p_ref[3]);
/* the last step's per-triangle force (3 per triangle), normal and shear
 * stress per triangle (MeshModuleStress::calc_total_force) -- cap >= ntri, any
 * of the three may be NULL -- and tot6 = f_total[3], torque_total[3] */
int gb2_download_mesh_stress(gb2_ctx *ctx, int ifix, int cap, double *tri_f, double *sigma_n, double *sigma_t,
                             double *tot6);
/* fix mesh/surface/stress ... wear finnie (MeshModuleStress::
 * add_particle_contribution, src/mesh_module_stress.cpp:306-352, with the
 * element area of TriMesh::calcArea as created): after gb2_add_mesh_stress,
 * before setup.  k_finnie is the peratomtypepair property (ntypes x ntypes,
 * row-major, ntypes * ntypes doubles); the row of the wall's atom type applies.  Device atomics: equal
 * to the reference to rounding.  The download gives the cumulative wear of
 * every element. */
int gb2_add_mesh_wear(gb2_ctx *ctx, int ifix, const double *k_finnie);
int gb2_download_mesh_wear(gb2_ctx *ctx, int ifix, int cap, double *wear);
/* restart of the cumulative wear (MeshModuleStress's restart property "wear",
 * src/mesh_module_stress.cpp:197): n = the mesh's element count, after
 * gb2_add_mesh_wear, before setup */
int gb2_upload_mesh_wear(gb2_ctx *ctx, int ifix, int n, const double *wear);
/* restart interoperability: the contact history in FixContactHistory's
 * per-atom partner layout (src/fix_contact_history.cpp:588-640 pack_restart /
 * unpack_restart): per atom npartner, then per partner its tag and 3 shear
 * values as seen from the atom, concatenated over atoms.  Upload: after
 * gb2_upload_atoms (same atom order), before gb2_setup; the setup's build
 * restores the history of pairs touching there.  Download: the current
 * history (FixContactHistory::pre_exchange from the current list), per owned
 * atom in the current order with its tag; *n atoms, *ntotal partners, and
 * with caps too small only the counts. */
int gb2_upload_history(gb2_ctx *ctx, int n, const int *npartner, const int *partner_tag, const double *hist);
int gb2_download_history(gb2_ctx *ctx, int cap_atoms, int cap_partners, int *n, int *ntotal, int *tag,
                         int *npartner, int *partner_tag, double *hist);
/* primitive-wall shear history of wall fix ifix for the uploaded atoms (3 per
 * atom, upload order), before gb2_setup (FixWallGran restart data) */
int gb2_upload_wall_history(gb2_ctx *ctx, int ifix, int n, const double *hist);
/* compute contact/atom (src/compute_contact_atom.cpp ComputeContactAtom::
 * compute_peratom, skin 0): per owned atom the number of half-list pairs with
 * rsq <= (r_i + r_j)^2, as a double, with its tag; cap < nlocal or contact ==
 * NULL only reports the count in *n.  Positions are those of the last step
 * (or of setup). */
int gb2_contact_atom(gb2_ctx *ctx, int cap, int *n, int *tag, double *contact);
int gb2_download_wall_history(gb2_ctx *ctx, int ifix, int cap, double *hist);
/* occupied mesh-contact slots of mesh fix ifix: (atom tag, triangle id, shear[3]) */
int gb2_download_mesh_contacts(gb2_ctx *ctx, int ifix, int cap, int *n, int *tag, int *tri, double *hist);
/* mesh contact history in the restart layout (FixContactHistoryMesh::
 * write_restart's sort_contacts, src/fix_contact_history_mesh.cpp:375-405
 * and :653-658, then FixContactHistory::pack_restart,
 * src/fix_contact_history.cpp:588-604): per owned atom (current order, with
 * its tag) the partner count; per partner, concatenated over atoms, the
 * triangle id and its 3 shear values.  The slot sort happens in place, as
 * in the reference.  Caps too small: only *n and *ntotal. */
int gb2_download_mesh_history(gb2_ctx *ctx, int ifix, int cap_atoms, int cap_entries, int *n, int *ntotal,
                              int *tag, int *npartner, int *tri, double *hist);
/* FixContactHistoryMesh::unpack_restart (src/fix_contact_history_mesh.cpp:
 * 613-650): after gb2_upload_atoms (same atom order), before gb2_setup */
int gb2_upload_mesh_history(gb2_ctx *ctx, int ifix, int n, const int *npartner, const int *tri,
                            const double *hist);
/* mesh topology after load: per triangle edge/corner active flags and obtuse index */
int gb2_mesh_topology(gb2_ctx *ctx, int ifix, int cap, int *ntri, unsigned char *edge_active,
                      unsigned char *corner_active, int *obtuse);

int gb2_get_stats(gb2_ctx *ctx, gb2_stats *st);
int gb2_census(gb2_ctx *ctx, gb2_contact_census *out);
/* gb2_census_noalloc: the same census for callers that cannot allocate
   device memory -- monitoring hooks inside a host framework whose pool owns
   every device allocation (a foreign cudaMalloc/cudaFree fragments that pool
   or makes the whole device wait), and processes already at their device
   memory cap.  It has no counterpart in the reference (LIGGGHTS allocates
   freely on the host).  Its scratch is a file-scope device array in
   libgranb200 of (GB2_NOALLOC_MAX_BLOCKS + 1) x 8 64-bit counters (1 MiB),
   held by every GPU that loads the library until process exit, so it serves
   at most GB2_NOALLOC_MAX_ATOMS owned atoms; larger contexts get
   GB2_ERR_CAPACITY, an empty context gets zeros.  No cudaMalloc, cudaFree or
   allocating library call is made.  The counts are read back synchronously
   on the context's stream: the call returns once they are on the host.  The
   first call on a device looks up the array's device address
   (cudaGetSymbolAddress); make that first call before any stream capture.
   All calls share the one array: two calls whose work overlaps on a GPU
   (different streams or host threads) race and may return wrong counts. */
#define GB2_NOALLOC_MAX_BLOCKS 16384
#define GB2_NOALLOC_MAX_ATOMS (GB2_NOALLOC_MAX_BLOCKS * 128)
int gb2_census_noalloc(gb2_ctx *ctx, gb2_contact_census *out);
/* per-kernel CUDA-event timing on the context stream (off by default):
 * on = 0 off, 1 every step, N > 1 every N-th step (events between the pair
 * step and its dependent tail kernel serialise the two on the steps timed) */
int gb2_set_profiling(gb2_ctx *ctx, int on);
/* CUDA-event timer on the context stream: start, then stop returns ms */
int gb2_timer_start(gb2_ctx *ctx);
int gb2_timer_stop(gb2_ctx *ctx, double *ms);
/* copies the last error message (NUL-terminated) into buf */
int gb2_last_error(gb2_ctx *ctx, char *buf, int len);
/* library version string, e.g. "granb200 0.1 sm_100a" */
const char *gb2_version(void);

/* ====================================================================
   Superquadric particles: pair_style gran model hertz tangential history
   surface superquadric + fix nve/asphere (integration_scheme 1) on
   atom_style superquadric (one blockiness per particle, n1 = n2), open
   domain, one atom type.  Replaces the run of PairGran::compute with the
   superquadric surface model (src/pair_gran_base.h:187-500,
   src/surface_model_superquadric.h:108-205) and FixNVEAsphereBase
   (src/fix_nve_asphere_base.cpp:319-620) under run_style verlet/b200.
   ==================================================================== */
typedef struct gb2_sq_ctx gb2_sq_ctx;

typedef struct {
    double dt, skin;
    double youngs, poisson, restitution, friction;   /* one atom type */
    int device;
} gb2_sq_params;

/* number of float parameters of the learned initial guess (see gb2_sq_set_learned_guess) */
#define GB2_SQ_MLP_SIZE 9576

int gb2_sq_create(const gb2_sq_params *p, gb2_sq_ctx **out);
int gb2_sq_destroy(gb2_sq_ctx *ctx);
/* per particle: x[3], v[3], quaternion[4] (w,i,j,k), angmom[3], shape[3]
   (half-axes), blockiness, rmass, inertia[3] (principal), volume --
   the AtomVecSuperquadric fields (src/atom_vec_superquadric.cpp) */
int gb2_sq_upload(gb2_sq_ctx *ctx, int n, const double *x, const double *v, const double *quat,
                  const double *angmom, const double *shape, const double *blockiness, const double *rmass,
                  const double *inertia, const double *volume);
/* learned initial guess for pairs without a previous contact point: the
   parameters of an MLP 14 -> 64 -> 64 -> 64 -> 4 (layout in gb2_sq_kernels.cuh);
   NULL switches it off.  No counterpart in the reference: the reference always
   starts those pairs from spheres (calc_contact_point_if_no_previous_point_avaialable,
   src/math_extra_liggghts_superquadric.cpp:1391), which stays the fallback. */
int gb2_sq_set_learned_guess(gb2_sq_ctx *ctx, const float *params, int nparams);
int gb2_sq_setup(gb2_sq_ctx *ctx);
int gb2_sq_run(gb2_sq_ctx *ctx, int nsteps);
/* gb2_sq_run timed with device events (ms) */
int gb2_sq_run_timed(gb2_sq_ctx *ctx, int nsteps, double *ms);
int gb2_sq_download(gb2_sq_ctx *ctx, int cap, double *x, double *v, double *quat, double *angmom,
                    double *omega, double *f, double *torque);
/* half-list pairs: owner and neighbour tags, contact state (0 far, 1 close,
   2 intersecting), contact point of the last solve, shear history */
int gb2_sq_download_pairs(gb2_sq_ctx *ctx, int cap, int *n, int *tag_i, int *tag_j, int *state, double *cp,
                          double *shear);
/* out[7]: Newton iterations, Newton solves, pairs solved, learned guesses
   accepted, learned guesses rejected (homotopy fallback), neighbour builds,
   half-list pairs */
int gb2_sq_counters(gb2_sq_ctx *ctx, long long *out);
int gb2_sq_last_error(gb2_sq_ctx *ctx, char *buf, int len);

/* --------------------------------------------------------------------
   Training of the learned initial guess (no counterpart in the reference).
   Samples are random superquadric pairs near contact (half-axes U(1, 2) mm,
   blockiness U(2, 8), random orientations, oriented boxes intersecting),
   labelled on the device by the plain solver (homotopy from spheres); the
   network is trained on the device by BF16 tensor-core forward/backward
   kernels with FP32 accumulation and Adam.
   -------------------------------------------------------------------- */
typedef struct gb2_mlp_ctx gb2_mlp_ctx;
int gb2_mlp_create(int device, gb2_mlp_ctx **out);
int gb2_mlp_destroy(gb2_mlp_ctx *ctx);
/* n samples from seed; out[3] = valid samples, mean Newton iterations and
   mean solves per sample of the plain solver */
int gb2_mlp_make_data(gb2_mlp_ctx *ctx, long n, unsigned long long seed, double *out);
/* normalisation statistics from the data, He-uniform weights */
int gb2_mlp_init(gb2_mlp_ctx *ctx, unsigned long long seed);
/* loss[2] = first mini-batch, mean of the last epoch */
int gb2_mlp_train(gb2_mlp_ctx *ctx, int epochs, int batch, float lr, float *loss);
int gb2_mlp_get_params(gb2_mlp_ctx *ctx, float *out, int n);
int gb2_mlp_set_params(gb2_mlp_ctx *ctx, const float *in, int n);
/* one forward + backward pass over nrows samples of 22 floats (features
   0..13, targets 14..17): loss and gradient (GB2_SQ_MLP_SIZE floats) */
int gb2_mlp_grad(gb2_mlp_ctx *ctx, int nrows, const float *samples, float *loss, float *grad);
/* learned guess vs plain method on n fresh pairs: stats[9] = pairs, plain
   iterations, plain solves, learned iterations, learned solves, learned
   guesses accepted, plain failures, learned failures, pairs whose two
   solutions differ by more than 1e-4 of the smallest half-axis; *maxdiff =
   largest such difference over the smallest half-axis */
int gb2_mlp_evaluate(gb2_mlp_ctx *ctx, long n, unsigned long long seed, long long *stats, double *maxdiff);
/* device time of the first-contact solve of n fresh pairs (those near
   contact): the plain homotopy from spheres against the learned guess with
   the homotopy as fallback, each launch timed alone with CUDA events after
   an untimed pass; counts[3] = pairs, plain iterations, learned iterations */
int gb2_mlp_time_solves(gb2_mlp_ctx *ctx, long n, unsigned long long seed, double *ms_plain, double *ms_learned,
                        long long *counts);
int gb2_mlp_last_error(gb2_mlp_ctx *ctx, char *buf, int len);

#ifdef __cplusplus
}
#endif
#endif
