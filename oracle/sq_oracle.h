/*
 * sq_oracle.h -- CPU oracle for superquadric particles (test infrastructure only).
 *
 * TEST INFRASTRUCTURE ONLY: a plain-C restatement of the reference's
 * superquadric contact detection and asphere integration (LIGGGHTS-PUBLIC
 * 3.8.0, SUPERQUADRIC_ACTIVE_FLAG), used by tests/, the smoke check and the
 * bench's CPU leg as the checker.  The product never links it.
 *
 * Parity status: tolerance-based.  The shape function uses pow() with
 * non-integer exponents (no bit-parity requirement), so the GPU path is held
 * to the converged contact tolerance (merit < 1e-10) and to relative force
 * tolerances; the oracle itself is unpinned against reference binaries (see
 * gran_oracle.h) and pinned by analytic known-answer tests (spheres and
 * ellipsoids, tests/test_sq_oracle.py).
 *
 * Scope and recorded choices:
 *   - one blockiness per particle (n1 = n2 = n, the reference's
 *     compDouble(n1, n2) branch of the shape function);
 *   - the 4x4 Newton system is solved by Gaussian elimination with partial
 *     pivoting (the reference: explicit cofactor inverse when |det| > 1,
 *     GMRES otherwise -- the same step up to rounding);
 *   - the oriented-box pre-test is the standard 15-axis separating test
 *     (the reference checks the same 15 inequalities, starting from the one
 *     that separated the pair last time, which changes only its speed);
 *   - pair style gran model hertz tangential history surface superquadric
 *     (curvatureLimitFactor 0), fix nve/asphere integration_scheme 1,
 *     open domain (no walls, no periodic images), one atom type.
 */
#ifndef SQ_ORACLE_H
#define SQ_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* one superquadric as the contact solver sees it */
typedef struct {
    double center[3];
    double quat[4];
    double shape[3];        /* half-axes a, b, c */
    double n;               /* blockiness (n1 = n2) */
} orc_sq_particle;

/* contact-point solve: initial-guess modes */
enum { ORC_SQ_GUESS_HOMOTOPY = 0,   /* first contact: spheres -> shape in N stages */
       ORC_SQ_GUESS_POINT = 1 };    /* one solve from a given point */

typedef struct {
    double point[3];        /* converged contact point (global frame) */
    double mu;              /* Lagrange multiplier sqrt(-gA.gB/|gB|^2) */
    double fi, fj;          /* shape functions at the point */
    double gradi[3], gradj[3];
    double merit;           /* max(sin^2(gA, gB), ((fA-fB)/max|f|)^2) */
    int iters;              /* Newton iterations over all stages */
    int solves;             /* calls of the Newton solver */
    int fail;
} orc_sq_solution;

/* MathExtraLiggghtsNonspherical::calc_contact_point and its callers
   (src/math_extra_liggghts_superquadric.cpp:778-1020, :1391-1470) */
void orc_sq_contact_point(const orc_sq_particle *A, const orc_sq_particle *B, int mode,
                          const double guess[3], orc_sq_solution *out);
/* shape function value, gradient and Hessian in the global frame
   (Superquadric::shape_function_props_global src/superquadric.cpp:316) */
void orc_sq_shape_props(const orc_sq_particle *P, const double x[3], double *f, double grad[3], double hess[9]);
/* bounding_sphere_radius_superquadric (src/math_extra_liggghts_superquadric.cpp:206), n1 = n2 = n */
double orc_sq_bounding_radius(const double shape[3], double n);

/* ---- a superquadric DEM run (open domain) ---- */
typedef struct orc_sq orc_sq;
typedef struct {
    double dt, skin;
    double youngs, poisson, restitution, friction;
} orc_sq_params;

/* per atom: x[3], v[3], quat[4], angmom[3], shape[3], blockiness, rmass,
   inertia[3] (principal), volume */
orc_sq *orc_sq_create(const orc_sq_params *p, int n, const double *x, const double *v, const double *quat,
                      const double *angmom, const double *shape, const double *blockiness,
                      const double *rmass, const double *inertia, const double *volume);
void orc_sq_destroy(orc_sq *s);
int orc_sq_setup(orc_sq *s);
int orc_sq_run(orc_sq *s, int nsteps);
void orc_sq_get_atoms(orc_sq *s, double *x, double *v, double *quat, double *angmom, double *omega,
                      double *f, double *torque);
/* pair list with history: returns count (arrays may be NULL) */
int orc_sq_get_pairs(orc_sq *s, int cap, int *tag_i, int *tag_j, int *state, double *cp, double *shear);
/* cumulative Newton iterations and solver calls */
void orc_sq_counters(orc_sq *s, long *iters, long *solves, long *pairs_solved, long *nbuilds);

#ifdef __cplusplus
}
#endif
#endif
