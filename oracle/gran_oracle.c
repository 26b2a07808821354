/*
 * gran_oracle.c -- CPU oracle (TEST INFRASTRUCTURE ONLY, see gran_oracle.h).
 *
 * A single-threaded C restatement of the LIGGGHTS-PUBLIC granular time step.
 * Every function cites the reference file:line it follows; the arithmetic is
 * written in the same operation order so that IEEE results coincide.
 * Parity status: unpinned against reference binaries (the reference needs
 * generated style headers to compile); pinned against analytic cases.
 */
#include "gran_oracle.h"

#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#define BIG 1.0e20
#define SMALL 1.0e-6            /* src/neighbor.cpp:58 */
#define CUT2BIN_RATIO 100
#define SMALL_TRIMESH 1.e-10    /* src/tri_mesh_I.h:48 */
#define LARGE_TRIMESH 1000000   /* src/tri_mesh_I.h:50 */
#define EPSILON_PRECISION 1e-8  /* src/multi_node_mesh.h:59 */
#define NEIGH_MAX 5             /* TriMesh = SurfaceMesh<3,5> */
#define CONTACT_NORMAL_MODEL 1  /* src/contact_model_constants.h:64 */
#define CONTACT_TANGENTIAL_MODEL 4
#define MAXFIX 16
#define NO_OBTUSE_ANGLE -1

/* ------------------------------------------------------------------ */
/* small vector helpers, same operation order as src/vector_liggghts.h  */

static inline double dot3(const double *a, const double *b) { return a[0]*b[0]+a[1]*b[1]+a[2]*b[2]; }
static inline double mag3(const double *v) { return sqrt(v[0]*v[0]+v[1]*v[1]+v[2]*v[2]); }
static inline void sub3(const double *a, const double *b, double *r) { r[0]=a[0]-b[0]; r[1]=a[1]-b[1]; r[2]=a[2]-b[2]; }
static inline void cross3(const double *a, const double *b, double *r)
{ r[0]=a[1]*b[2]-a[2]*b[1]; r[1]=a[2]*b[0]-a[0]*b[2]; r[2]=a[0]*b[1]-a[1]*b[0]; }
static inline void sdiv3(double *v, double s) { const double sinv = 1./s; v[0]=sinv*v[0]; v[1]=sinv*v[1]; v[2]=sinv*v[2]; }
static inline int comp_double(double a, double b, double prec)   /* src/math_extra_liggghts.h:536 */
{
    if (a == b) return 1;
    if (b == 0) return a < prec && a > -prec;
    double x = (a-b);
    return x < prec && x > -prec;
}

/* ------------------------------------------------------------------ */

typedef struct {
    int dim; double pos; int wtype; int rolling;
    int cyl; double cyl_r, cyl_c1, cyl_c2;   /* {x,y,z}cylinder radius and axis position */
    int rebuild;            /* rebuildPrimitiveNeighlist_ */
    int *list; int nlist, caplist;
    double *hist;           /* property/atom history, 3 per atom */
} wall_plane;

typedef struct {
    int ntri;
    double (*node)[3][3];
    double (*center)[3];
    double *rbound;
    double (*edgevec)[3][3];
    double (*edgelen)[3];
    double (*edgenorm)[3][3];
    double (*surfnorm)[3];
    int *obtuse;
    unsigned char (*edge_active)[3];
    unsigned char (*corner_active)[3];
    int *nneigh; int (*neighfaces)[NEIGH_MAX];
    double curvature, precision;
    int wtype, rolling;
    /* FixNeighlistMesh */
    int **tri_list; int *tri_n; int *tri_cap;
    int **tri_bins; int *tri_nbins;
    double nl_skin, nl_distmax;
    long last_bin_update;
    int build_neighlist_nl;   /* FixNeighlistMesh::buildNeighList */
    /* FixContactHistoryMesh, per atom */
    int build_neighlist_ch;   /* FixContactHistoryMesh::build_neighlist_ */
    int *nneighs; int *npartner; int **partner; double **chist;
    unsigned char **keep; unsigned char **isect;
    /* fix move/mesh rotate (MeshMoverRotate) and FixMesh rebuild trigger */
    int moving;            /* 0 static, 1 rotate, 2 linear */
    double mv_point[3], mv_axis[3], mv_omega;
    double mv_vel[3];
    double (*vnode)[3][3];       /* element property "v" */
    double (*node_last)[3][3];   /* nodesLastRe_ */
    long next_reneighbor;        /* FixMesh::next_reneighbor */
    /* mesh/surface/stress (MeshModuleStress): per-element force, totals */
    int stress; double p_ref[3]; double (*tri_f)[3]; double f_total[3], torque_total[3];
    double (*area_ev)[2][3]; double (*area_el)[2];   /* edge vectors and lengths as created (calcArea) */
    double *wear, *kfin;   /* Finnie wear per element; k_finnie of the wall type against each atom type */
} wall_mesh;

typedef struct { int kind; double xacc, yacc, zacc; wall_plane *wp; wall_mesh *wm; int imesh; } fixrec;

struct orc_sim {
    orc_params p;
    int ntypes;
    double **Yeff, **Geff, **betaeff, **mu, **mur;
    /* atoms */
    int nlocal, nghost, nmax;
    double *x, *v, *omega, *f, *torque, *radius, *rmass;
    int *type, *tag;
    /* ghosts: source index and swap shift */
    int *gsrc; double *gshift;   /* per ghost: 3 shifts */
    int nswap; int swapfirst[8], swapnum[8];
    /* domain */
    double boxlo[3], boxhi[3], prd[3];
    /* neighbor */
    double cutneighmax, cutneighmaxsq, triggersq, cutghost;
    double *maxrad;
    double bboxlo[3], bboxhi[3];
    int nbinx, nbiny, nbinz, mbinx, mbiny, mbinz, mbinxlo, mbinylo, mbinzlo, mbins;
    double binsizex, binsizey, binsizez, bininvx, bininvy, bininvz;
    int *binhead, *bins; int nstencil; int *stencil;
    int ago; long ntimestep; int nbuilds;
    double *xhold;
    /* half list */
    int *nstart, *nnum; int *nbr, *flag; double *hist; int npairs, cappairs;
    /* FixContactHistory partner arrays */
    int *npartner; int **partner; double **phist; int computeflag;
    /* sort */
    long nextsort; int snbinx, snbiny, snbinz; double sbboxlo[3], sbininvx, sbininvy, sbininvz;
    /* fixes */
    int nfix; fixrec fix[MAXFIX]; int has_nve;
    struct ins_state *ins;   /* fix insert/pack, at most one */
    int setupflag;
    char err[256];
};

struct ins_state;
static void ins_max_rad(const struct ins_state *I, int type, double *mx);
static long ins_next(const struct ins_state *I);

static void fail(orc_sim *s, const char *fmt, ...)
{
    va_list ap; va_start(ap, fmt); vsnprintf(s->err, sizeof s->err, fmt, ap); va_end(ap);
}

static void *xrealloc(void *p, size_t n) { void *q = realloc(p, n ? n : 1); if (!q) { fprintf(stderr, "oracle: out of memory\n"); abort(); } return q; }
static double **matrix(int n) { double **m = malloc(sizeof(double*)*n); double *d = calloc((size_t)n*n, sizeof(double)); for (int i = 0; i < n; i++) m[i] = d + (size_t)i*n; return m; }
static void free_matrix(double **m) { if (m) { free(m[0]); free(m); } }

/* ------------------------------------------------------------------ */
/* material matrices: src/global_properties.cpp:411-560                */

static void setup_materials(orc_sim *s)
{
    const int nt = s->ntypes;
    s->Yeff = matrix(nt+1); s->Geff = matrix(nt+1); s->betaeff = matrix(nt+1);
    s->mu = matrix(nt+1); s->mur = matrix(nt+1);
    const orc_params *p = &s->p;
    for (int i = 1; i <= nt; i++)
        for (int j = 1; j <= nt; j++) {
            const double Yi = p->youngs[i-1], Yj = p->youngs[j-1];
            const double vi = p->poisson[i-1], vj = p->poisson[j-1];
            s->Yeff[i][j] = 1./((1.-pow(vi,2.))/Yi+(1.-pow(vj,2.))/Yj);          /* :432 */
            s->Geff[i][j] = 1./(2.*(2.-vi)*(1.+vi)/Yi+2.*(2.-vj)*(1.+vj)/Yj);   /* :461 */
            const double lg = log(p->restitution[(i-1)*nt+(j-1)]);              /* :508 */
            s->betaeff[i][j] = lg / sqrt(pow(lg,2.)+pow(M_PI,2.));               /* :540 */
            s->mu[i][j] = p->friction[(i-1)*nt+(j-1)];
            s->mur[i][j] = p->rollfriction ? p->rollfriction[(i-1)*nt+(j-1)] : 0.0;
        }
}

/* ------------------------------------------------------------------ */
/* the contact-model chain surface->normal->tangential->rolling
   src/contact_models.h:228-238, for sphere pairs and walls             */

typedef struct {
    int is_wall;
    double radi, radj, radsum, r, rinv, rsq, deltan;
    double delta[3], en[3];
    const double *v_i, *v_j, *omega_i, *omega_j;
    double meff, mi, mj;
    int itype, jtype;
    int *contact_flags; double *contact_history;
    int computeflag, shearupdate;
    /* filled by the models */
    double vn, wr1, wr2, wr3, vtr1, vtr2, vtr3, cri, crj, Fn, kn, kt, gamman, gammat;
} sidata_t;

typedef struct { double F[3], T[3]; } force_t;

/* src/surface_model_default.h:150-204 */
static void surface_default(sidata_t *sd)
{
    const double enx = sd->en[0], eny = sd->en[1], enz = sd->en[2];
    const double vr1 = sd->v_i[0] - sd->v_j[0];
    const double vr2 = sd->v_i[1] - sd->v_j[1];
    const double vr3 = sd->v_i[2] - sd->v_j[2];
    const double vn = vr1 * enx + vr2 * eny + vr3 * enz;
    const double vn1 = vn * enx, vn2 = vn * eny, vn3 = vn * enz;
    const double vt1 = vr1 - vn1, vt2 = vr2 - vn2, vt3 = vr3 - vn3;
    const double deltan = sd->radsum - sd->r;
    const double dx = sd->delta[0], dy = sd->delta[1], dz = sd->delta[2];
    const double rinv = sd->rinv;
    double wr1, wr2, wr3;
    if (sd->is_wall) {
        const double cr = sd->radi - 0.5*sd->deltan;
        wr1 = cr * sd->omega_i[0] * rinv;
        wr2 = cr * sd->omega_i[1] * rinv;
        wr3 = cr * sd->omega_i[2] * rinv;
        sd->cri = cr;
    } else {
        const double cri = sd->radi - 0.5 * deltan;
        const double crj = sd->radj - 0.5 * deltan;
        wr1 = (cri * sd->omega_i[0] + crj * sd->omega_j[0]) * rinv;
        wr2 = (cri * sd->omega_i[1] + crj * sd->omega_j[1]) * rinv;
        wr3 = (cri * sd->omega_i[2] + crj * sd->omega_j[2]) * rinv;
        sd->cri = cri; sd->crj = crj;
    }
    sd->vtr1 = vt1 - (dz * wr2 - dy * wr3);
    sd->vtr2 = vt2 - (dx * wr3 - dz * wr1);
    sd->vtr3 = vt3 - (dy * wr1 - dx * wr2);
    sd->vn = vn; sd->deltan = deltan;
    sd->wr1 = wr1; sd->wr2 = wr2; sd->wr3 = wr3;
}

/* src/normal_model_hertz.h:202-393 (energy/heating/bond options off) */
static void normal_hertz(orc_sim *s, sidata_t *sd, force_t *fi, force_t *fj)
{
    if (sd->contact_flags) *sd->contact_flags |= CONTACT_NORMAL_MODEL;
    const int it = sd->itype, jt = sd->jtype;
    const double radi = sd->radi, radj = sd->radj;
    const double reff = sd->is_wall ? radi : (radi*radj/(radi+radj));
    const double meff = sd->meff;
    const double sqrtval = sqrt(reff*sd->deltan);
    const double deltan = sd->deltan;
    const double Sn = 2.*s->Yeff[it][jt]*sqrtval;
    const double St = 8.*s->Geff[it][jt]*sqrtval;
    double kn = 4./3.*s->Yeff[it][jt]*sqrtval;
    double kt = St;
    const double sqrtFiveOverSix = 0.91287092917527685576161630466800355658790782499663875;
    const double gamman = -2.*sqrtFiveOverSix*s->betaeff[it][jt]*sqrt(Sn*meff);
    const double gammat = s->p.tangential_damping ? -2.*sqrtFiveOverSix*s->betaeff[it][jt]*sqrt(St*meff) : 0.0;
    kn /= 1.0;  /* force->nktv2p = 1 in si */
    kt /= 1.0;
    const double Fn_damping = -gamman*sd->vn;
    const double Fn_contact = kn*deltan;
    const double Fn = Fn_damping + Fn_contact;
    sd->Fn = Fn; sd->kn = kn; sd->kt = kt; sd->gamman = gamman; sd->gammat = gammat;
    if (sd->is_wall) {
        const double Fn_ = Fn * 1.0;   /* area_ratio */
        fi->F[0] += Fn_ * sd->en[0];
        fi->F[1] += Fn_ * sd->en[1];
        fi->F[2] += Fn_ * sd->en[2];
    } else {
        fi->F[0] += sd->Fn * sd->en[0];
        fi->F[1] += sd->Fn * sd->en[1];
        fi->F[2] += sd->Fn * sd->en[2];
        fj->F[0] += -fi->F[0];
        fj->F[1] += -fi->F[1];
        fj->F[2] += -fi->F[2];
    }
}

/* src/tangential_model_history.h:130-339 */
static void tangential_history(orc_sim *s, sidata_t *sd, force_t *fi, force_t *fj)
{
    const double enx = sd->en[0], eny = sd->en[1], enz = sd->en[2];
    if (sd->contact_flags) *sd->contact_flags |= CONTACT_TANGENTIAL_MODEL;
    double *const shear = sd->contact_history;
    const int update_history = sd->computeflag && sd->shearupdate;
    if (update_history) {
        const double dt = s->p.dt;
        shear[0] += sd->vtr1 * dt;
        shear[1] += sd->vtr2 * dt;
        shear[2] += sd->vtr3 * dt;
        double rsht = shear[0]*enx + shear[1]*eny + shear[2]*enz;
        shear[0] -= rsht * enx;
        shear[1] -= rsht * eny;
        shear[2] -= rsht * enz;
    }
    const double shrmag = sqrt(shear[0]*shear[0] + shear[1]*shear[1] + shear[2]*shear[2]);
    const double kt = sd->kt;
    const double xmu = s->mu[sd->itype][sd->jtype];
    double Ft1 = -(kt * shear[0]);
    double Ft2 = -(kt * shear[1]);
    double Ft3 = -(kt * shear[2]);
    const double Ft_shear = kt * shrmag;
    const double Ft_friction = xmu * fabs(sd->Fn);
    if (Ft_shear > Ft_friction) {
        if (shrmag != 0.0) {
            const double ratio = Ft_friction / Ft_shear;
            Ft1 *= ratio; Ft2 *= ratio; Ft3 *= ratio;
            if (update_history) {
                shear[0] = -Ft1/kt;
                shear[1] = -Ft2/kt;
                shear[2] = -Ft3/kt;
            }
        } else Ft1 = Ft2 = Ft3 = 0.0;
    } else {
        const double gammat = sd->gammat;
        Ft1 -= (gammat*sd->vtr1);
        Ft2 -= (gammat*sd->vtr2);
        Ft3 -= (gammat*sd->vtr3);
    }
    const double tor1 = eny * Ft3 - enz * Ft2;
    const double tor2 = enz * Ft1 - enx * Ft3;
    const double tor3 = enx * Ft2 - eny * Ft1;
    double torque_i[3], torque_j[3] = {0, 0, 0};
    torque_i[0] = -sd->cri * tor1;
    torque_i[1] = -sd->cri * tor2;
    torque_i[2] = -sd->cri * tor3;
    if (!sd->is_wall) {
        torque_j[0] = -sd->crj * tor1;
        torque_j[1] = -sd->crj * tor2;
        torque_j[2] = -sd->crj * tor3;
    }
    if (sd->is_wall) {
        const double area_ratio = 1.0;
        fi->F[0] += Ft1 * area_ratio; fi->F[1] += Ft2 * area_ratio; fi->F[2] += Ft3 * area_ratio;
        fi->T[0] += torque_i[0] * area_ratio; fi->T[1] += torque_i[1] * area_ratio; fi->T[2] += torque_i[2] * area_ratio;
    } else {
        fi->F[0] += Ft1; fi->F[1] += Ft2; fi->F[2] += Ft3;
        fj->F[0] += -Ft1; fj->F[1] += -Ft2; fj->F[2] += -Ft3;
        fi->T[0] += torque_i[0]; fi->T[1] += torque_i[1]; fi->T[2] += torque_i[2];
        fj->T[0] += torque_j[0]; fj->T[1] += torque_j[1]; fj->T[2] += torque_j[2];
    }
}

/* src/rolling_model_cdt.h:89-159 (torsionTorque off) */
static void rolling_cdt(orc_sim *s, sidata_t *sd, force_t *fi, force_t *fj)
{
    const double rmu = s->mur[sd->itype][sd->jtype];
    double r_torque[3] = {0., 0., 0.}, wr_roll[3];
    const double radi = sd->radi, radj = sd->radj;
    const double reff = sd->is_wall ? radi : (radi*radj/(radi+radj));
    if (sd->is_wall) {
        const double wr1 = sd->wr1, wr2 = sd->wr2, wr3 = sd->wr3;
        const double wrmag = sqrt(wr1*wr1+wr2*wr2+wr3*wr3);
        if (wrmag > 0.) {
            const double kn = sd->kn;
            const double enx = sd->en[0], eny = sd->en[1], enz = sd->en[2];
            const double Fn = sd->deltan*kn;
            r_torque[0] = rmu*Fn*wr1/wrmag*reff;
            r_torque[1] = rmu*Fn*wr2/wrmag*reff;
            r_torque[2] = rmu*Fn*wr3/wrmag*reff;
            double d = r_torque[0]*enx+ r_torque[1]*eny + r_torque[2]*enz;
            double rn[3] = {enx * d, eny * d, enz * d};
            r_torque[0] = r_torque[0]-rn[0]; r_torque[1] = r_torque[1]-rn[1]; r_torque[2] = r_torque[2]-rn[2];
        }
    } else {
        sub3(sd->omega_i, sd->omega_j, wr_roll);
        const double wr_rollmag = mag3(wr_roll);
        if (wr_rollmag > 0.) {
            const double enx = sd->en[0], eny = sd->en[1], enz = sd->en[2];
            const double sc = rmu*sd->kn*sd->deltan*reff/wr_rollmag;
            r_torque[0] = sc*wr_roll[0]; r_torque[1] = sc*wr_roll[1]; r_torque[2] = sc*wr_roll[2];
            const double d = r_torque[0]*enx + r_torque[1]*eny + r_torque[2]*enz;
            double rn[3] = {enx * d, eny * d, enz * d};
            r_torque[0] = r_torque[0]-rn[0]; r_torque[1] = r_torque[1]-rn[1]; r_torque[2] = r_torque[2]-rn[2];
        }
    }
    fi->T[0] -= r_torque[0]; fi->T[1] -= r_torque[1]; fi->T[2] -= r_torque[2];
    fj->T[0] += r_torque[0]; fj->T[1] += r_torque[1]; fj->T[2] += r_torque[2];
}

static void contact_chain(orc_sim *s, sidata_t *sd, force_t *fi, force_t *fj, int rolling)
{
    surface_default(sd);
    normal_hertz(s, sd, fi, fj);
    tangential_history(s, sd, fi, fj);
    if (rolling) rolling_cdt(s, sd, fi, fj);
}

/* ------------------------------------------------------------------ */
/* atoms                                                                */

static void grow_atoms(orc_sim *s, int nmax)
{
    if (nmax <= s->nmax) return;
    int old = s->nmax;
    s->nmax = nmax;
    s->x = xrealloc(s->x, sizeof(double)*3*nmax);
    s->v = xrealloc(s->v, sizeof(double)*3*nmax);
    s->omega = xrealloc(s->omega, sizeof(double)*3*nmax);
    s->f = xrealloc(s->f, sizeof(double)*3*nmax);
    s->torque = xrealloc(s->torque, sizeof(double)*3*nmax);
    s->radius = xrealloc(s->radius, sizeof(double)*nmax);
    s->rmass = xrealloc(s->rmass, sizeof(double)*nmax);
    s->type = xrealloc(s->type, sizeof(int)*nmax);
    s->tag = xrealloc(s->tag, sizeof(int)*nmax);
    s->bins = xrealloc(s->bins, sizeof(int)*nmax);
    (void)old;
}

/* grow every per-atom array (atoms and per-atom fix data) to nmax */
static void grow_all(orc_sim *s, int nmax)
{
    int old = s->nmax;
    if (nmax <= old) return;
    grow_atoms(s, nmax);
    s->npartner = xrealloc(s->npartner, sizeof(int)*s->nmax);
    s->partner = xrealloc(s->partner, sizeof(int*)*s->nmax);
    s->phist = xrealloc(s->phist, sizeof(double*)*s->nmax);
    s->xhold = xrealloc(s->xhold, sizeof(double)*3*s->nmax);
    for (int i = old; i < s->nmax; i++) { s->npartner[i] = 0; s->partner[i] = NULL; s->phist[i] = NULL; }
    for (int k = 0; k < s->nfix; k++) {
        if (s->fix[k].wp) { s->fix[k].wp->hist = xrealloc(s->fix[k].wp->hist, sizeof(double)*3*s->nmax); memset(s->fix[k].wp->hist + 3*old, 0, sizeof(double)*3*(s->nmax-old)); }
        if (s->fix[k].wm) {
            wall_mesh *m = s->fix[k].wm;
            m->nneighs = xrealloc(m->nneighs, sizeof(int)*s->nmax);
            m->npartner = xrealloc(m->npartner, sizeof(int)*s->nmax);
            m->partner = xrealloc(m->partner, sizeof(int*)*s->nmax);
            m->chist = xrealloc(m->chist, sizeof(double*)*s->nmax);
            m->keep = xrealloc(m->keep, sizeof(unsigned char*)*s->nmax);
            m->isect = xrealloc(m->isect, sizeof(unsigned char*)*s->nmax);
            for (int i = old; i < s->nmax; i++) { m->nneighs[i] = 0; m->npartner[i] = 0; m->partner[i] = NULL; m->chist[i] = NULL; m->keep[i] = NULL; m->isect[i] = NULL; }
        }
    }
}

orc_sim *orc_create(const orc_params *p, int n, const double *x, const double *v, const double *omega,
                    const double *radius, const double *rmass, const int *type, const int *tag)
{
    orc_sim *s = calloc(1, sizeof(orc_sim));
    s->p = *p;
    s->ntypes = p->ntypes;
    setup_materials(s);
    grow_atoms(s, n > 16 ? 2*n : 32);
    s->nlocal = n;
    memcpy(s->x, x, sizeof(double)*3*n);
    memcpy(s->v, v, sizeof(double)*3*n);
    memcpy(s->omega, omega, sizeof(double)*3*n);
    memcpy(s->radius, radius, sizeof(double)*n);
    memcpy(s->rmass, rmass, sizeof(double)*n);
    memcpy(s->type, type, sizeof(int)*n);
    memcpy(s->tag, tag, sizeof(int)*n);
    memset(s->f, 0, sizeof(double)*3*n);
    memset(s->torque, 0, sizeof(double)*3*n);
    for (int d = 0; d < 3; d++) { s->boxlo[d] = p->boxlo[d]; s->boxhi[d] = p->boxhi[d]; s->prd[d] = p->boxhi[d]-p->boxlo[d]; }
    s->npartner = calloc(s->nmax, sizeof(int));
    s->partner = calloc(s->nmax, sizeof(int*));
    s->phist = calloc(s->nmax, sizeof(double*));
    s->xhold = calloc((size_t)3*s->nmax, sizeof(double));
    return s;
}

void orc_destroy(orc_sim *s)
{
    if (!s) return;
    free(s->x); free(s->v); free(s->omega); free(s->f); free(s->torque); free(s->radius); free(s->rmass);
    free(s->type); free(s->tag); free(s->bins); free(s->binhead); free(s->stencil); free(s->xhold);
    free(s->gsrc); free(s->gshift); free(s->maxrad); free(s->ins);
    free(s->nstart); free(s->nnum); free(s->nbr); free(s->flag); free(s->hist);
    for (int i = 0; i < s->nmax; i++) { if (s->partner) free(s->partner[i]); if (s->phist) free(s->phist[i]); }
    free(s->npartner); free(s->partner); free(s->phist);
    for (int k = 0; k < s->nfix; k++) {
        if (s->fix[k].wp) { free(s->fix[k].wp->list); free(s->fix[k].wp->hist); free(s->fix[k].wp); }
        if (s->fix[k].wm) {
            wall_mesh *m = s->fix[k].wm;
            for (int t = 0; t < m->ntri; t++) { if (m->tri_list) free(m->tri_list[t]); if (m->tri_bins) free(m->tri_bins[t]); }
            free(m->tri_list); free(m->tri_n); free(m->tri_cap); free(m->tri_bins); free(m->tri_nbins);
            for (int i = 0; i < s->nmax; i++) {
                if (m->partner) free(m->partner[i]);
                if (m->chist) free(m->chist[i]);
                if (m->keep) free(m->keep[i]);
                if (m->isect) free(m->isect[i]);
            }
            free(m->nneighs); free(m->npartner); free(m->partner); free(m->chist); free(m->keep); free(m->isect);
            free(m->node); free(m->center); free(m->rbound); free(m->edgevec); free(m->edgelen); free(m->edgenorm);
            free(m->surfnorm); free(m->obtuse); free(m->edge_active); free(m->corner_active); free(m->nneigh); free(m->neighfaces);
            free(m->vnode); free(m->node_last); free(m->tri_f); free(m->area_ev); free(m->area_el);
            if (s->fix[k].kind == ORC_FIX_WALL_MESH) free(m);
        }
    }
    free_matrix(s->Yeff); free_matrix(s->Geff); free_matrix(s->betaeff); free_matrix(s->mu); free_matrix(s->mur);
    free(s);
}

const char *orc_error(orc_sim *s) { return s->err; }
int orc_nlocal(orc_sim *s) { return s->nlocal; }
int orc_nghost(orc_sim *s) { return s->nghost; }
long orc_ntimestep(orc_sim *s) { return s->ntimestep; }
int orc_nbuilds(orc_sim *s) { return s->nbuilds; }

/* ------------------------------------------------------------------ */
/* fixes                                                                */

int orc_add_gravity(orc_sim *s, double mag, double dx, double dy, double dz)
{
    /* src/fix_gravity.cpp:376-397 (style vector, 3d) */
    fixrec *fr = &s->fix[s->nfix++];
    fr->kind = ORC_FIX_GRAVITY;
    double length = sqrt(dx*dx + dy*dy + dz*dz);
    double xg = dx/length, yg = dy/length, zg = dz/length;
    fr->xacc = mag*xg; fr->yacc = mag*yg; fr->zacc = mag*zg;
    return s->nfix-1;
}

int orc_add_wall_plane(orc_sim *s, int dim, double pos, int wall_type, int rolling_cdt)
{
    fixrec *fr = &s->fix[s->nfix++];
    fr->kind = ORC_FIX_WALL_PLANE;
    wall_plane *w = calloc(1, sizeof(wall_plane));
    w->dim = dim; w->pos = pos; w->wtype = wall_type; w->rolling = rolling_cdt;
    w->hist = calloc((size_t)3*s->nmax, sizeof(double));
    fr->wp = w;
    return s->nfix-1;
}

/* fix wall/gran ... primitive type <wtype> {x,y,z}cylinder <radius> <c1> <c2> */
int orc_add_wall_cylinder(orc_sim *s, int dim, double radius, double c1, double c2, int wall_type, int rolling_cdt)
{
    int k = orc_add_wall_plane(s, dim, 0.0, wall_type, rolling_cdt);
    wall_plane *w = s->fix[k].wp;
    w->cyl = 1; w->cyl_r = radius; w->cyl_c1 = c1; w->cyl_c2 = c2;
    return k;
}

/* forward decl */
static void mesh_build_topology(orc_sim *s, wall_mesh *m);

int orc_add_wall_mesh(orc_sim *s, int ntri, const double *nodes, int wall_type, double curvature, int rolling_cdt)
{
    fixrec *fr = &s->fix[s->nfix++];
    fr->kind = ORC_FIX_WALL_MESH;
    wall_mesh *m = calloc(1, sizeof(wall_mesh));
    m->wtype = wall_type; m->rolling = rolling_cdt;
    m->curvature = curvature > 0 ? curvature : 1.-0.00001;   /* src/surface_mesh_I.h:58 */
    m->precision = EPSILON_PRECISION;
    m->node = malloc(sizeof(double)*9*(ntri > 0 ? ntri : 1));
    m->center = malloc(sizeof(double)*3*(ntri > 0 ? ntri : 1));
    m->rbound = malloc(sizeof(double)*(ntri > 0 ? ntri : 1));
    /* MultiNodeMesh::addElement src/multi_node_mesh_I.h:139-190 */
    int n = 0;
    for (int t = 0; t < ntri; t++) {
        double nd[3][3];
        memcpy(nd, nodes + 9*t, sizeof nd);
        int eq = 0;
        for (int a = 0; a < 3 && !eq; a++)
            for (int b = a+1; b < 3 && !eq; b++) {
                int all = 1;
                for (int c = 0; c < 3; c++) if (!comp_double(nd[a][c], nd[b][c], m->precision)) all = 0;
                if (all) eq = 1;
            }
        if (eq) continue;
        memcpy(m->node[n], nd, sizeof nd);
        double avg[3] = {0., 0., 0.};
        for (int i = 0; i < 3; i++) { avg[0] = nd[i][0]+avg[0]; avg[1] = nd[i][1]+avg[1]; avg[2] = nd[i][2]+avg[2]; }
        sdiv3(avg, 3.0);
        memcpy(m->center[n], avg, sizeof avg);
        double rb = 0.;
        for (int i = 0; i < 3; i++) { double vec[3]; sub3(m->center[n], nd[i], vec); double mg = mag3(vec); rb = rb > mg ? rb : mg; }
        m->rbound[n] = rb;
        n++;
    }
    m->ntri = n;
    mesh_build_topology(s, m);
    m->tri_list = calloc(n > 0 ? n : 1, sizeof(int*));
    m->tri_n = calloc(n > 0 ? n : 1, sizeof(int));
    m->tri_cap = calloc(n > 0 ? n : 1, sizeof(int));
    m->tri_bins = calloc(n > 0 ? n : 1, sizeof(int*));
    m->tri_nbins = calloc(n > 0 ? n : 1, sizeof(int));
    m->last_bin_update = -1;
    m->nl_skin = -1; m->nl_distmax = -1;
    m->nneighs = calloc(s->nmax, sizeof(int));
    m->npartner = calloc(s->nmax, sizeof(int));
    m->partner = calloc(s->nmax, sizeof(int*));
    m->chist = calloc(s->nmax, sizeof(double*));
    m->keep = calloc(s->nmax, sizeof(unsigned char*));
    m->isect = calloc(s->nmax, sizeof(unsigned char*));
    fr->wm = m;
    return s->nfix-1;
}

/* fix move/mesh ... rotate origin <p> axis <a> period <T>
   (MeshMoverRotate constructor src/mesh_mover_rotation.cpp:66-96,
   FixMoveMesh::setup src/fix_move_mesh.cpp:195-216: node velocities 0) */
int orc_add_move_mesh_rotate(orc_sim *s, int ifix_mesh, double ox, double oy, double oz,
                             double ax, double ay, double az, double period)
{
    if (ifix_mesh < 0 || ifix_mesh >= s->nfix || s->fix[ifix_mesh].kind != ORC_FIX_WALL_MESH) return -1;
    if (!(period != 0.0)) return -1;
    wall_mesh *m = s->fix[ifix_mesh].wm;
    if (m->moving) return -1;   /* one mover per mesh */
    fixrec *fr = &s->fix[s->nfix++];
    fr->kind = ORC_FIX_MOVE_MESH;
    fr->imesh = ifix_mesh;
    m->moving = 1;
    m->mv_point[0] = ox; m->mv_point[1] = oy; m->mv_point[2] = oz;
    m->mv_axis[0] = ax; m->mv_axis[1] = ay; m->mv_axis[2] = az;
    {   /* vectorNormalize3D src/vector_liggghts.h:62 */
        double *v = m->mv_axis;
        const double norm = sqrt(v[0]*v[0]+v[1]*v[1]+v[2]*v[2]);
        const double invnorm = (norm == 0.) ? 0. : 1./norm;
        v[0] *= invnorm; v[1] *= invnorm; v[2] *= invnorm;
    }
    m->mv_omega = 2.*M_PI/period;
    int nt = m->ntri > 0 ? m->ntri : 1;
    m->vnode = calloc((size_t)nt, sizeof(double)*9);
    m->node_last = calloc((size_t)nt, sizeof(double)*9);
    m->next_reneighbor = -1;
    return s->nfix-1;
}

int orc_get_mesh_nodes(orc_sim *s, int ifix, double *nodes, double *vnode)
{
    if (ifix < 0 || ifix >= s->nfix || !s->fix[ifix].wm) return -1;
    wall_mesh *m = s->fix[ifix].wm;
    if (nodes) memcpy(nodes, m->node, sizeof(double)*9*m->ntri);
    if (vnode) {
        if (m->vnode) memcpy(vnode, m->vnode, sizeof(double)*9*m->ntri);
        else memset(vnode, 0, sizeof(double)*9*m->ntri);
    }
    return m->ntri;
}

/* per element: centre 3, bounding radius, unit edge vectors 9, edge lengths 3,
   edge normals 9, surface normal 3, precision -- the layout of the reference
   harness's element geometry record */
int orc_get_mesh_geom(orc_sim *s, int ifix, double *geom)
{
    if (ifix < 0 || ifix >= s->nfix || !s->fix[ifix].wm) return -1;
    wall_mesh *m = s->fix[ifix].wm;
    for (int t = 0; t < m->ntri && geom; t++) {
        double *g = &geom[29*(size_t)t];
        for (int c = 0; c < 3; c++) g[c] = m->center[t][c];
        g[3] = m->rbound[t];
        for (int a = 0; a < 3; a++)
            for (int c = 0; c < 3; c++) { g[4+3*a+c] = m->edgevec[t][a][c]; g[16+3*a+c] = m->edgenorm[t][a][c]; }
        for (int a = 0; a < 3; a++) g[13+a] = m->edgelen[t][a];
        for (int c = 0; c < 3; c++) g[25+c] = m->surfnorm[t][c];
        g[28] = m->precision;
    }
    return m->ntri;
}

/* fix move/mesh ... linear vx vy vz (MeshMoverLinear constructor
   src/mesh_mover_linear.cpp:66-77) */
int orc_add_move_mesh_linear(orc_sim *s, int ifix_mesh, double vx, double vy, double vz)
{
    if (ifix_mesh < 0 || ifix_mesh >= s->nfix || s->fix[ifix_mesh].kind != ORC_FIX_WALL_MESH) return -1;
    wall_mesh *m = s->fix[ifix_mesh].wm;
    if (m->moving) return -1;
    fixrec *fr = &s->fix[s->nfix++];
    fr->kind = ORC_FIX_MOVE_MESH;
    fr->imesh = ifix_mesh;
    m->moving = 2;
    m->mv_vel[0] = vx; m->mv_vel[1] = vy; m->mv_vel[2] = vz;
    int nt = m->ntri > 0 ? m->ntri : 1;
    m->vnode = calloc((size_t)nt, sizeof(double)*9);
    m->node_last = calloc((size_t)nt, sizeof(double)*9);
    m->next_reneighbor = -1;
    return s->nfix-1;
}

/* MeshMoverLinear::initial_integrate src/mesh_mover_linear.cpp:94-112 with
   MultiNodeMesh::move src/multi_node_mesh_I.h:502-513: nodes and centres
   shifted by v dt (no translation-variant element property on a surface
   mesh), node velocities 0 + v */
static void move_mesh_linear(orc_sim *s, wall_mesh *m)
{
    double dx[3] = {m->mv_vel[0]*s->p.dt, m->mv_vel[1]*s->p.dt, m->mv_vel[2]*s->p.dt};
    for (int t = 0; t < m->ntri; t++) {
        for (int j = 0; j < 3; j++)
            for (int c = 0; c < 3; c++) m->node[t][j][c] = m->node[t][j][c] + dx[c];
        for (int c = 0; c < 3; c++) m->center[t][c] = m->center[t][c] + dx[c];
    }
    for (int t = 0; t < m->ntri; t++)
        for (int j = 0; j < 3; j++)
            for (int c = 0; c < 3; c++) m->vnode[t][j][c] = 0. + m->mv_vel[c];
}

/* MathExtraLiggghts::vec_quat_rotate src/math_extra_liggghts.h:451-468 with
   MathExtra::quatquat src/math_extra.h:596 and qconjugate :560 */
static void vec_quat_rotate(double *vec, const double *q)
{
    double vq[4] = {0., vec[0], vec[1], vec[2]};
    double qc[4] = {q[0], -q[1], -q[2], -q[3]};
    double t[4], r[4];
    t[0] = q[0]*vq[0] - q[1]*vq[1] - q[2]*vq[2] - q[3]*vq[3];
    t[1] = q[0]*vq[1] + vq[0]*q[1] + q[2]*vq[3] - q[3]*vq[2];
    t[2] = q[0]*vq[2] + vq[0]*q[2] + q[3]*vq[1] - q[1]*vq[3];
    t[3] = q[0]*vq[3] + vq[0]*q[3] + q[1]*vq[2] - q[2]*vq[1];
    r[0] = t[0]*qc[0] - t[1]*qc[1] - t[2]*qc[2] - t[3]*qc[3];
    r[1] = t[0]*qc[1] + qc[0]*t[1] + t[2]*qc[3] - t[3]*qc[2];
    r[2] = t[0]*qc[2] + qc[0]*t[2] + t[3]*qc[1] - t[1]*qc[3];
    r[3] = t[0]*qc[3] + qc[0]*t[3] + t[1]*qc[2] - t[2]*qc[1];
    vec[0] = r[1]; vec[1] = r[2]; vec[2] = r[3];
}

/* MeshMoverRotate::initial_integrate src/mesh_mover_rotation.cpp:110-138:
   FixMoveMesh::initial_integrate zeroes "v" (first mover), FixMesh::rotate ->
   MultiNodeMesh::rotate(dAngle, axis, p) src/multi_node_mesh_I.h:620-660
   (nodes and centres) and TrackingMesh::rotate src/tracking_mesh_I.h:375
   (edgeVec, edgeNorm, surfaceNorm are rotated, src/surface_mesh_I.h:75-77),
   then v += omega x (node - p) */
static void move_mesh_rotate(orc_sim *s, wall_mesh *m)
{
    const double dAngle = m->mv_omega*s->p.dt;
    double axisNorm[3] = {m->mv_axis[0], m->mv_axis[1], m->mv_axis[2]};
    sdiv3(axisNorm, mag3(axisNorm));
    double dQ[4];
    dQ[0] = cos(dAngle*0.5);
    for (int i = 0; i < 3; i++) dQ[i+1] = axisNorm[i]*sin(dAngle*0.5);
    const double *origin = m->mv_point;
    const int trans = (origin[0]*origin[0] + origin[1]*origin[1] + origin[2]*origin[2]) > 0.;
    for (int t = 0; t < m->ntri; t++) {
        m->center[t][0] = m->center[t][1] = m->center[t][2] = 0.;
        for (int j = 0; j < 3; j++) {
            double *nd = m->node[t][j];
            if (trans) sub3(nd, origin, nd);
            vec_quat_rotate(nd, dQ);
            if (trans) { nd[0] = nd[0]+origin[0]; nd[1] = nd[1]+origin[1]; nd[2] = nd[2]+origin[2]; }
            for (int c = 0; c < 3; c++) m->center[t][c] = nd[c] + m->center[t][c];
        }
        sdiv3(m->center[t], 3.0);
        for (int j = 0; j < 3; j++) { vec_quat_rotate(m->edgevec[t][j], dQ); vec_quat_rotate(m->edgenorm[t][j], dQ); }
        vec_quat_rotate(m->surfnorm[t], dQ);
    }
    double omegaVec[3] = {m->mv_axis[0]*m->mv_omega, m->mv_axis[1]*m->mv_omega, m->mv_axis[2]*m->mv_omega};
    for (int t = 0; t < m->ntri; t++)
        for (int j = 0; j < 3; j++) {
            double rPA[3], vRot[3];
            m->vnode[t][j][0] = m->vnode[t][j][1] = m->vnode[t][j][2] = 0.;
            sub3(m->node[t][j], m->mv_point, rPA);
            cross3(omegaVec, rPA, vRot);
            for (int c = 0; c < 3; c++) m->vnode[t][j][c] = m->vnode[t][j][c] + vRot[c];
        }
}

/* MultiNodeMesh::decideRebuild src/multi_node_mesh_I.h:791-823 */
static int mesh_decide_rebuild(orc_sim *s, wall_mesh *m)
{
    if (!m->moving) return 0;
    const double triggersq = 0.25*s->p.skin*s->p.skin;
    for (int t = 0; t < m->ntri; t++) {
        int flag = 0;
        for (int j = 0; j < 3; j++) {
            double d[3]; sub3(m->node[t][j], m->node_last[t][j], d);
            double distSq = d[0]*d[0] + d[1]*d[1] + d[2]*d[2];
            if (distSq > triggersq) flag = 1;
        }
        if (flag) return 1;
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* mesh topology: src/surface_mesh_I.h:282-446 (element properties),
   :453-555 buildNeighbours, :1035-1152 edges/corners                   */

static int mesh_nodes_equal(wall_mesh *m, const double *a, const double *b)
{
    for (int i = 0; i < 3; i++) if (!comp_double(a[i], b[i], m->precision)) return 0;
    return 1;
}

static int mesh_n_shared(wall_mesh *m, int a, int b)   /* src/multi_node_mesh_I.h:328 */
{
    double dist[3]; sub3(m->center[a], m->center[b], dist);
    double radsum = m->rbound[a] + m->rbound[b];
    if (dot3(dist, dist) > radsum*radsum) return 0;
    int ns = 0;
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++) if (mesh_nodes_equal(m, m->node[a][i], m->node[b][j])) ns++;
    return ns;
}

static int mesh_share_edge(wall_mesh *m, int a, int b, int *ie, int *je)  /* src/surface_mesh_I.h:1003 */
{
    double dist[3]; sub3(m->center[a], m->center[b], dist);
    double radsum = m->rbound[a] + m->rbound[b];
    if (dot3(dist, dist) > radsum*radsum) return 0;
    int i1 = -1, j1 = -1, i2 = -1, j2 = -1, ns = 0;
    for (int i = 0; i < 3; i++) for (int j = 0; j < 3; j++)
        if (mesh_nodes_equal(m, m->node[a][i], m->node[b][j])) {
            if (ns == 0) { i1 = i; j1 = j; }
            else if (ns == 1) { i2 = i; j2 = j; goto found; }
            ns++;
        }
    return 0;
found:
    *ie = (2 == i1+i2) ? 2 : (i1 < i2 ? i1 : i2);
    *je = (2 == j1+j2) ? 2 : (j1 < j2 ? j1 : j2);
    return 1;
}

/* Surface properties of one element from its current nodes, as
   SurfaceMesh::calcSurfPropertiesOfNewElement computes them on import
   (src/surface_mesh_I.h:282-330) and recalcLocalSurfProperties recomputes
   them whenever a moving mesh is re-parallelised (:163-200) */
static void mesh_surf_props(wall_mesh *m, int t)
{
    /* calcEdgeVecLen :361 */
    for (int i = 0; i < 3; i++) {
        sub3(m->node[t][(i+1)%3], m->node[t][i], m->edgevec[t][i]);
        m->edgelen[t][i] = mag3(m->edgevec[t][i]);
        sdiv3(m->edgevec[t][i], m->edgelen[t][i]);
    }
    /* calcSurfaceNorm :374 (degenerate fallbacks omitted: duplicates removed) */
    double *sn = m->surfnorm[t];
    cross3(m->edgevec[t][0], m->edgevec[t][1], sn);
    if (mag3(sn) < 1e-15) cross3(m->edgevec[t][1], m->edgevec[t][2], sn);
    if (mag3(sn) < 1e-15) cross3(m->edgevec[t][2], m->edgevec[t][0], sn);
    sdiv3(sn, mag3(sn));
    /* calcEdgeNormals :417 */
    for (int i = 0; i < 3; i++) {
        cross3(m->edgevec[t][i], sn, m->edgenorm[t][i]);
        if (mag3(m->edgenorm[t][i]) < 1e-15) memcpy(m->edgenorm[t][i], m->edgevec[t][(i+1)%3], sizeof(double)*3);
        else sdiv3(m->edgenorm[t][i], mag3(m->edgenorm[t][i]));
    }
    /* calcObtuseAngleIndex :435, called for iNode = 0,1,2 -- each call
       overwrites the element's index, so the last call decides */
    m->obtuse[t] = NO_OBTUSE_ANGLE;
    for (int i = 0; i < 3; i++) {
        double d = dot3(m->edgevec[t][i], m->edgevec[t][(i+2)%3]);
        m->obtuse[t] = (d > 0.) ? i : NO_OBTUSE_ANGLE;
    }
}

/* FixMesh::pre_force on a re-neighbour step (src/fix_mesh.cpp:564-574):
   MultiNodeMeshParallel::pbcExchangeBorders (src/multi_node_mesh_parallel_I.h:
   652-700) returns at once for a static mesh; a moving mesh goes through
   refreshOwned, i.e. MultiNodeMesh::refreshOwned (storeNodePosRebuild,
   src/multi_node_mesh_I.h:212-225) and SurfaceMesh::recalcLocalSurfProperties
   (edge vectors and lengths, normal, edge normals, obtuse index and area from
   the current nodes, src/surface_mesh_I.h:163-200).  Centres and bounding
   radii stay (updateCenterRbound runs only for deforming meshes). */
static void mesh_refresh_owned(wall_mesh *m)
{
    if (!m->moving) return;
    memcpy(m->node_last, m->node, sizeof(double)*9*m->ntri);
    for (int t = 0; t < m->ntri; t++) {
        mesh_surf_props(m, t);
        if (m->area_ev) {   /* TriMesh::calcArea src/tri_mesh_I.h:305 reads edge vectors 0, 1 and lengths */
            memcpy(m->area_ev[t][0], m->edgevec[t][0], sizeof(double)*3);
            memcpy(m->area_ev[t][1], m->edgevec[t][1], sizeof(double)*3);
            m->area_el[t][0] = m->edgelen[t][0]; m->area_el[t][1] = m->edgelen[t][1];
        }
    }
}

static void mesh_build_topology(orc_sim *s, wall_mesh *m)
{
    const int n = m->ntri;
    (void)s;
    m->edgevec = malloc(sizeof(double)*9*(n?n:1)); m->edgelen = malloc(sizeof(double)*3*(n?n:1));
    m->edgenorm = malloc(sizeof(double)*9*(n?n:1)); m->surfnorm = malloc(sizeof(double)*3*(n?n:1));
    m->obtuse = malloc(sizeof(int)*(n?n:1));
    m->edge_active = malloc(3*(n?n:1)); m->corner_active = malloc(3*(n?n:1));
    m->nneigh = calloc(n?n:1, sizeof(int)); m->neighfaces = malloc(sizeof(int)*NEIGH_MAX*(n?n:1));
    for (int t = 0; t < n; t++) {
        mesh_surf_props(m, t);
        for (int i = 0; i < 3; i++) { m->edge_active[t][i] = 1; m->corner_active[t][i] = 1; }
        for (int i = 0; i < NEIGH_MAX; i++) m->neighfaces[t][i] = -1;
    }
    /* buildNeighbours: every pair sharing an edge (the bounding-sphere
       overlap search of :505-524 finds every such pair); element ids are
       the element indices (src/tracking_mesh_I.h:91) */
    for (int i = 0; i < n; i++)
        for (int j = 0; j < i; j++) {
            int ie, je;
            if (!mesh_share_edge(m, i, j, &ie, &je)) continue;
            /* areCoplanar :844 */
            int coplanar = fabs(dot3(m->surfnorm[i], m->surfnorm[j])) >= m->curvature;
            /* handleSharedEdge :1035 (neighflag true) */
            if (m->nneigh[i] < NEIGH_MAX) m->neighfaces[i][m->nneigh[i]] = j;
            if (m->nneigh[j] < NEIGH_MAX) m->neighfaces[j][m->nneigh[j]] = i;
            m->nneigh[i]++; m->nneigh[j]++;
            int overlap = 0;
            if (coplanar) {   /* coplanarNeighsOverlap :935 */
                double pRef[3], edgeN[3], vecI[3], vecJ[3];
                memcpy(pRef, m->node[i][ie], sizeof pRef);
                memcpy(edgeN, m->edgenorm[i][ie], sizeof edgeN);
                sub3(m->node[i][(ie+2)%3], pRef, vecI);
                sub3(m->node[j][(je+2)%3], pRef, vecJ);
                double d1 = dot3(vecI, edgeN), d2 = dot3(vecJ, edgeN);
                overlap = d1*d2 > 0.;
            }
            if (!coplanar || overlap) {
                if (i < j) { m->edge_active[i][ie] = 0; m->edge_active[j][je] = 1; }
                else { m->edge_active[i][ie] = 1; m->edge_active[j][je] = 0; }
            } else { m->edge_active[i][ie] = 0; m->edge_active[j][je] = 0; }
        }
    /* handleCorner :1109 with checkNodeRecursive :1159 (depth-first over
       edge neighbours that contain the node) */
    int *visited = malloc(sizeof(int)*(n?n:1)), *hasnode = malloc(sizeof(int)*(n?n:1));
    int *stack = malloc(sizeof(int)*(n?n:1)*(NEIGH_MAX+1));
    double (*edgelist)[3] = malloc(sizeof(double)*3*2*(n?n:1));
    double (*endpt)[3] = malloc(sizeof(double)*3*2*(n?n:1));
    unsigned char *vis = calloc(n?n:1, 1);
    for (int t = 0; t < n; t++)
        for (int inode = 0; inode < 3; inode++) {
            double nc[3]; memcpy(nc, m->node[t][inode], sizeof nc);
            int nvis = 0, nhas = 0, anyActive = 0, ne = 0;
            /* recursion order does not change the sets collected */
            int sp = 0; stack[sp++] = t;
            while (sp > 0) {
                int e = stack[--sp];
                if (vis[e]) continue;
                vis[e] = 1; visited[nvis++] = e;
                int in = -1;
                for (int q = 0; q < 3; q++)
                    if (comp_double(m->node[e][q][0], nc[0], m->precision) && comp_double(m->node[e][q][1], nc[1], m->precision) &&
                        comp_double(m->node[e][q][2], nc[2], m->precision)) { in = q; break; }
                if (in < 0) continue;
                hasnode[nhas++] = e;
                memcpy(edgelist[ne], m->edgevec[e][in], sizeof(double)*3);
                memcpy(endpt[ne], m->node[e][(in+1)%3], sizeof(double)*3); ne++;
                memcpy(edgelist[ne], m->edgevec[e][(in+2)%3], sizeof(double)*3);
                memcpy(endpt[ne], m->node[e][(in+2)%3], sizeof(double)*3); ne++;
                if (m->edge_active[e][in]) anyActive = 1;
                else if (m->edge_active[e][(in+2)%3]) anyActive = 1;
                int nn = m->nneigh[e] < NEIGH_MAX ? m->nneigh[e] : NEIGH_MAX;
                for (int k = nn-1; k >= 0; k--) { int nb = m->neighfaces[e][k]; if (nb >= 0 && !vis[nb]) stack[sp++] = nb; }
            }
            for (int q = 0; q < nvis; q++) vis[visited[q]] = 0;
            int maxId = -1;
            for (int q = 0; q < nhas; q++) maxId = maxId > hasnode[q] ? maxId : hasnode[q];
            int colinear = 0;
            for (int a = 0; a < ne; a++)
                for (int b = a+1; b < ne; b++)
                    if (fabs(dot3(edgelist[a], edgelist[b])) > m->curvature && !mesh_nodes_equal(m, endpt[a], endpt[b])) colinear = 1;
            if (colinear || !anyActive) m->corner_active[t][inode] = 0;
            else if (t == maxId) m->corner_active[t][inode] = 1;
            else m->corner_active[t][inode] = 0;
        }
    free(visited); free(hasnode); free(stack); free(edgelist); free(endpt); free(vis);
}

/* areCoplanarNodeNeighs src/surface_mesh_I.h:892 */
static int mesh_coplanar_node_neighs(wall_mesh *m, int a, int b)
{
    int areNeighs = 0;
    int nn = m->nneigh[a] < NEIGH_MAX ? m->nneigh[a] : NEIGH_MAX;
    for (int i = 0; i < nn; i++) if (m->neighfaces[a][i] == b) areNeighs = 1;
    int found = 0;
    if (!areNeighs) if (mesh_n_shared(m, a, b) != 0) found = 1;
    if (!areNeighs && !found) return 0;
    double d = dot3(m->surfnorm[a], m->surfnorm[b]);
    return fabs(d) > m->curvature;
}

int orc_get_mesh_topology(orc_sim *s, int ifix, unsigned char *edge_active, unsigned char *corner_active, int *obtuse)
{
    wall_mesh *m = s->fix[ifix].wm;
    if (!m) return -1;
    for (int t = 0; t < m->ntri; t++) {
        for (int i = 0; i < 3; i++) {
            if (edge_active) edge_active[3*t+i] = m->edge_active[t][i];
            if (corner_active) corner_active[3*t+i] = m->corner_active[t][i];
        }
        if (obtuse) obtuse[t] = m->obtuse[t];
    }
    return m->ntri;
}

/* ------------------------------------------------------------------ */
/* neighbor: cutoffs src/neighbor.cpp:292-332, src/pair_gran.cpp:623;
   bins src/neighbor.cpp:1642-1808; stencil src/neigh_stencil.cpp:116  */

static void neighbor_init(orc_sim *s)
{
    const int nt = s->ntypes;
    free(s->maxrad);
    s->maxrad = calloc(nt+1, sizeof(double));
    if (s->ins)   /* future particles count as dynamic, src/pair_gran.cpp:540-554 */
        for (int t = 1; t <= nt; t++) ins_max_rad(s->ins, t, &s->maxrad[t]);
    for (int i = 0; i < s->nlocal; i++)
        if (s->radius[i] > s->maxrad[s->type[i]]) s->maxrad[s->type[i]] = s->radius[i];
    s->triggersq = 0.25*s->p.skin*s->p.skin;
    s->cutneighmax = 0.0;
    for (int i = 1; i <= nt; i++)
        for (int j = 1; j <= nt; j++) {
            double cut = (s->maxrad[i]+s->maxrad[j]) * 1.0;   /* init_one * contactDistanceFactor */
            double cutsq = cut*cut;
            double cutoff = sqrt(cutsq);
            double delta = cutoff > 0.0 ? s->p.skin : 0.0;
            double c = cutoff + delta;
            if (c > s->cutneighmax) s->cutneighmax = c;
        }
    s->cutneighmaxsq = s->cutneighmax * s->cutneighmax;
    s->cutghost = s->cutneighmax;   /* src/comm.cpp:456, cutghostuser = 0 */
}

static double bin_distance(orc_sim *s, int i, int j, int k)
{
    double delx, dely, delz;
    if (i > 0) delx = (i-1)*s->binsizex; else if (i == 0) delx = 0.0; else delx = (i+1)*s->binsizex;
    if (j > 0) dely = (j-1)*s->binsizey; else if (j == 0) dely = 0.0; else dely = (j+1)*s->binsizey;
    if (k > 0) delz = (k-1)*s->binsizez; else if (k == 0) delz = 0.0; else delz = (k+1)*s->binsizez;
    return (delx*delx + dely*dely + delz*delz);
}

static void setup_bins(orc_sim *s)
{
    double bbox[3], bsubboxlo[3], bsubboxhi[3];
    for (int d = 0; d < 3; d++) {
        s->bboxlo[d] = s->boxlo[d]; s->bboxhi[d] = s->boxhi[d];
        bsubboxlo[d] = s->boxlo[d] - s->cutghost;
        bsubboxhi[d] = s->boxhi[d] + s->cutghost;
        bbox[d] = s->bboxhi[d] - s->bboxlo[d];
    }
    double binsize_optimal = 0.5*s->cutneighmax;
    if (binsize_optimal == 0.0) binsize_optimal = bbox[0];
    double binsizeinv = 1.0/binsize_optimal;
    s->nbinx = (int)(bbox[0]*binsizeinv);
    s->nbiny = (int)(bbox[1]*binsizeinv);
    s->nbinz = (int)(bbox[2]*binsizeinv);
    if (s->nbinx == 0) s->nbinx = 1;
    if (s->nbiny == 0) s->nbiny = 1;
    if (s->nbinz == 0) s->nbinz = 1;
    s->binsizex = bbox[0]/s->nbinx; s->binsizey = bbox[1]/s->nbiny; s->binsizez = bbox[2]/s->nbinz;
    s->bininvx = 1.0 / s->binsizex; s->bininvy = 1.0 / s->binsizey; s->bininvz = 1.0 / s->binsizez;
    int mbinxhi, mbinyhi, mbinzhi;
    double coord;
    coord = bsubboxlo[0] - SMALL*bbox[0];
    s->mbinxlo = (int)((coord-s->bboxlo[0])*s->bininvx);
    if (coord < s->bboxlo[0]) s->mbinxlo = s->mbinxlo - 1;
    coord = bsubboxhi[0] + SMALL*bbox[0];
    mbinxhi = (int)((coord-s->bboxlo[0])*s->bininvx);
    coord = bsubboxlo[1] - SMALL*bbox[1];
    s->mbinylo = (int)((coord-s->bboxlo[1])*s->bininvy);
    if (coord < s->bboxlo[1]) s->mbinylo = s->mbinylo - 1;
    coord = bsubboxhi[1] + SMALL*bbox[1];
    mbinyhi = (int)((coord-s->bboxlo[1])*s->bininvy);
    coord = bsubboxlo[2] - SMALL*bbox[2];
    s->mbinzlo = (int)((coord-s->bboxlo[2])*s->bininvz);
    if (coord < s->bboxlo[2]) s->mbinzlo = s->mbinzlo - 1;
    coord = bsubboxhi[2] + SMALL*bbox[2];
    mbinzhi = (int)((coord-s->bboxlo[2])*s->bininvz);
    s->mbinxlo -= 1; mbinxhi += 1; s->mbinx = mbinxhi - s->mbinxlo + 1;
    s->mbinylo -= 1; mbinyhi += 1; s->mbiny = mbinyhi - s->mbinylo + 1;
    s->mbinzlo -= 1; mbinzhi += 1; s->mbinz = mbinzhi - s->mbinzlo + 1;
    s->mbins = s->mbinx*s->mbiny*s->mbinz;
    s->binhead = xrealloc(s->binhead, sizeof(int)*s->mbins);
    int sx = (int)(s->cutneighmax*s->bininvx); if (sx*s->binsizex < s->cutneighmax) sx++;
    int sy = (int)(s->cutneighmax*s->bininvy); if (sy*s->binsizey < s->cutneighmax) sy++;
    int sz = (int)(s->cutneighmax*s->bininvz); if (sz*s->binsizez < s->cutneighmax) sz++;
    int smax = (2*sx+1)*(2*sy+1)*(2*sz+1);
    s->stencil = xrealloc(s->stencil, sizeof(int)*smax);
    s->nstencil = 0;
    for (int k = -sz; k <= sz; k++)
        for (int j = -sy; j <= sy; j++)
            for (int i = -sx; i <= sx; i++)
                if (bin_distance(s, i, j, k) < s->cutneighmaxsq)
                    s->stencil[s->nstencil++] = k*s->mbiny*s->mbinx + j*s->mbinx + i;
}

/* src/neighbor.cpp:2112 (index triple relative to mbin*lo) */
static int coord2bin3(orc_sim *s, const double *x, int *ix, int *iy, int *iz)
{
    if (x[0] >= s->bboxhi[0]) *ix = (int)((x[0]-s->bboxhi[0])*s->bininvx) + s->nbinx;
    else if (x[0] >= s->bboxlo[0]) { *ix = (int)((x[0]-s->bboxlo[0])*s->bininvx); if (*ix > s->nbinx-1) *ix = s->nbinx-1; }
    else *ix = (int)((x[0]-s->bboxlo[0])*s->bininvx) - 1;
    if (x[1] >= s->bboxhi[1]) *iy = (int)((x[1]-s->bboxhi[1])*s->bininvy) + s->nbiny;
    else if (x[1] >= s->bboxlo[1]) { *iy = (int)((x[1]-s->bboxlo[1])*s->bininvy); if (*iy > s->nbiny-1) *iy = s->nbiny-1; }
    else *iy = (int)((x[1]-s->bboxlo[1])*s->bininvy) - 1;
    if (x[2] >= s->bboxhi[2]) *iz = (int)((x[2]-s->bboxhi[2])*s->bininvz) + s->nbinz;
    else if (x[2] >= s->bboxlo[2]) { *iz = (int)((x[2]-s->bboxlo[2])*s->bininvz); if (*iz > s->nbinz-1) *iz = s->nbinz-1; }
    else *iz = (int)((x[2]-s->bboxlo[2])*s->bininvz) - 1;
    *ix -= s->mbinxlo; *iy -= s->mbinylo; *iz -= s->mbinzlo;
    return (*iz)*s->mbiny*s->mbinx + (*iy)*s->mbinx + (*ix);
}

static int coord2bin(orc_sim *s, const double *x)   /* src/neighbor.cpp:2077 */
{
    int ix, iy, iz;
    return coord2bin3(s, x, &ix, &iy, &iz);
}

static void bin_atoms(orc_sim *s)   /* src/neighbor.cpp:2027 */
{
    for (int i = 0; i < s->mbins; i++) s->binhead[i] = -1;
    int nall = s->nlocal + s->nghost;
    for (int i = nall-1; i >= 0; i--) {
        int ibin = coord2bin(s, &s->x[3*i]);
        s->bins[i] = s->binhead[ibin];
        s->binhead[ibin] = i;
    }
}

/* ------------------------------------------------------------------ */
/* domain / comm                                                        */

static void domain_pbc(orc_sim *s)   /* src/domain.cpp:530 */
{
    for (int i = 0; i < s->nlocal; i++)
        for (int d = 0; d < 3; d++) {
            if (!s->p.periodic[d]) continue;
            double *xc = &s->x[3*i+d];
            if (*xc < s->boxlo[d]) *xc += s->prd[d];
            if (*xc >= s->boxhi[d]) { *xc -= s->prd[d]; if (*xc < s->boxlo[d]) *xc = s->boxlo[d]; }
        }
}

static int comm_exchange_check(orc_sim *s)   /* src/comm.cpp:901, one proc */
{
    for (int i = 0; i < s->nlocal; i++)
        for (int d = 0; d < 3; d++)
            if (s->x[3*i+d] < s->boxlo[d] || s->x[3*i+d] >= s->boxhi[d]) {
                fail(s, "atom tag %d left the box in dim %d (lost atoms are not supported)", s->tag[i], d);
                return -1;
            }
    return 0;
}

/* Comm::borders src/comm.cpp:1028 with Comm::decide src/comm_I.h:66 and
   the swap slabs of Comm::setup src/comm.cpp:655-712 (one proc) */
static void comm_borders(orc_sim *s)
{
    s->nghost = 0;
    s->nswap = 0;
    const double c = s->cutghost / 2. + s->p.skin/2.;
    int nlast = 0;
    for (int dim = 0; dim < 3; dim++) {
        if (!s->p.periodic[dim]) continue;   /* maxneed = 0 for a non-periodic dim with one proc */
        nlast = 0;
        int nfirst = 0;
        for (int ineed = 0; ineed < 2; ineed++) {
            double lo, hi, shift;
            if (ineed % 2 == 0) { lo = -BIG; hi = s->boxlo[dim] + c; shift = 1*s->prd[dim]; }
            else { lo = s->boxhi[dim] - c; hi = BIG; shift = -1*s->prd[dim]; }
            if (ineed % 2 == 0) { nfirst = nlast; nlast = s->nlocal + s->nghost; }
            (void)nfirst;
            int first = s->nlocal + s->nghost;
            int nsend = 0;
            for (int i = 0; i < nlast; i++) {
                double xd = s->x[3*i+dim];
                int send = (ineed % 2 == 0) ? (xd >= lo && xd <= (hi + s->radius[i]))
                                            : (xd >= (lo - s->radius[i]) && xd <= hi);
                if (!send) continue;
                int g = first + nsend;
                if (g >= s->nmax) grow_all(s, 2*s->nmax);
                s->gsrc = xrealloc(s->gsrc, sizeof(int)*(g - s->nlocal + 1));
                s->gshift = xrealloc(s->gshift, sizeof(double)*3*(g - s->nlocal + 1));
                int gi = g - s->nlocal;
                s->gsrc[gi] = i;
                double sh[3] = {0.0, 0.0, 0.0}; sh[dim] = shift;
                /* dx = pbc[0]*xprd etc: only the swap dimension is nonzero */
                for (int d = 0; d < 3; d++) { s->gshift[3*gi+d] = (d == dim) ? shift : 0*s->prd[d]; s->x[3*g+d] = s->x[3*i+d] + s->gshift[3*gi+d]; }
                (void)sh;
                s->v[3*g] = s->v[3*i]; s->v[3*g+1] = s->v[3*i+1]; s->v[3*g+2] = s->v[3*i+2];
                s->omega[3*g] = s->omega[3*i]; s->omega[3*g+1] = s->omega[3*i+1]; s->omega[3*g+2] = s->omega[3*i+2];
                s->radius[g] = s->radius[i]; s->rmass[g] = s->rmass[i]; s->type[g] = s->type[i]; s->tag[g] = s->tag[i];
                nsend++;
            }
            s->swapfirst[s->nswap] = first; s->swapnum[s->nswap] = nsend; s->nswap++;
            s->nghost += nsend;
        }
    }
}

static void comm_forward(orc_sim *s)   /* src/comm.cpp:773 with pack_comm_vel */
{
    for (int gi = 0; gi < s->nghost; gi++) {
        int g = s->nlocal + gi, i = s->gsrc[gi];
        for (int d = 0; d < 3; d++) s->x[3*g+d] = s->x[3*i+d] + s->gshift[3*gi+d];
        for (int d = 0; d < 3; d++) { s->v[3*g+d] = s->v[3*i+d]; s->omega[3*g+d] = s->omega[3*i+d]; }
    }
}

/* ------------------------------------------------------------------ */
/* atom sort src/atom.cpp:1309-1398, bins :1405-1480                    */

static void setup_sort_bins(orc_sim *s)
{
    double binsize = s->p.sortbinsize > 0.0 ? s->p.sortbinsize : 0.5 * s->cutneighmax;
    double bininv = 1.0/binsize;
    for (int d = 0; d < 3; d++) s->sbboxlo[d] = s->boxlo[d];
    s->snbinx = (int)((s->boxhi[0]-s->boxlo[0]) * bininv);
    s->snbiny = (int)((s->boxhi[1]-s->boxlo[1]) * bininv);
    s->snbinz = (int)((s->boxhi[2]-s->boxlo[2]) * bininv);
    if (s->snbinx == 0) s->snbinx = 1;
    if (s->snbiny == 0) s->snbiny = 1;
    if (s->snbinz == 0) s->snbinz = 1;
    s->sbininvx = s->snbinx / (s->boxhi[0]-s->boxlo[0]);
    s->sbininvy = s->snbiny / (s->boxhi[1]-s->boxlo[1]);
    s->sbininvz = s->snbinz / (s->boxhi[2]-s->boxlo[2]);
}

#define PERMUTE(arr, type, width) do { type *tmp_ = malloc(sizeof(type)*(width)*(size_t)(n>0?n:1)); \
    for (int q_ = 0; q_ < n; q_++) memcpy(tmp_ + (size_t)(width)*q_, (arr) + (size_t)(width)*perm[q_], sizeof(type)*(width)); \
    memcpy((arr), tmp_, sizeof(type)*(width)*(size_t)n); free(tmp_); } while (0)

static void atom_sort(orc_sim *s)
{
    s->nextsort = (s->ntimestep/s->p.sortfreq)*s->p.sortfreq + s->p.sortfreq;
    int nbins = s->snbinx*s->snbiny*s->snbinz;
    if (nbins == 1) return;
    const int n = s->nlocal;
    int *binhead = malloc(sizeof(int)*nbins), *next = malloc(sizeof(int)*(n>0?n:1)), *perm = malloc(sizeof(int)*(n>0?n:1));
    for (int i = 0; i < nbins; i++) binhead[i] = -1;
    for (int i = n-1; i >= 0; i--) {
        int ix = (int)((s->x[3*i]-s->sbboxlo[0])*s->sbininvx);
        int iy = (int)((s->x[3*i+1]-s->sbboxlo[1])*s->sbininvy);
        int iz = (int)((s->x[3*i+2]-s->sbboxlo[2])*s->sbininvz);
        if (ix < 0) ix = 0; if (iy < 0) iy = 0; if (iz < 0) iz = 0;
        if (ix > s->snbinx-1) ix = s->snbinx-1; if (iy > s->snbiny-1) iy = s->snbiny-1; if (iz > s->snbinz-1) iz = s->snbinz-1;
        int ibin = iz*s->snbiny*s->snbinx + iy*s->snbinx + ix;
        next[i] = binhead[ibin]; binhead[ibin] = i;
    }
    int k = 0;
    for (int m = 0; m < nbins; m++) for (int i = binhead[m]; i >= 0; i = next[i]) perm[k++] = i;
    /* perm[new] = old; every per-atom array moves with its atom */
    PERMUTE(s->x, double, 3); PERMUTE(s->v, double, 3); PERMUTE(s->omega, double, 3);
    PERMUTE(s->f, double, 3); PERMUTE(s->torque, double, 3);
    PERMUTE(s->radius, double, 1); PERMUTE(s->rmass, double, 1);
    PERMUTE(s->type, int, 1); PERMUTE(s->tag, int, 1);
    PERMUTE(s->npartner, int, 1); PERMUTE(s->partner, int*, 1); PERMUTE(s->phist, double*, 1);
    for (int q = 0; q < s->nfix; q++) {
        if (s->fix[q].wp) PERMUTE(s->fix[q].wp->hist, double, 3);
        if (s->fix[q].wm) {
            wall_mesh *m = s->fix[q].wm;
            PERMUTE(m->nneighs, int, 1); PERMUTE(m->npartner, int, 1); PERMUTE(m->partner, int*, 1);
            PERMUTE(m->chist, double*, 1); PERMUTE(m->keep, unsigned char*, 1); PERMUTE(m->isect, unsigned char*, 1);
        }
    }
    free(binhead); free(next); free(perm);
}

/* ------------------------------------------------------------------ */
/* FixContactHistory::pre_exchange src/fix_contact_history.cpp:305-425 */

static void history_pre_exchange(orc_sim *s)
{
    s->computeflag = 0;
    const int nl = s->nlocal;
    for (int i = 0; i < nl; i++) { free(s->partner[i]); free(s->phist[i]); s->partner[i] = NULL; s->phist[i] = NULL; s->npartner[i] = 0; }
    int inum = s->npairs > 0 || nl > 0 ? nl : 0;
    int nlocal_neigh = inum;  /* ilist[inum-1]+1 */
    int *cnt = calloc(nl > 0 ? nl : 1, sizeof(int));
    for (int i = 0; i < nl; i++)
        for (int jj = 0; jj < s->nnum[i]; jj++) {
            int e = s->nstart[i] + jj;
            if (s->flag[e]) { cnt[i]++; int j = s->nbr[e]; if (j < nlocal_neigh) cnt[j]++; }
        }
    for (int i = 0; i < nl; i++) {
        s->partner[i] = malloc(sizeof(int)*(cnt[i] > 0 ? cnt[i] : 1));
        s->phist[i] = malloc(sizeof(double)*3*(cnt[i] > 0 ? cnt[i] : 1));
    }
    for (int i = 0; i < nl; i++)
        for (int jj = 0; jj < s->nnum[i]; jj++) {
            int e = s->nstart[i] + jj;
            if (!s->flag[e]) continue;
            double *h = &s->hist[3*e];
            int j = s->nbr[e];
            int m = s->npartner[i];
            s->partner[i][m] = s->tag[j];
            for (int d = 0; d < 3; d++) s->phist[i][3*m+d] = h[d];
            s->npartner[i]++;
            if (j < nlocal_neigh) {
                m = s->npartner[j];
                s->partner[j][m] = s->tag[i];
                for (int d = 0; d < 3; d++) s->phist[j][3*m+d] = -h[d];   /* newtonflag = 1 for shear */
                s->npartner[j]++;
            }
        }
    free(cnt);
}

/* ------------------------------------------------------------------ */
/* Neighbor::granular_bin_no_newton src/neigh_gran.cpp:485-639         */

static void neighbor_build(orc_sim *s)
{
    s->ago = 0;
    s->nbuilds++;
    for (int i = 0; i < 3*s->nlocal; i++) s->xhold[i] = s->x[i];
    bin_atoms(s);
    const int nl = s->nlocal;
    s->nstart = xrealloc(s->nstart, sizeof(int)*(nl > 0 ? nl : 1));
    s->nnum = xrealloc(s->nnum, sizeof(int)*(nl > 0 ? nl : 1));
    s->npairs = 0;
    const double skin = s->p.skin;
    for (int i = 0; i < nl; i++) {
        s->nstart[i] = s->npairs;
        int n = 0;
        const double xtmp = s->x[3*i], ytmp = s->x[3*i+1], ztmp = s->x[3*i+2];
        const double radi = s->radius[i];
        int ibin = coord2bin(s, &s->x[3*i]);
        for (int k = 0; k < s->nstencil; k++)
            for (int j = s->binhead[ibin+s->stencil[k]]; j >= 0; j = s->bins[j]) {
                if (j <= i) continue;
                double delx = xtmp - s->x[3*j], dely = ytmp - s->x[3*j+1], delz = ztmp - s->x[3*j+2];
                double rsq = delx*delx + dely*dely + delz*delz;
                double radsum = (radi + s->radius[j]) * 1.0;
                double cutsq = (radsum+skin) * (radsum+skin);
                if (rsq <= cutsq) {
                    if (s->npairs >= s->cappairs) {
                        s->cappairs = s->cappairs ? 2*s->cappairs : 1024;
                        s->nbr = xrealloc(s->nbr, sizeof(int)*s->cappairs);
                        s->flag = xrealloc(s->flag, sizeof(int)*s->cappairs);
                        s->hist = xrealloc(s->hist, sizeof(double)*3*s->cappairs);
                    }
                    int e = s->npairs++;
                    s->nbr[e] = j;
                    int m = 0;
                    if (rsq < radsum*radsum) {
                        for (m = 0; m < s->npartner[i]; m++) if (s->partner[i][m] == s->tag[j]) break;
                        if (m < s->npartner[i]) {
                            s->flag[e] = 1;
                            for (int d = 0; d < 3; d++) s->hist[3*e+d] = s->phist[i][3*m+d];
                        } else {
                            s->flag[e] = 0;
                            for (int d = 0; d < 3; d++) s->hist[3*e+d] = 0.0;
                        }
                    } else {
                        s->flag[e] = 0;
                        for (int d = 0; d < 3; d++) s->hist[3*e+d] = 0.0;
                    }
                    n++;
                }
            }
        s->nnum[i] = n;
    }
}

/* Neighbor::decide / check_distance src/neighbor.cpp:1357-1460 */
static int neighbor_decide(orc_sim *s)
{
    /* must_check: fixes with force_reneighbor (FixMesh::next_reneighbor) src/neighbor.cpp:1359-1364 */
    for (int k = 0; k < s->nfix; k++)
        if (s->fix[k].kind == ORC_FIX_WALL_MESH && s->fix[k].wm->moving && s->fix[k].wm->next_reneighbor == s->ntimestep)
            return 1;
    if (s->ins && ins_next(s->ins) == s->ntimestep) return 1;   /* FixInsert::next_reneighbor */
    s->ago++;
    if (s->ago >= s->p.delay && s->ago % s->p.every == 0) {
        if (!s->p.check) return 1;
        const double deltasq = s->triggersq;
        int flag = 0;
        for (int i = 0; i < s->nlocal; i++) {
            double delx = s->x[3*i] - s->xhold[3*i];
            double dely = s->x[3*i+1] - s->xhold[3*i+1];
            double delz = s->x[3*i+2] - s->xhold[3*i+2];
            double rsq = delx*delx + dely*dely + delz*delz;
            if (rsq > deltasq) flag = 1;
        }
        return flag;
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* pair compute src/pair_gran_base.h:187-430                            */

static void pair_compute(orc_sim *s, int shearupdate)
{
    s->computeflag = 1;
    for (int i = 0; i < s->nlocal; i++) {
        const double xtmp = s->x[3*i], ytmp = s->x[3*i+1], ztmp = s->x[3*i+2];
        const double radi = s->radius[i];
        for (int jj = 0; jj < s->nnum[i]; jj++) {
            const int e = s->nstart[i] + jj;
            const int j = s->nbr[e];
            const double delx = xtmp - s->x[3*j], dely = ytmp - s->x[3*j+1], delz = ztmp - s->x[3*j+2];
            const double rsq = delx * delx + dely * dely + delz * delz;
            const double radj = s->radius[j];
            const double radsum = radi + radj;
            if (!(rsq < radsum * radsum)) continue;   /* surfacesClose unreachable with cdf = 1 */
            sidata_t sd; memset(&sd, 0, sizeof sd);
            force_t fi, fj; memset(&fi, 0, sizeof fi); memset(&fj, 0, sizeof fj);
            sd.is_wall = 0;
            sd.radi = radi; sd.radj = radj; sd.radsum = radsum; sd.rsq = rsq;
            sd.delta[0] = delx; sd.delta[1] = dely; sd.delta[2] = delz;
            sd.contact_flags = &s->flag[e];
            sd.contact_history = &s->hist[3*e];
            sd.v_i = &s->v[3*i]; sd.v_j = &s->v[3*j];
            sd.itype = s->type[i]; sd.jtype = s->type[j];
            sd.computeflag = 1; sd.shearupdate = shearupdate;
            const double r = sqrt(rsq);
            const double rinv = 1.0 / r;
            const double mi = s->rmass[i], mj = s->rmass[j];
            const double meff = mi * mj / (mi + mj);
            sd.r = r; sd.rinv = rinv; sd.meff = meff; sd.mi = mi; sd.mj = mj;
            sd.en[0] = delx * rinv; sd.en[1] = dely * rinv; sd.en[2] = delz * rinv;
            sd.omega_i = &s->omega[3*i]; sd.omega_j = &s->omega[3*j];
            contact_chain(s, &sd, &fi, &fj, s->p.rolling_cdt);
            for (int c = 0; c < 3; c++) { s->f[3*i+c] += 1.0*fi.F[c]; s->torque[3*i+c] += 1.0*fi.T[c]; }
            if (j < s->nlocal)
                for (int c = 0; c < 3; c++) { s->f[3*j+c] += 1.0*fj.F[c]; s->torque[3*j+c] += 1.0*fj.T[c]; }
        }
    }
}

void orc_pair_force(const orc_params *p, const double xi[3], const double xj[3], const double vi[3], const double vj[3],
                    const double wi[3], const double wj[3], double ri, double rj, double mi, double mj, int ti, int tj,
                    double shear[3], int shearupdate, double fi_out[3], double ti_out[3], double fj_out[3], double tj_out[3])
{
    orc_sim tmp; memset(&tmp, 0, sizeof tmp);
    tmp.p = *p; tmp.ntypes = p->ntypes; setup_materials(&tmp);
    sidata_t sd; memset(&sd, 0, sizeof sd);
    force_t fi, fj; memset(&fi, 0, sizeof fi); memset(&fj, 0, sizeof fj);
    const double delx = xi[0]-xj[0], dely = xi[1]-xj[1], delz = xi[2]-xj[2];
    const double rsq = delx*delx + dely*dely + delz*delz;
    int flagv = 0;
    if (rsq < (ri+rj)*(ri+rj)) {
        sd.radi = ri; sd.radj = rj; sd.radsum = ri+rj; sd.rsq = rsq;
        sd.delta[0] = delx; sd.delta[1] = dely; sd.delta[2] = delz;
        sd.contact_flags = &flagv; sd.contact_history = shear;
        sd.v_i = vi; sd.v_j = vj; sd.itype = ti; sd.jtype = tj; sd.computeflag = 1; sd.shearupdate = shearupdate;
        const double r = sqrt(rsq), rinv = 1.0/r;
        sd.r = r; sd.rinv = rinv; sd.meff = mi*mj/(mi+mj); sd.mi = mi; sd.mj = mj;
        sd.en[0] = delx*rinv; sd.en[1] = dely*rinv; sd.en[2] = delz*rinv;
        sd.omega_i = wi; sd.omega_j = wj;
        contact_chain(&tmp, &sd, &fi, &fj, p->rolling_cdt);
    }
    for (int c = 0; c < 3; c++) { fi_out[c] = fi.F[c]; ti_out[c] = fi.T[c]; fj_out[c] = fj.F[c]; tj_out[c] = fj.T[c]; }
    free_matrix(tmp.Yeff); free_matrix(tmp.Geff); free_matrix(tmp.betaeff); free_matrix(tmp.mu); free_matrix(tmp.mur);
}

/* ------------------------------------------------------------------ */
/* walls: Walls::Granular::compute_force src/fix_wall_gran_base.h:148  */

static void wall_compute_force(orc_sim *s, int ip, sidata_t *sd, const double *vwall, int wtype, int rolling, int shearupdate,
                               double *fout)
{
    force_t fi, fj; memset(&fi, 0, sizeof fi); memset(&fj, 0, sizeof fj);
    sd->v_i = &s->v[3*ip]; sd->v_j = vwall; sd->omega_i = &s->omega[3*ip];
    sd->r = sd->radi - sd->deltan;
    sd->rsq = sd->r*sd->r;
    const double rinv = 1.0/sd->r;
    sd->rinv = rinv;
    sd->contact_flags = NULL;
    sd->itype = s->type[ip];
    sd->meff = s->rmass[ip]; sd->mi = s->rmass[ip];
    sd->computeflag = 1; sd->shearupdate = shearupdate;
    sd->jtype = wtype;
    sd->en[0] = sd->delta[0] * rinv; sd->en[1] = sd->delta[1] * rinv; sd->en[2] = sd->delta[2] * rinv;
    sd->radsum = sd->radi;
    contact_chain(s, sd, &fi, &fj, rolling);
    for (int c = 0; c < 3; c++) { s->f[3*ip+c] += fi.F[c]; s->torque[3*ip+c] += fi.T[c]; }
    if (fout) for (int c = 0; c < 3; c++) fout[c] = fi.F[c];
}

/* FixWallGran::pre_force (primitive neighlist) src/fix_wall_gran.cpp:708,
   PrimitiveWall::buildNeighList src/primitive_wall.h:129,
   Plane::resolveNeighlist src/primitive_wall_definitions.h:145 */
/* Cylinder<dim>::calcRadialDistance src/primitive_wall_definitions.h:165 */
static double cyl_radial(const wall_plane *w, const double *pos, double *dy, double *dz)
{
    *dy = pos[(w->dim+1)%3] - w->cyl_c1;
    *dz = pos[(w->dim+2)%3] - w->cyl_c2;
    return sqrt((*dy)*(*dy) + (*dz)*(*dz));
}

static void wall_plane_pre_force(orc_sim *s, wall_plane *w)
{
    if (!w->rebuild) return;
    w->rebuild = 0;
    w->nlist = 0;
    for (int i = 0; i < s->nlocal; i++) {
        double dMax = s->radius[i] + s->p.skin;
        int in;
        if (w->cyl) {   /* Cylinder<dim>::resolveNeighlist :201 (as written: near inside, or beyond dMax outside) */
            double dy, dz;
            double dist = cyl_radial(w, &s->x[3*i], &dy, &dz) - w->cyl_r;
            in = (dMax < dist || -dMax < dist);
        } else {
            double dist = s->x[3*i+w->dim] - w->pos;
            double absdist = (dist > 0.0) ? dist : -dist;
            in = absdist <= dMax;
        }
        if (in) {
            if (w->nlist >= w->caplist) { w->caplist = w->caplist ? 2*w->caplist : 256; w->list = xrealloc(w->list, sizeof(int)*w->caplist); }
            w->list[w->nlist++] = i;
        }
    }
}

/* FixWallGran::post_force_primitive src/fix_wall_gran.cpp:1024-1148 */
static void wall_plane_post_force(orc_sim *s, wall_plane *w, int shearupdate)
{
    const double vwall[3] = {0., 0., 0.};
    for (int ic = 0; ic < w->nlist; ic++) {
        int ip = w->list[ic];
        sidata_t sd; memset(&sd, 0, sizeof sd);
        sd.is_wall = 1;
        sd.radi = s->radius[ip];
        double delta[3] = {0., 0., 0.}, deltan;
        const double *pos = &s->x[3*ip];
        if (w->cyl) {   /* Cylinder<dim>::resolveContact src/primitive_wall_definitions.h:172-197 */
            double dy, dz;
            const double dist = cyl_radial(w, pos, &dy, &dz);
            const int y = (w->dim+1)%3, z = (w->dim+2)%3;
            if (dist < 1e-13 && dist > -1e-13) {   /* compDouble(dist, 0.0) */
                deltan = 0.0;
            } else if (dist > w->cyl_r) {
                deltan = dist - w->cyl_r - sd.radi;
                const double fact = (dist - w->cyl_r) / dist;
                delta[y] = -dy*fact; delta[z] = -dz*fact;
            } else {
                deltan = w->cyl_r - dist - sd.radi;
                const double fact = (w->cyl_r - dist) / dist;
                delta[y] = +dy*fact; delta[z] = +dz*fact;
            }
        } else {        /* Plane<dim>::resolveContact src/primitive_wall_definitions.h:133 */
            delta[w->dim] = w->pos - pos[w->dim];
            if (pos[w->dim] > w->pos) deltan = pos[w->dim] - w->pos - sd.radi;
            else deltan = w->pos - pos[w->dim] - sd.radi;
        }
        if (deltan > s->cutneighmax) continue;
        double *hist = &w->hist[3*ip];
        if (deltan <= 0 || deltan < 0.0*s->radius[ip]) {
            sd.contact_history = hist;
            sd.deltan = -deltan;
            sd.delta[0] = -delta[0]; sd.delta[1] = -delta[1]; sd.delta[2] = -delta[2];
            wall_compute_force(s, ip, &sd, vwall, w->wtype, w->rolling, shearupdate, NULL);
        } else {
            hist[0] = hist[1] = hist[2] = 0.0;
        }
    }
}

/* ------------------------------------------------------------------ */
/* mesh neighbor list: FixNeighlistMesh src/fix_neighlist_mesh.cpp:230-503,
   TriMesh::resolveTriSphereNeighbuild src/tri_mesh_I.h:255-283          */

static double dist_to_plane(const double *p, const double *pPlane, const double *nPlane)
{
    double v[3]; sub3(p, pPlane, v); return dot3(nPlane, v);
}

static int tri_sphere_neighbuild(wall_mesh *m, int t, double rSphere, const double *cSphere, double treshold)
{
    double maxDist = rSphere + treshold;
    double dNorm = fabs(dist_to_plane(cSphere, m->center[t], m->surfnorm[t]));
    if (dNorm > maxDist) return 0;
    double dParaMax = maxDist*maxDist;
    for (int i = 0; i < 3; i++) {
        double d = dist_to_plane(cSphere, m->node[t][i], m->edgenorm[t][i]);
        if (d > 0 && d*d > dParaMax) return 0;
    }
    return 1;
}

static void mesh_bin_bounds(orc_sim *s, wall_mesh *m, int t, int *lo, int *hi)
{
    /* getElementBoundingBoxOnSubdomain + getBinBoundariesFromBoundingBox */
    double blo[3], bhi[3];
    for (int d = 0; d < 3; d++) { blo[d] = BIG; bhi[d] = -BIG; }
    for (int i = 0; i < 3; i++)
        for (int d = 0; d < 3; d++) {
            if (m->node[t][i][d] < blo[d]) blo[d] = m->node[t][i][d];
            if (m->node[t][i][d] > bhi[d]) bhi[d] = m->node[t][i][d];
        }
    for (int d = 0; d < 3; d++) {   /* shrinkToSubbox */
        if (blo[d] < s->boxlo[d]) blo[d] = s->boxlo[d];
        if (bhi[d] > s->boxhi[d]) bhi[d] = s->boxhi[d];
    }
    double delta = m->nl_distmax;
    double tmin[3] = {blo[0]-delta, blo[1]-delta, blo[2]-delta};
    double tmax[3] = {bhi[0]+delta, bhi[1]+delta, bhi[2]+delta};
    coord2bin3(s, tmin, &lo[0], &lo[1], &lo[2]);
    coord2bin3(s, tmax, &hi[0], &hi[1], &hi[2]);
}

static void mesh_neighlist_pre_force(orc_sim *s, wall_mesh *m)
{
    if (!m->build_neighlist_nl) return;
    m->build_neighlist_nl = 0;
    for (int i = 0; i < s->nlocal + s->nghost; i++) m->nneighs[i] = 0;
    double prev_skin = m->nl_skin, prev_distmax = m->nl_distmax;
    double rmax = 0.5*(s->cutneighmax - s->p.skin);
    if (m->moving) {   /* changingMesh src/fix_neighlist_mesh.cpp:252-258 */
        m->nl_skin = s->p.skin;
        m->nl_distmax = s->cutneighmax + m->nl_skin/(70.*M_PI);
    } else {
        m->nl_skin = 0.5*s->p.skin;
        m->nl_distmax = s->cutneighmax - rmax + m->nl_skin/(70.*M_PI);
    }
    if (m->moving) {
        /* handleTriangle with changingMesh: every bin of the current bounding
           box +- distmax, src/fix_neighlist_mesh.cpp:383-395 */
        for (int t = 0; t < m->ntri; t++) {
            m->tri_n[t] = 0;
            if (!s->nlocal) continue;
            int lo[3], hi[3];
            mesh_bin_bounds(s, m, t, lo, hi);
            for (int ix = lo[0]; ix <= hi[0]; ix++)
                for (int iy = lo[1]; iy <= hi[1]; iy++)
                    for (int iz = lo[2]; iz <= hi[2]; iz++) {
                        int iBin = iz*s->mbiny*s->mbinx + iy*s->mbinx + ix;
                        if (iBin < 0 || iBin >= s->mbins) continue;
                        for (int ia = s->binhead[iBin]; ia != -1; ia = s->bins[ia]) {
                            if (tri_sphere_neighbuild(m, t, s->radius[ia]*1.0, &s->x[3*ia], m->nl_skin)) {
                                if (m->tri_n[t] >= m->tri_cap[t]) { m->tri_cap[t] = m->tri_cap[t] ? 2*m->tri_cap[t] : 8; m->tri_list[t] = xrealloc(m->tri_list[t], sizeof(int)*m->tri_cap[t]); }
                                m->tri_list[t][m->tri_n[t]++] = ia;
                                m->nneighs[ia]++;
                            }
                        }
                    }
        }
        m->last_bin_update = s->ntimestep;
        return;
    }
    if (m->nl_skin != prev_skin || m->nl_distmax != prev_distmax || m->last_bin_update < 0) {
        /* generate_bin_list :456 */
        double dx = s->binsizex / 2.0, dy = s->binsizey / 2.0, dz = s->binsizez / 2.0;
        double maxdiag = sqrt(dx * dx + dy * dy + dz * dz);
        for (int t = 0; t < m->ntri; t++) {
            int lo[3], hi[3];
            mesh_bin_bounds(s, m, t, lo, hi);
            m->tri_nbins[t] = 0;
            int cap = 0; free(m->tri_bins[t]); m->tri_bins[t] = NULL;
            for (int ix = lo[0]; ix <= hi[0]; ix++)
                for (int iy = lo[1]; iy <= hi[1]; iy++)
                    for (int iz = lo[2]; iz <= hi[2]; iz++) {
                        int iBin = iz*s->mbiny*s->mbinx + iy*s->mbinx + ix;
                        if (iBin < 0 || iBin >= s->mbins) continue;
                        double center[3];
                        center[0] = (s->mbinxlo + ix + 0.5) * s->binsizex + s->bboxlo[0];
                        center[1] = (s->mbinylo + iy + 0.5) * s->binsizey + s->bboxlo[1];
                        center[2] = (s->mbinzlo + iz + 0.5) * s->binsizez + s->bboxlo[2];
                        if (tri_sphere_neighbuild(m, t, maxdiag, center, m->nl_distmax + m->nl_skin)) {
                            if (m->tri_nbins[t] >= cap) { cap = cap ? 2*cap : 16; m->tri_bins[t] = xrealloc(m->tri_bins[t], sizeof(int)*cap); }
                            m->tri_bins[t][m->tri_nbins[t]++] = iBin;
                        }
                    }
        }
        m->last_bin_update = s->ntimestep;
    }
    for (int t = 0; t < m->ntri; t++) {
        m->tri_n[t] = 0;
        if (!s->nlocal) continue;
        for (int b = 0; b < m->tri_nbins[t]; b++) {
            int iBin = m->tri_bins[t][b];
            for (int ia = s->binhead[iBin]; ia != -1; ia = s->bins[ia]) {
                /* (iAtom > nlocal) && !periodic ghost: every ghost here is periodic */
                if (tri_sphere_neighbuild(m, t, s->radius[ia]*1.0, &s->x[3*ia], m->nl_skin)) {
                    if (m->tri_n[t] >= m->tri_cap[t]) { m->tri_cap[t] = m->tri_cap[t] ? 2*m->tri_cap[t] : 8; m->tri_list[t] = xrealloc(m->tri_list[t], sizeof(int)*m->tri_cap[t]); }
                    m->tri_list[t][m->tri_n[t]++] = ia;
                    m->nneighs[ia]++;
                }
            }
        }
    }
}

/* FixContactHistoryMesh::sort_contacts src/fix_contact_history_mesh.cpp:375 */
static void mesh_swap(wall_mesh *m, int i, int a, int b, int keepswap)
{
    int t = m->partner[i][a]; m->partner[i][a] = m->partner[i][b]; m->partner[i][b] = t;
    double h[3]; memcpy(h, &m->chist[i][3*a], sizeof h);
    memcpy(&m->chist[i][3*a], &m->chist[i][3*b], sizeof h);
    memcpy(&m->chist[i][3*b], h, sizeof h);
    if (keepswap) {
        unsigned char k = m->keep[i][a]; m->keep[i][a] = m->keep[i][b]; m->keep[i][b] = k;
        k = m->isect[i][a]; m->isect[i][a] = m->isect[i][b]; m->isect[i][b] = k;
    }
}

static void mesh_sort_contacts(orc_sim *s, wall_mesh *m)
{
    for (int i = 0; i < s->nlocal; i++) {
        int nn = m->nneighs[i];
        if (0 == nn) continue;
        int fe, lf;
        do {
            fe = lf = -1;
            for (int j = 0; j < nn; j++) {
                if (-1 == fe && -1 == m->partner[i][j]) fe = j;
                if (m->partner[i][j] >= 0) lf = j;
            }
            if (fe > -1 && lf > -1 && fe < lf) mesh_swap(m, i, fe, lf, 1);
        } while (fe > -1 && lf > -1 && fe < lf);
    }
}

static int tri_contains_atom(wall_mesh *m, int t, int i)   /* FixNeighlistMesh::contactInList */
{
    for (int k = 0; k < m->tri_n[t]; k++) if (m->tri_list[t][k] == i) return 1;
    return 0;
}

/* FixContactHistoryMesh::pre_force src/fix_contact_history_mesh.cpp:315-373
   with cleanUpContactJumps :466 */
static void mesh_history_pre_force(orc_sim *s, wall_mesh *m)
{
    if (!m->build_neighlist_ch) return;
    m->build_neighlist_ch = 0;
    const int nl = s->nlocal;
    for (int i = 0; i < nl; i++) {
        int ip = 0;
        while (ip < m->npartner[i]) {
            int tri = m->partner[i][ip];
            if (tri < 0) { fail(s, "mesh history internal error"); return; }
            if (!tri_contains_atom(m, tri, i)) {
                m->partner[i][ip] = -1;
                m->chist[i][3*ip] = m->chist[i][3*ip+1] = m->chist[i][3*ip+2] = 0.0;
                mesh_swap(m, i, ip, m->npartner[i]-1, 0);
                m->npartner[i]--;
            } else ip++;
        }
    }
    for (int i = 0; i < nl; i++) {
        int nn = m->nneighs[i];
        int *np = malloc(sizeof(int)*(nn > 0 ? nn : 1));
        double *nh = calloc((size_t)3*(nn > 0 ? nn : 1), sizeof(double));
        for (int k = 0; k < nn; k++) np[k] = -1;
        if (m->npartner[i] > nn) { fail(s, "mesh history internal error (npartner > nneighs)"); free(np); free(nh); return; }
        for (int k = 0; k < m->npartner[i]; k++) {
            np[k] = m->partner[i][k];
            memcpy(&nh[3*k], &m->chist[i][3*k], sizeof(double)*3);
        }
        free(m->partner[i]); free(m->chist[i]);
        m->partner[i] = np; m->chist[i] = nh;
        free(m->keep[i]); free(m->isect[i]);
        m->keep[i] = calloc(nn > 0 ? nn : 1, 1);
        m->isect[i] = calloc(nn > 0 ? nn : 1, 1);
    }
}

/* ------------------------------------------------------------------ */
/* triangle-sphere narrow phase src/tri_mesh_I.h:65-251                 */

static double calc_dist(const double *cs, const double *cp, double *delta)
{
    sub3(cp, cs, delta);
    double d2 = (cs[0]-cp[0]) * (cs[0]-cp[0]) + (cs[1]-cp[1]) * (cs[1]-cp[1]) + (cs[2]-cp[2]) * (cs[2]-cp[2]);
    return sqrt(d2);
}

static double resolve_edge(wall_mesh *m, int t, int iEdge, const double *p, double *delta, double *bary)
{
    int ip = (iEdge+1)%3, ipp = (iEdge+2)%3;
    double nodeToP[3], d;
    double (*n)[3] = m->node[t];
    sub3(p, n[iEdge], nodeToP);
    double distFromNode = dot3(nodeToP, m->edgevec[t][iEdge]);
    if (distFromNode < -SMALL_TRIMESH) {
        if (!m->corner_active[t][iEdge]) return LARGE_TRIMESH;
        d = calc_dist(p, n[iEdge], delta);
        bary[iEdge] = 1.; bary[ip] = 0.; bary[ipp] = 0.;
    } else if (distFromNode > m->edgelen[t][iEdge] + SMALL_TRIMESH) {
        if (!m->corner_active[t][ip]) return LARGE_TRIMESH;
        d = calc_dist(p, n[ip], delta);
        bary[iEdge] = 0.; bary[ip] = 1.; bary[ipp] = 0.;
    } else {
        double cp[3];
        if (!m->edge_active[t][iEdge]) return LARGE_TRIMESH;
        cp[0] = n[iEdge][0]+distFromNode*m->edgevec[t][iEdge][0];
        cp[1] = n[iEdge][1]+distFromNode*m->edgevec[t][iEdge][1];
        cp[2] = n[iEdge][2]+distFromNode*m->edgevec[t][iEdge][2];
        d = calc_dist(p, cp, delta);
        bary[ipp] = 0.;
        bary[iEdge] = 1. - distFromNode/m->edgelen[t][iEdge];
        bary[ip] = 1. - bary[iEdge];
    }
    return d;
}

static double resolve_corner(wall_mesh *m, int t, int iNode, int obtuse, const double *p, double *delta, double *bary)
{
    int ip = (iNode+1)%3, ipp = (iNode+2)%3;
    const double *n = m->node[t][iNode];
    if (obtuse) {
        double (*edge)[3] = m->edgevec[t];
        double nodeToP[3], cp[3];
        sub3(p, n, nodeToP);
        double distFromNode = dot3(nodeToP, edge[ipp]);
        if (distFromNode < SMALL_TRIMESH) {
            if (distFromNode > -m->edgelen[t][ipp]) {
                if (!m->edge_active[t][ipp]) return LARGE_TRIMESH;
                cp[0] = n[0]+distFromNode*edge[ipp][0]; cp[1] = n[1]+distFromNode*edge[ipp][1]; cp[2] = n[2]+distFromNode*edge[ipp][2];
                bary[ip] = 0.;
                bary[iNode] = 1. + distFromNode/m->edgelen[t][ipp];
                bary[ipp] = 1. - bary[iNode];
                return calc_dist(p, cp, delta);
            } else {
                if (!m->corner_active[t][ipp]) return LARGE_TRIMESH;
                bary[ipp] = 1.; bary[iNode] = bary[ip] = 0.;
                return calc_dist(p, m->node[t][ipp], delta);
            }
        }
        distFromNode = dot3(nodeToP, edge[iNode]);
        if (distFromNode > -SMALL_TRIMESH) {
            if (distFromNode < m->edgelen[t][iNode]) {
                if (!m->edge_active[t][iNode]) return LARGE_TRIMESH;
                cp[0] = n[0]+distFromNode*edge[iNode][0]; cp[1] = n[1]+distFromNode*edge[iNode][1]; cp[2] = n[2]+distFromNode*edge[iNode][2];
                bary[ipp] = 0.;
                bary[iNode] = 1. - distFromNode/m->edgelen[t][iNode];
                bary[ip] = 1. - bary[iNode];
                return calc_dist(p, cp, delta);
            } else {
                if (!m->corner_active[t][ip]) return LARGE_TRIMESH;
                bary[ip] = 1.; bary[iNode] = bary[ipp] = 0.;
                return calc_dist(p, m->node[t][ip], delta);
            }
        }
    }
    if (!m->corner_active[t][iNode]) return LARGE_TRIMESH;
    bary[iNode] = 1.; bary[ip] = bary[ipp] = 0.;
    return calc_dist(p, m->node[t][iNode], delta);
}

static double resolve_tri_sphere(wall_mesh *m, int t, double rSphere, const double *cs, double *delta, double *bary, int *barySign)
{
    int obt = m->obtuse[t];
    bary[0] = bary[1] = bary[2] = 0.;
    double n0ToC[3];
    sub3(cs, m->node[t][0], n0ToC);
    /* calcBaryTriCoords src/math_extra_liggghts.h:559 */
    double a = dot3(n0ToC, m->edgevec[t][0]);
    double b = dot3(n0ToC, m->edgevec[t][2]);
    double c = dot3(m->edgevec[t][0], m->edgevec[t][2]);
    double oneMinCSqr = 1 - c*c;
    bary[1] = (a - b*c)/(m->edgelen[t][0] * oneMinCSqr);
    bary[2] = (a*c - b)/(m->edgelen[t][2] * oneMinCSqr);
    bary[0] = 1. - bary[1] - bary[2];
    double invlen = 1./(2.*m->rbound[t]);
    double prec = m->precision;
    *barySign = (bary[0] > -prec*invlen) + 2*(bary[1] > -prec*invlen) + 4*(bary[2] > -prec*invlen);
    double d = 0.;
    switch (*barySign) {
    case 1: d = resolve_corner(m, t, 0, obt == 0, cs, delta, bary); break;
    case 2: d = resolve_corner(m, t, 1, obt == 1, cs, delta, bary); break;
    case 3: d = resolve_edge(m, t, 0, cs, delta, bary); break;
    case 4: d = resolve_corner(m, t, 2, obt == 2, cs, delta, bary); break;
    case 5: d = resolve_edge(m, t, 2, cs, delta, bary); break;
    case 6: d = resolve_edge(m, t, 1, cs, delta, bary); break;
    case 7: {
        const double *sn = m->surfnorm[t];
        double dNorm = dot3(sn, n0ToC);
        double tmp[3] = {dNorm*sn[0], dNorm*sn[1], dNorm*sn[2]};
        double csPlane[3]; sub3(cs, tmp, csPlane);
        d = calc_dist(cs, csPlane, delta);
        break;
    }
    default: d = 1.; break;
    }
    return d - rSphere;
}

/* ------------------------------------------------------------------ */
/* FixWallGran::post_force_mesh src/fix_wall_gran.cpp:845-1018 with
   FixContactHistoryMesh::handleContact src/fix_contact_history_mesh_I.h:51-216 */

static int mesh_handle_contact(orc_sim *s, wall_mesh *m, int iP, int idTri, double **history, int intersect, int faceflag)
{
    const int nn = m->nneighs[iP];
    for (int i = 0; i < nn; i++)
        if (m->partner[iP][i] == idTri) {
            *history = &m->chist[iP][3*i];
            m->keep[iP][i] = 1; m->isect[iP][i] = (unsigned char)intersect;
            return 1;
        }
    if (faceflag) {   /* coplanarContactAlready */
        for (int i = 0; i < nn; i++) {
            int idp = m->partner[iP][i];
            if (idp >= 0 && idp != idTri && mesh_coplanar_node_neighs(m, idp, idTri))
                if (m->keep[iP][i]) return 0;
        }
    }
    /* addNewTriContactToExistingParticle */
    int ic = -1;
    if (m->npartner[iP] >= nn) { fail(s, "mesh history: npartner >= nneighs"); return 0; }
    for (int k = 0; k < nn; k++) if (-1 == m->partner[iP][k]) { ic = k; break; }
    if (ic < 0) { fail(s, "mesh history: no free slot"); return 0; }
    m->partner[iP][ic] = idTri; m->keep[iP][ic] = 1; m->isect[iP][ic] = (unsigned char)intersect;
    *history = &m->chist[iP][3*ic];
    (*history)[0] = (*history)[1] = (*history)[2] = 0.0;
    m->npartner[iP]++;
    if (faceflag) {   /* checkCoplanarContactHistory */
        for (int i = 0; i < nn; i++) {
            int tri = m->partner[iP][i];
            if (tri >= 0 && tri != idTri && mesh_coplanar_node_neighs(m, tri, idTri))
                memcpy(*history, &m->chist[iP][3*i], sizeof(double)*3);
        }
    }
    return 1;
}

static void mesh_post_force(orc_sim *s, wall_mesh *m, int shearupdate)
{
    const int nl = s->nlocal;
    /* markAllContacts */
    for (int i = 0; i < nl; i++) memset(m->keep[i], 0, m->nneighs[i] > 0 ? m->nneighs[i] : 0);
    const double vwall[3] = {0., 0., 0.};
    for (int t = 0; t < m->ntri; t++) {
        for (int ic = 0; ic < m->tri_n[t]; ic++) {
            const int ip = m->tri_list[t][ic];
            if (ip >= nl) continue;
            double delta[3], bary[3]; int barysign = -1;
            sidata_t sd; memset(&sd, 0, sizeof sd);
            sd.is_wall = 1;
            sd.radi = s->radius[ip];
            double deltan = resolve_tri_sphere(m, t, sd.radi, &s->x[3*ip], delta, bary, &barysign);
            if (deltan > s->cutneighmax) continue;
            int intersectflag = (deltan <= 0);
            if (deltan <= 0 || (deltan < 0.0*s->radius[ip])) {
                double *hist = NULL;
                if (!mesh_handle_contact(s, m, ip, t, &hist, intersectflag, 7 == barysign)) continue;
                double vw[3] = {vwall[0], vwall[1], vwall[2]};
                if (m->moving)   /* barycentric wall velocity src/fix_wall_gran.cpp:992-996 */
                    for (int c = 0; c < 3; c++)
                        vw[c] = (bary[0]*m->vnode[t][0][c] + bary[1]*m->vnode[t][1][c] + bary[2]*m->vnode[t][2][c]);
                sd.deltan = -deltan;
                sd.delta[0] = -delta[0]; sd.delta[1] = -delta[1]; sd.delta[2] = -delta[2];
                sd.contact_history = hist;
                double frc[3];
                wall_compute_force(s, ip, &sd, vw, m->wtype, m->rolling, shearupdate, frc);
                if (m->stress) {   /* MeshModuleStress::add_particle_contribution src/mesh_module_stress.cpp:276-304 */
                    double cp[3], tmp[3], tq[3];
                    for (int c = 0; c < 3; c++) frc[c] = -frc[c];
                    for (int c = 0; c < 3; c++) cp[c] = s->x[3*ip+c] + delta[c];
                    for (int c = 0; c < 3; c++) m->tri_f[t][c] += frc[c];
                    for (int c = 0; c < 3; c++) m->f_total[c] += frc[c];
                    for (int c = 0; c < 3; c++) tmp[c] = cp[c] - m->p_ref[c];
                    tq[0] = tmp[1]*frc[2] - tmp[2]*frc[1];
                    tq[1] = tmp[2]*frc[0] - tmp[0]*frc[2];
                    tq[2] = tmp[0]*frc[1] - tmp[1]*frc[0];
                    for (int c = 0; c < 3; c++) m->torque_total[c] += tq[c];
                    if (m->wear) {   /* wear finnie src/mesh_module_stress.cpp:306-352 */
                        double vr[3], cr[3];
                        const double *sn = m->surfnorm[t];
                        for (int c = 0; c < 3; c++) vr[c] = s->v[3*ip+c] - vw[c];
                        double cdot = delta[0]*vr[0] + delta[1]*vr[1] + delta[2]*vr[2];
                        double vm = sqrt(vr[0]*vr[0] + vr[1]*vr[1] + vr[2]*vr[2]);
                        if (!(cdot < 0.) && !(0.0000001 > vm)) {
                            cross3(vr, sn, cr);
                            double sg = fabs(vr[0]*sn[0] + vr[1]*sn[1] + vr[2]*sn[2]) / vm;
                            double cg = fabs(sqrt(cr[0]*cr[0] + cr[1]*cr[1] + cr[2]*cr[2])) / vm;
                            if (cg > 1.) cg = 1.;
                            if (sg > 1.) sg = 1.;
                            double E;
                            if (cg < 0.0001 || 3.*sg > cg) E = 0.33333 * cg * cg;
                            else E = 2. * sg * cg - 3. * sg * sg;
                            E *= 2.*m->kfin[s->type[ip]] * vm * sqrt(frc[0]*frc[0] + frc[1]*frc[1] + frc[2]*frc[2]);
                            double ev[3];
                            cross3(m->area_ev[t][0], m->area_ev[t][1], ev);
                            double area = 0.5*sqrt(ev[0]*ev[0] + ev[1]*ev[1] + ev[2]*ev[2]) * m->area_el[t][0] * m->area_el[t][1];
                            m->wear[t] += E*s->p.dt / area;
                        }
                    }
                }
            }
        }
    }
    /* cleanUpContacts :437 */
    for (int i = 0; i < nl; i++)
        for (int j = 0; j < m->nneighs[i]; j++)
            if (!m->keep[i][j]) {
                if (m->partner[i][j] > -1) m->npartner[i]--;
                m->partner[i][j] = -1;
                m->isect[i][j] = 0;
                m->chist[i][3*j] = m->chist[i][3*j+1] = m->chist[i][3*j+2] = 0.0;
            }
}

/* ------------------------------------------------------------------ */
/* integrate src/fix_nve_sphere.cpp:138-246                             */

static void nve_initial(orc_sim *s)
{
    const double dtv = s->p.dt, dtf = 0.5 * s->p.dt * 1.0;
    const double dtfrotate = dtf / 0.4;
    for (int i = 0; i < s->nlocal; i++) {
        double dtfm = dtf / (s->rmass[i]*1.0);
        s->v[3*i] += dtfm * s->f[3*i]; s->v[3*i+1] += dtfm * s->f[3*i+1]; s->v[3*i+2] += dtfm * s->f[3*i+2];
        s->x[3*i] += dtv * s->v[3*i]; s->x[3*i+1] += dtv * s->v[3*i+1]; s->x[3*i+2] += dtv * s->v[3*i+2];
        double dtirotate = dtfrotate / (s->radius[i]*s->radius[i]*s->rmass[i]);
        s->omega[3*i] += dtirotate * s->torque[3*i]; s->omega[3*i+1] += dtirotate * s->torque[3*i+1]; s->omega[3*i+2] += dtirotate * s->torque[3*i+2];
    }
}

static void nve_final(orc_sim *s)
{
    const double dtf = 0.5 * s->p.dt * 1.0;
    const double dtfrotate = dtf / 0.4;
    for (int i = 0; i < s->nlocal; i++) {
        double dtfm = dtf / (s->rmass[i]*1.0);
        s->v[3*i] += dtfm * s->f[3*i]; s->v[3*i+1] += dtfm * s->f[3*i+1]; s->v[3*i+2] += dtfm * s->f[3*i+2];
        double dtirotate = dtfrotate / (s->radius[i]*s->radius[i]*s->rmass[i]);
        s->omega[3*i] += dtirotate * s->torque[3*i]; s->omega[3*i+1] += dtirotate * s->torque[3*i+1]; s->omega[3*i+2] += dtirotate * s->torque[3*i+2];
    }
}

static void gravity_post_force(orc_sim *s, fixrec *fr)   /* src/fix_gravity.cpp:301-337 */
{
    for (int i = 0; i < s->nlocal; i++) {
        double massone = s->rmass[i] * 1.;
        s->f[3*i] += massone*fr->xacc; s->f[3*i+1] += massone*fr->yacc; s->f[3*i+2] += massone*fr->zacc;
    }
}

static void force_clear(orc_sim *s)
{
    int nall = s->nlocal + s->nghost;
    memset(s->f, 0, sizeof(double)*3*nall);
    memset(s->torque, 0, sizeof(double)*3*nall);
}

static void post_force_all(orc_sim *s, int shearupdate)
{
    for (int k = 0; k < s->nfix; k++) {
        fixrec *fr = &s->fix[k];
        if (fr->kind == ORC_FIX_GRAVITY) gravity_post_force(s, fr);
        else if (fr->kind == ORC_FIX_WALL_PLANE) wall_plane_post_force(s, fr->wp, shearupdate);
        else if (fr->kind == ORC_FIX_WALL_MESH) mesh_post_force(s, fr->wm, shearupdate);
    }
}

static void pre_force_all(orc_sim *s, int reneigh)
{
    for (int k = 0; k < s->nfix; k++) {
        fixrec *fr = &s->fix[k];
        if (fr->kind == ORC_FIX_WALL_MESH && fr->wm->moving) {
            /* FixMesh::pre_force src/fix_mesh.cpp:564-588 */
            if (reneigh) mesh_refresh_owned(fr->wm);
            else if (mesh_decide_rebuild(s, fr->wm)) fr->wm->next_reneighbor = s->ntimestep + 1;
        }
        if (fr->kind == ORC_FIX_WALL_PLANE) wall_plane_pre_force(s, fr->wp);
        else if (fr->kind == ORC_FIX_WALL_MESH) { mesh_neighlist_pre_force(s, fr->wm); mesh_history_pre_force(s, fr->wm); }
        if (fr->kind == ORC_FIX_WALL_MESH && fr->wm->stress) {
            /* FixMesh::pre_force clearReverse (per-element "f"), MeshModuleStress::pre_force (totals) */
            memset(fr->wm->tri_f, 0, sizeof(double)*3*fr->wm->ntri);
            memset(fr->wm->f_total, 0, sizeof fr->wm->f_total);
            memset(fr->wm->torque_total, 0, sizeof fr->wm->torque_total);
        }
    }
}

static void pre_neighbor_all(orc_sim *s)
{
    for (int k = 0; k < s->nfix; k++) {
        fixrec *fr = &s->fix[k];
        if (fr->kind == ORC_FIX_WALL_PLANE) fr->wp->rebuild = 1;
        else if (fr->kind == ORC_FIX_WALL_MESH) { fr->wm->build_neighlist_nl = 1; fr->wm->build_neighlist_ch = 1; }
    }
}

/* ------------------------------------------------------------------ */
/* fix insert/pack (restated; see the header)                           */

typedef struct { int seed, save; double second; } park_t;

/* RanPark::uniform src/random_park.cpp:56-62 */
static double park_uniform(park_t *r)
{
    int k = r->seed / 127773;
    r->seed = 16807 * (r->seed - k * 127773) - 2836 * k;
    if (r->seed < 0) r->seed += 2147483647;
    return (1.0 / 2147483647) * r->seed;
}

/* RanPark::gaussian src/random_park.cpp:68-91 */
static double park_gaussian(park_t *r)
{
    double first;
    if (!r->save) {
        double v1, v2, rsq;
        int again = 1;
        while (again) {
            v1 = 2.0 * park_uniform(r) - 1.0;
            v2 = 2.0 * park_uniform(r) - 1.0;
            rsq = v1 * v1 + v2 * v2;
            if (rsq < 1.0 && rsq != 0.0) again = 0;
        }
        double fac = sqrt(-2.0 * log(rsq) / rsq);
        r->second = v1 * fac;
        first = v2 * fac;
        r->save = 1;
    } else {
        first = r->second;
        r->save = 0;
    }
    return first;
}

struct ins_state {
    orc_insert_pack p;
    park_t rnd, rreg, rdist, rtmpl[8];
    double rlo[8], rhi[8], h1[8], h2[8];   /* radius pdf bounds, uniform's h1/h2 */
    double distweight[8], tvol[8], tmass[8];
    int distorder[8];
    double volexpect, massexpect, maxrad, maxrbound;
    double region_volume, region_volume_local, insertion_ratio;
    long next_reneighbor, most_recent, ninserted;
    double massinserted;
    int props;
};

/* MathExtraLiggghts::isPrime-style check of Random::Random src/random.cpp:79-95 */
static int seed_valid(int seed)
{
    if (seed < 10000) return 0;
    for (int d = 2; (long)d * d <= seed; d++) if (seed % d == 0) return 0;
    return 1;
}

/* RegBlock::inside src/region_block.cpp:147-152 */
/* RegCylinder: the two coordinates across the axis, in x, y, z order */
static void cyl_axes(const orc_insert_pack *p, int *a1, int *a2)
{
    if (p->cyl_axis == 0) { *a1 = 1; *a2 = 2; }
    else if (p->cyl_axis == 1) { *a1 = 0; *a2 = 2; }
    else { *a1 = 0; *a2 = 1; }
}

static int blk_inside(const orc_insert_pack *p, const double *x)
{
    if (p->region_style == 1) {   /* RegCylinder::inside src/region_cylinder.cpp:213-239 */
        int a1, a2, ax = p->cyl_axis; cyl_axes(p, &a1, &a2);
        double del1 = x[a1] - p->cyl_c1, del2 = x[a2] - p->cyl_c2;
        double dist = sqrt(del1*del1 + del2*del2);
        return dist <= p->cyl_radius && x[ax] >= p->cyl_lo && x[ax] <= p->cyl_hi;
    }
    return x[0] >= p->region_lo[0] && x[0] <= p->region_hi[0] && x[1] >= p->region_lo[1] && x[1] <= p->region_hi[1]
        && x[2] >= p->region_lo[2] && x[2] <= p->region_hi[2];
}

/* RegBlock::surface_interior src/region_block.cpp:161-220 (contact count) */
static int blk_surface_interior(const orc_insert_pack *p, const double *x, double cutoff)
{
    if (p->region_style == 1) {   /* RegCylinder::surface_interior src/region_cylinder.cpp:249-330 */
        int a1, a2, ax = p->cyl_axis; cyl_axes(p, &a1, &a2);
        double del1 = x[a1] - p->cyl_c1, del2 = x[a2] - p->cyl_c2;
        double r = sqrt(del1*del1 + del2*del2);
        if (r > p->cyl_radius || x[ax] < p->cyl_lo || x[ax] > p->cyl_hi) return 0;
        int n = 0;
        if (p->cyl_radius - r < cutoff && r > 0.0) n++;
        if (x[ax] - p->cyl_lo < cutoff) n++;
        if (p->cyl_hi - x[ax] < cutoff) n++;
        return n;
    }
    const double *lo = p->region_lo, *hi = p->region_hi;
    if (x[0] < lo[0] || x[0] > hi[0] || x[1] < lo[1] || x[1] > hi[1] || x[2] < lo[2] || x[2] > hi[2]) return 0;
    int n = 0;
    for (int d = 0; d < 3; d++) {
        if (x[d] - lo[d] < cutoff) n++;
        if (hi[d] - x[d] < cutoff) n++;
    }
    return n;
}

/* RegBlock::surface_exterior src/region_block.cpp:228-259 with Region::add_contact src/region.cpp:248-257 */
static int blk_surface_exterior(const orc_insert_pack *p, const double *x, double cutoff)
{
    if (p->region_style == 1) {   /* RegCylinder::surface_exterior src/region_cylinder.cpp:338-470 */
        int a1, a2, ax = p->cyl_axis; cyl_axes(p, &a1, &a2);
        double del1 = x[a1] - p->cyl_c1, del2 = x[a2] - p->cyl_c2;
        double r = sqrt(del1*del1 + del2*del2);
        const double R = p->cyl_radius, lo = p->cyl_lo, hi = p->cyl_hi;
        if (r >= R+cutoff || x[ax] <= lo-cutoff || x[ax] >= hi+cutoff) return 0;
        if (r < R && x[ax] > lo && x[ax] < hi) return 0;
        double q[3];
        if (r > R) { q[a1] = p->cyl_c1 + del1*R/r; q[a2] = p->cyl_c2 + del2*R/r; }
        else { q[a1] = x[a1]; q[a2] = x[a2]; }
        if (x[ax] < lo) q[ax] = lo; else if (x[ax] > hi) q[ax] = hi; else q[ax] = x[ax];
        double delx = x[0] - q[0], dely = x[1] - q[1], delz = x[2] - q[2];
        return sqrt(delx*delx + dely*dely + delz*delz) < cutoff;
    }
    const double *lo = p->region_lo, *hi = p->region_hi;
    if (x[0] <= lo[0]-cutoff || x[0] >= hi[0]+cutoff || x[1] <= lo[1]-cutoff || x[1] >= hi[1]+cutoff ||
        x[2] <= lo[2]-cutoff || x[2] >= hi[2]+cutoff) return 0;
    if (x[0] > lo[0] && x[0] < hi[0] && x[1] > lo[1] && x[1] < hi[1] && x[2] > lo[2] && x[2] < hi[2]) return 0;
    double xp, yp, zp;
    if (x[0] < lo[0]) xp = lo[0]; else if (x[0] > hi[0]) xp = hi[0]; else xp = x[0];
    if (x[1] < lo[1]) yp = lo[1]; else if (x[1] > hi[1]) yp = hi[1]; else yp = x[1];
    if (x[2] < lo[2]) zp = lo[2]; else if (x[2] > hi[2]) zp = hi[2]; else zp = x[2];
    double delx = x[0] - xp, dely = x[1] - yp, delz = x[2] - zp;
    double r = sqrt(delx*delx + dely*dely + delz*delz);
    return r < cutoff;
}

static void ins_max_rad(const struct ins_state *I, int type, double *mx)
{
    double m = 0.;
    for (int i = 0; i < I->p.ntemplates; i++)
        if (I->p.tmpl_type[i] == type && I->rhi[i] > m) m = I->rhi[i];   /* pdf_max(pdf_radius) */
    *mx = m;
}

int orc_add_insert_pack(orc_sim *s, const orc_insert_pack *p)
{
    if (s->ins) { fail(s, "one fix insert/pack"); return -1; }
    if (!seed_valid(p->seed) || !seed_valid(p->dist_seed)) { fail(s, "seeds must be primes > 10000"); return -1; }
    if (p->ntemplates < 1 || p->ntemplates > 8) { fail(s, "illegal number of templates"); return -1; }
    int ndef = (p->volumefraction_region > 0.) + (p->particles_in_region > 0) + (p->mass_in_region > 0.);
    if (ndef != 1) { fail(s, "exactly one insertion target"); return -1; }
    struct ins_state *I = calloc(1, sizeof *I);
    I->p = *p;
    if (p->region_style == 1) {   /* RegCylinder extents (bounding box) src/region_cylinder.cpp:159-183 */
        int a1, a2, ax = p->cyl_axis; cyl_axes(p, &a1, &a2);
        I->p.region_lo[ax] = p->cyl_lo; I->p.region_hi[ax] = p->cyl_hi;
        I->p.region_lo[a1] = p->cyl_c1 - p->cyl_radius; I->p.region_hi[a1] = p->cyl_c1 + p->cyl_radius;
        I->p.region_lo[a2] = p->cyl_c2 - p->cyl_radius; I->p.region_hi[a2] = p->cyl_c2 + p->cyl_radius;
    }
    const int nt = p->ntemplates;
    /* FixTemplateSphere: cubic_expectancy(radius)*4.*M_PI/3., density * volume (src/fix_template_sphere.cpp:244-245) */
    for (int i = 0; i < nt; i++) {
        double mu = p->tmpl_radius[i], s2 = p->tmpl_radius2[i], ce;
        if (!seed_valid(p->tmpl_seed[i])) { free(I); fail(s, "template seed"); return -1; }
        I->rtmpl[i].seed = p->tmpl_seed[i];
        /* PDF::set_params and cubic_expectancy_value, src/probability_distribution.h:120-200 */
        if (p->tmpl_radius_style[i] == 1) {
            I->rlo[i] = mu; I->rhi[i] = s2;
            I->h1[i] = 2./(1./(mu*mu)-1./(s2*s2));
            I->h2[i] = I->h1[i]/(2.*mu*mu);
            ce = 0.25*(s2*s2*s2 + s2*s2*mu + s2*mu*mu + mu*mu*mu);
        } else if (p->tmpl_radius_style[i] == 2) {
            I->rlo[i] = mu-3.*s2; I->rhi[i] = mu+3.*s2;
            ce = mu*(mu*mu+3*s2*s2);
        } else {
            I->rlo[i] = I->rhi[i] = mu;
            ce = mu*mu*mu;
        }
        I->tvol[i] = ce*4.*M_PI/3.;
        I->tmass[i] = p->tmpl_density[i] * I->tvol[i];
        I->distweight[i] = p->tmpl_weight[i];
    }
    /* FixParticledistributionDiscrete constructor src/fix_particledistribution_discrete.cpp:130-220 */
    double wsum = 0;
    for (int i = 0; i < nt; i++) wsum += I->distweight[i];
    for (int i = 0; i < nt; i++) I->distweight[i] /= wsum;
    if (p->dist_mass_based) {
        for (int i = 0; i < nt; i++) I->distweight[i] = I->distweight[i] / I->tmass[i];
        wsum = 0;
        for (int i = 0; i < nt; i++) wsum += I->distweight[i];
        for (int i = 0; i < nt; i++) I->distweight[i] /= wsum;
    }
    I->volexpect = 0.; I->massexpect = 0.;
    for (int i = 0; i < nt; i++) {
        I->volexpect += I->tvol[i] * I->distweight[i];
        I->massexpect += I->tmass[i] * I->distweight[i];
    }
    for (int i = 0; i < nt; i++) I->distorder[i] = i;
    int swaped, n = nt;
    do {
        swaped = 0;
        for (int i = 0; i < nt-1; i++)
            if (I->tvol[I->distorder[i]] < I->tvol[I->distorder[i+1]]) {
                int tmp = I->distorder[i]; I->distorder[i] = I->distorder[i+1]; I->distorder[i+1] = tmp;
                swaped = 1;
            }
        n--;
    } while (swaped && n > 0);
    I->maxrbound = 0.;
    for (int i = 0; i < nt; i++) if (I->rhi[i] > I->maxrbound) I->maxrbound = I->rhi[i];
    I->maxrad = 0.;
    for (int t = 1; t <= s->ntypes; t++) { double m; ins_max_rad(I, t, &m); if (m > I->maxrad) I->maxrad = m; }
    I->rnd.seed = p->seed;
    I->rdist.seed = p->dist_seed;
    I->next_reneighbor = p->start > 0 ? p->start : s->ntimestep + 1;
    I->most_recent = -1;
    s->ins = I;
    return 0;
}

static long ins_next(const struct ins_state *I) { return I->next_reneighbor; }

/* state of the Park-Miller generator after n uniform() draws from seed */
int orc_park_after(int seed, int n)
{
    park_t r = {seed, 0, 0.};
    for (int i = 0; i < n; i++) park_uniform(&r);
    return r.seed;
}

int orc_insert_stats(orc_sim *s, long *ninserted, double *massinserted, long *next_step)
{
    if (!s->ins) return -1;
    *ninserted = s->ins->ninserted;
    *massinserted = s->ins->massinserted;
    *next_step = s->ins->next_reneighbor;
    return 0;
}

/* FixInsertPack::calc_insertion_properties with Region::volume_mc src/region.cpp:634-703 */
static void ins_setup(orc_sim *s)
{
    struct ins_state *I = s->ins;
    if (I->props) return;
    I->props = 1;
    I->rreg.seed = I->p.seed + 12; I->rreg.save = 0;
    const double *lo = I->p.region_lo, *hi = I->p.region_hi;
    int n_in_global = 0, n_in_local = 0;
    for (int i = 0; i < I->p.ntry_mc; i++) {
        double pos[3];
        pos[0] = lo[0] + park_uniform(&I->rreg) * (hi[0] - lo[0]);
        pos[1] = lo[1] + park_uniform(&I->rreg) * (hi[1] - lo[1]);
        pos[2] = lo[2] + park_uniform(&I->rreg) * (hi[2] - lo[2]);
        int in_domain = pos[0] >= s->p.boxlo[0] && pos[0] <= s->p.boxhi[0] && pos[1] >= s->p.boxlo[1] &&
                        pos[1] <= s->p.boxhi[1] && pos[2] >= s->p.boxlo[2] && pos[2] <= s->p.boxhi[2];
        if (!in_domain) continue;
        if (!I->p.all_in) {
            if (blk_inside(&I->p, pos)) { n_in_global++; n_in_local++; }
        } else {
            if (blk_inside(&I->p, pos)) {
                n_in_global++;
                if (!blk_surface_interior(&I->p, pos, I->maxrbound)) n_in_local++;
            }
        }
    }
    if (n_in_global == 0) { fail(s, "Unable to calculate region volume"); return; }
    double vol_bbox = (hi[0]-lo[0]) * (hi[1]-lo[1]) * (hi[2]-lo[2]);
    double vol_global = (double)n_in_global / (double)(I->p.ntry_mc * 1) * vol_bbox;
    double vol_local = (double)n_in_local / (double)I->p.ntry_mc * vol_bbox;
    double vol_local_all = vol_local;
    if (vol_local_all < 1.e-10) { fail(s, "Unable to calculate region volume"); return; }
    vol_local *= (vol_global / vol_local_all);
    I->region_volume = vol_global;
    I->region_volume_local = vol_local;
    if (I->region_volume <= 0. || I->region_volume_local < 0. ||
        (I->region_volume_local - I->region_volume) / I->region_volume > 1e-3)
        fail(s, "Fix insert: Region volume calculation with MC failed");
}

/* Region::generate_random(_shrinkby_cut) src/region.cpp:531-573, subdomain = box */
static int ins_random_pos(orc_sim *s, struct ins_state *I, double rbound, double *pos)
{
    const orc_insert_pack *p = &I->p;
    double lo[3], hi[3], diff[3];
    for (int d = 0; d < 3; d++) {
        lo[d] = p->region_lo[d] > s->p.boxlo[d] ? p->region_lo[d] : s->p.boxlo[d];
        hi[d] = p->region_hi[d] < s->p.boxhi[d] ? p->region_hi[d] : s->p.boxhi[d];
        diff[d] = hi[d] - lo[d];
    }
    if (p->all_in) {
        for (int d = 0; d < 3; d++) if (p->region_hi[d] - p->region_lo[d] < 2.*rbound) return -1;
        do {
            pos[0] = lo[0] + park_uniform(&I->rreg)*diff[0];
            pos[1] = lo[1] + park_uniform(&I->rreg)*diff[1];
            pos[2] = lo[2] + park_uniform(&I->rreg)*diff[2];
        } while (!blk_inside(p, pos) || blk_surface_interior(p, pos, rbound));
    } else {
        do {
            pos[0] = lo[0] + park_uniform(&I->rreg)*diff[0];
            pos[1] = lo[1] + park_uniform(&I->rreg)*diff[1];
            pos[2] = lo[2] + park_uniform(&I->rreg)*diff[2];
        } while (!blk_inside(p, pos));
    }
    return 0;
}

/* FixInsert::generate_random_velocity src/fix_insert.cpp:956-972 */
static void ins_velocity(struct ins_state *I, double *v)
{
    const orc_insert_pack *p = &I->p;
    v[0] = p->vel[0]; v[1] = p->vel[1]; v[2] = p->vel[2];
    if (p->vel_style == 1) {
        v[0] = p->vel[0] + p->vel_fluct[0] * 2.0 * (park_uniform(&I->rnd)-0.50);
        v[1] = p->vel[1] + p->vel_fluct[1] * 2.0 * (park_uniform(&I->rnd)-0.50);
        v[2] = p->vel[2] + p->vel_fluct[2] * 2.0 * (park_uniform(&I->rnd)-0.50);
    } else if (p->vel_style == 2) {
        v[0] = p->vel[0] + p->vel_fluct[0] * park_gaussian(&I->rnd);
        v[1] = p->vel[1] + p->vel_fluct[1] * park_gaussian(&I->rnd);
        v[2] = p->vel[2] + p->vel_fluct[2] * park_gaussian(&I->rnd);
    }
}

/* Domain::dist_subbox_borders src/domain_I.h:126-142 (subdomain = box) */
static double ins_dist_borders(orc_sim *s, const double *pos)
{
    double dl[3], dh[3];
    for (int d = 0; d < 3; d++) { dl[d] = fabs(s->p.boxlo[d] - pos[d]); dh[d] = fabs(s->p.boxhi[d] - pos[d]); }
    double dlo = dl[0], dhi = dh[0];
    for (int d = 1; d < 3; d++) { if (dl[d] < dlo) dlo = dl[d]; if (dh[d] < dhi) dhi = dh[d]; }
    return dlo < dhi ? dlo : dhi;
}

/* FixInsert::pre_exchange src/fix_insert.cpp:652-827 for fix insert/pack on
   one process; appends the new atoms after the owned ones (in the first
   ghost slots, as Atom::avec->create_atom does, after the contact histories
   were packed) with tags from tag_extend */
static void ins_pre_exchange(orc_sim *s)
{
    struct ins_state *I = s->ins;
    const orc_insert_pack *p = &I->p;
    if (I->next_reneighbor != s->ntimestep || I->most_recent == s->ntimestep) return;
    I->most_recent = s->ntimestep;
    /* FixInsertPack::calc_ninsert_this src/fix_insert_pack.cpp:254-351 */
    int np_region = 0;
    double vol_region = 0., mass_region = 0.;
    double _4Pi3 = 4.*M_PI/3.;
    for (int i = 0; i < s->nlocal; i++)
        if (blk_inside(p, &s->x[3*i])) {
            np_region++;
            vol_region += _4Pi3*s->radius[i]*s->radius[i]*s->radius[i];
            mass_region += s->rmass[i];
        }
    int ninsert_this;
    if (p->volumefraction_region > 0.) {
        ninsert_this = (int)((p->volumefraction_region*I->region_volume - vol_region) / I->volexpect + park_uniform(&I->rnd));
        I->insertion_ratio = vol_region / (p->volumefraction_region*I->region_volume);
    } else if (p->particles_in_region > 0) {
        ninsert_this = p->particles_in_region - np_region;
        I->insertion_ratio = (double)np_region / (double)p->particles_in_region;
    } else {
        ninsert_this = (int)((p->mass_in_region - mass_region) / I->massexpect + park_uniform(&I->rnd));
        I->insertion_ratio = mass_region / p->mass_in_region;
    }
    if (ninsert_this < 0) ninsert_this = 0;
    if (I->insertion_ratio < 0.) I->insertion_ratio = 0.;
    if (I->insertion_ratio > 1.) I->insertion_ratio = 1.;
    /* distribute_ninsert_this src/fix_insert.cpp:829-914, nprocs = 1 */
    double fraction_local = I->region_volume_local / I->region_volume;
    int nloc;
    if (!p->exact_number) nloc = (int)(fraction_local*(double)ninsert_this + park_uniform(&I->rnd));
    else {
        double fr = fraction_local;
        if (fr < 0.02 / 1.) fr = 0.;
        double sum = 0. + fr;
        if (sum == 0.) { fail(s, "Internal error distributing particles to processes"); return; }
        fr /= sum;
        nloc = (int)(fr*(double)ninsert_this);
        double rem = fr*(double)ninsert_this - nloc;
        int ngap = (int)round(rem);
        for (int g = 0; g < ngap; g++) { park_uniform(&I->rnd); nloc++; }
    }
    /* randomize_list src/fix_particledistribution_discrete.cpp:398-480 */
    const int nt = p->ntemplates;
    int parttogen[8];
    if (!p->exact_number) {
        for (int i = 0; i < nt; i++) parttogen[i] = (int)((double)nloc*I->distweight[i] + park_uniform(&I->rdist));
    } else {
        int ntrunc = 0; double remainder[8];
        for (int i = 0; i < nt; i++) {
            parttogen[i] = (int)((double)nloc*I->distweight[i]);
            ntrunc += parttogen[i];
            remainder[i] = (double)nloc*I->distweight[i] - (double)parttogen[i];
        }
        int gap = nloc - ntrunc;
        for (int i = 0; i < gap; i++) {
            double r = park_uniform(&I->rdist) * (double)gap;
            int j = 0; double rsum = remainder[0];
            while (rsum < r && j < nt-1) { j++; rsum += remainder[j]; }
            parttogen[j]++;
        }
    }
    int ntot = 0;
    for (int i = 0; i < nt; i++) ntot += parttogen[i];
    if (ntot == 0) {
        if (p->insert_every) I->next_reneighbor += p->insert_every;
        else I->next_reneighbor = -1;
        return;
    }
    /* FixTemplateSphere::randomize_ptilist (src/fix_template_sphere.cpp:333-361), template by template */
    double *trad = malloc(sizeof(double)*ntot);
    int *tstart = calloc(nt + 1, sizeof(int));
    for (int i = 0; i < nt; i++) tstart[i+1] = tstart[i] + parttogen[i];
    for (int i = 0; i < nt; i++)
        for (int j = 0; j < parttogen[i]; j++) {
            double r = p->tmpl_radius[i];
            if (p->tmpl_radius_style[i] == 1) {
                double rn = park_uniform(&I->rtmpl[i]);
                r = sqrt(I->h1[i]/(2.*(I->h2[i]-rn)));
            } else if (p->tmpl_radius_style[i] == 2) {
                do r = p->tmpl_radius[i] + park_gaussian(&I->rtmpl[i]) * p->tmpl_radius2[i];
                while (r < I->rlo[i] || r > I->rhi[i]);
            }
            trad[tstart[i] + j] = r;
        }
    int *plist = malloc(sizeof(int)*ntot), q = 0;
    double *prad = malloc(sizeof(double)*ntot);
    for (int i = 0; i < nt; i++)
        for (int j = 0; j < parttogen[I->distorder[i]]; j++) {
            prad[q] = trad[tstart[I->distorder[i]] + j];
            plist[q++] = I->distorder[i];
        }
    free(trad); free(tstart);
    /* load_xnear src/fix_insert.cpp:916-954: owned and ghost atoms near the region, within getBoundingBox */
    const int nall = s->nlocal + s->nghost;
    double *near = malloc(sizeof(double)*4*(nall + ntot + 1));
    int nnear = 0;
    if (p->overlapcheck) {
        double blo[3], bhi[3];
        for (int d = 0; d < 3; d++) {
            blo[d] = p->region_lo[d]; bhi[d] = p->region_hi[d];
            if (blo[d] < s->p.boxlo[d]) blo[d] = s->p.boxlo[d];
            if (bhi[d] > s->p.boxhi[d]) bhi[d] = s->p.boxhi[d];
            blo[d] = blo[d] - (2*I->maxrad + 0.);
            bhi[d] = bhi[d] + (2*I->maxrad + 0.);
        }
        for (int i = 0; i < nall; i++) {
            const double *xi = &s->x[3*i];
            double cut = p->all_in ? I->maxrad : s->radius[i] + I->maxrad;
            int nearby = blk_inside(p, xi) || blk_surface_exterior(p, xi, cut);
            int inbb = xi[0] >= blo[0] && xi[0] <= bhi[0] && xi[1] >= blo[1] && xi[1] <= bhi[1] && xi[2] >= blo[2] && xi[2] <= bhi[2];
            if (nearby && inbb) {
                near[4*nnear] = xi[0]; near[4*nnear+1] = xi[1]; near[4*nnear+2] = xi[2]; near[4*nnear+3] = s->radius[i];
                nnear++;
            }
        }
    }
    /* x_v_omega src/fix_insert_pack.cpp:415-514 */
    double *nx = malloc(sizeof(double)*9*ntot);
    int *nty = malloc(sizeof(int)*ntot);
    double *nr = malloc(sizeof(double)*ntot), *nm = malloc(sizeof(double)*ntot);
    int done = 0, ntry = 0;
    int maxtry = I->insertion_ratio >= 1. ? ntot*p->maxattempt : (int)((double)(ntot*p->maxattempt) / (1.-I->insertion_ratio));
    double mass_this = 0.;
    while (done < ntot && (!p->overlapcheck || ntry < maxtry)) {
        int t = plist[done];
        double rb = prad[done];
        double pos[3], v[3];
        int ok = 0;
        if (!p->overlapcheck) {
            if (ins_random_pos(s, I, rb, pos)) { fail(s, "region too small"); break; }
            ins_velocity(I, v);
            if (pos[0] == 0. && pos[1] == 0. && pos[2] == 0.) { fail(s, "illegal position"); break; }
            ok = 1;
        } else {
            while (!ok && ntry < maxtry) {
                do {
                    if (ins_random_pos(s, I, rb, pos)) { fail(s, "region too small"); goto out; }
                    ntry++;
                } while (p->check_dist_from_subdomain_border && ntry < maxtry && ins_dist_borders(s, pos) < rb);
                if (ntry == maxtry) break;
                ins_velocity(I, v);
                int hit = 0;
                for (int k = 0; k < nnear && !hit; k++) {
                    double del[3] = {pos[0]-near[4*k], pos[1]-near[4*k+1], pos[2]-near[4*k+2]};
                    double rsq = del[0]*del[0] + del[1]*del[1] + del[2]*del[2];
                    double radsum = rb + near[4*k+3];
                    if (rsq <= radsum*radsum) hit = 1;
                }
                if (!hit) {
                    near[4*nnear] = pos[0]; near[4*nnear+1] = pos[1]; near[4*nnear+2] = pos[2]; near[4*nnear+3] = rb;
                    nnear++;
                    ok = 1;
                }
            }
        }
        if (!ok) break;
        for (int d = 0; d < 3; d++) { nx[9*done+d] = pos[d]; nx[9*done+3+d] = v[d]; nx[9*done+6+d] = p->omega[d]; }
        nty[done] = p->tmpl_type[t];
        nr[done] = rb;
        nm[done] = p->tmpl_density[t] * (rb*rb*rb*4.*M_PI/3.);
        mass_this += nm[done];
        done++;
    }
out:
    if (!s->err[0] && done > 0) {
        /* ParticleToInsert::insert src/particleToInsert.cpp:101-158 and Atom::tag_extend */
        int maxtag = 0;
        for (int i = 0; i < s->nlocal; i++) if (s->tag[i] > maxtag) maxtag = s->tag[i];
        const int nl = s->nlocal;
        if (nl + done > s->nmax) grow_all(s, 2*(nl + done) + 64);
        for (int k = 0; k < done; k++) {
            int m = nl + k;
            memcpy(&s->x[3*m], &nx[9*k], sizeof(double)*3);
            memcpy(&s->v[3*m], &nx[9*k+3], sizeof(double)*3);
            memcpy(&s->omega[3*m], &nx[9*k+6], sizeof(double)*3);
            s->radius[m] = nr[k]; s->rmass[m] = nm[k]; s->type[m] = nty[k];
            s->tag[m] = maxtag + 1 + k;
            s->f[3*m] = s->f[3*m+1] = s->f[3*m+2] = 0.;
            s->torque[3*m] = s->torque[3*m+1] = s->torque[3*m+2] = 0.;
            free(s->partner[m]); free(s->phist[m]); s->partner[m] = NULL; s->phist[m] = NULL; s->npartner[m] = 0;
            for (int f = 0; f < s->nfix; f++) {
                if (s->fix[f].wp) { double *h = s->fix[f].wp->hist; h[3*m] = h[3*m+1] = h[3*m+2] = 0.; }
                if (s->fix[f].wm) {
                    wall_mesh *wm = s->fix[f].wm;
                    wm->nneighs[m] = 0; wm->npartner[m] = 0;
                    free(wm->partner[m]); free(wm->chist[m]); free(wm->keep[m]); free(wm->isect[m]);
                    wm->partner[m] = NULL; wm->chist[m] = NULL; wm->keep[m] = NULL; wm->isect[m] = NULL;
                }
            }
        }
        s->nlocal = nl + done;
        s->nstart = xrealloc(s->nstart, sizeof(int)*s->nlocal);
        s->nnum = xrealloc(s->nnum, sizeof(int)*s->nlocal);
        for (int k = nl; k < s->nlocal; k++) { s->nstart[k] = 0; s->nnum[k] = 0; }
        I->ninserted += done;
        I->massinserted += mass_this;
    }
    free(plist); free(prad); free(near); free(nx); free(nty); free(nr); free(nm);
    if (s->err[0]) return;
    if (p->insert_every) I->next_reneighbor += p->insert_every;
    else I->next_reneighbor = 0;
}

/* ------------------------------------------------------------------ */
/* Verlet::setup src/verlet.cpp:134-197                                 */

int orc_setup(orc_sim *s)
{
    s->setupflag = 1;
    grow_all(s, 4*s->nlocal + 64);
    for (int i = 0; i < s->nlocal; i++)
        if (s->radius[i] == 0.0) { fail(s, "Fix nve/sphere requires extended particles"); return -1; }
    neighbor_init(s);
    if (s->p.sortfreq > 0) setup_sort_bins(s);
    /* setup_pre_exchange: FixContactHistory only if computeflag; mesh sort */
    if (s->computeflag) history_pre_exchange(s);
    for (int k = 0; k < s->nfix; k++) if (s->fix[k].wm) mesh_sort_contacts(s, s->fix[k].wm);
    domain_pbc(s);
    setup_bins(s);
    if (comm_exchange_check(s)) return -1;
    if (s->p.sortfreq > 0) atom_sort(s);
    comm_borders(s);
    pre_neighbor_all(s);
    neighbor_build(s);
    force_clear(s);
    pre_force_all(s, 1);
    pair_compute(s, 0);
    post_force_all(s, 0);
    if (s->ins) ins_setup(s);   /* FixInsert::setup */
    s->setupflag = 0;
    return s->err[0] ? -1 : 0;
}

/* Verlet::run src/verlet.cpp:264-388 */
int orc_run(orc_sim *s, int nsteps)
{
    for (int step = 0; step < nsteps; step++) {
        s->ntimestep++;
        nve_initial(s);
        for (int k = 0; k < s->nfix; k++)
            if (s->fix[k].kind == ORC_FIX_MOVE_MESH) {
                wall_mesh *mm = s->fix[s->fix[k].imesh].wm;
                if (mm->moving == 2) move_mesh_linear(s, mm);
                else move_mesh_rotate(s, mm);
            }
        int nflag = neighbor_decide(s);
        if (nflag == 0) comm_forward(s);
        else {
            /* Modify::list_init_pre_exchange (src/modify.cpp:1342-1367) calls the
               contact-history fixes first: histories are packed with the ghost
               tags of the last build, then fix insert appends its atoms */
            history_pre_exchange(s);
            for (int k = 0; k < s->nfix; k++) if (s->fix[k].wm) mesh_sort_contacts(s, s->fix[k].wm);
            if (s->ins) { ins_pre_exchange(s); if (s->err[0]) return -1; }
            domain_pbc(s);
            if (comm_exchange_check(s)) return -1;
            if (s->p.sortfreq > 0 && s->ntimestep >= s->nextsort) atom_sort(s);
            comm_borders(s);
            pre_neighbor_all(s);
            neighbor_build(s);
        }
        force_clear(s);
        pre_force_all(s, nflag);
        pair_compute(s, 1);
        post_force_all(s, 1);
        nve_final(s);
        if (s->err[0]) return -1;
    }
    return 0;
}

/* ------------------------------------------------------------------ */
/* accessors                                                            */

void orc_get_atoms(orc_sim *s, double *x, double *v, double *omega, double *f, double *torque, int *tag)
{
    int n = s->nlocal;
    if (x) memcpy(x, s->x, sizeof(double)*3*n);
    if (v) memcpy(v, s->v, sizeof(double)*3*n);
    if (omega) memcpy(omega, s->omega, sizeof(double)*3*n);
    if (f) memcpy(f, s->f, sizeof(double)*3*n);
    if (torque) memcpy(torque, s->torque, sizeof(double)*3*n);
    if (tag) memcpy(tag, s->tag, sizeof(int)*n);
}

void orc_get_radius_mass(orc_sim *s, double *radius, double *rmass)
{
    memcpy(radius, s->radius, sizeof(double)*s->nlocal);
    memcpy(rmass, s->rmass, sizeof(double)*s->nlocal);
}

int orc_get_pairs(orc_sim *s, int cap, int *tag_i, int *tag_j, int *flag, double *hist)
{
    int k = 0;
    for (int i = 0; i < s->nlocal; i++)
        for (int jj = 0; jj < s->nnum[i]; jj++) {
            int e = s->nstart[i] + jj;
            if (k < cap) {
                if (tag_i) tag_i[k] = s->tag[i];
                if (tag_j) tag_j[k] = s->tag[s->nbr[e]];
                if (flag) flag[k] = s->flag[e];
                if (hist) memcpy(&hist[3*k], &s->hist[3*e], sizeof(double)*3);
            }
            k++;
        }
    return k;
}

/* Domain::remap, src/domain.cpp:1136-1173 (orthogonal box) */
static double pgl_remap(const orc_sim *s, int d, double x)
{
    if (!s->p.periodic[d]) return x;
    const double lo = s->p.boxlo[d], hi = s->p.boxhi[d], prd = hi - lo;
    while (x < lo) x += prd;
    while (x >= hi) x -= prd;
    return x > lo ? x : lo;
}

/* component of c along the unit vector x_j - x_i, as add_pair builds
   force_normal / torque_normal (src/compute_pair_gran_local.cpp:481-545 with
   vectorNormalize3D, src/vector_liggghts.h:62-69) */
static void pgl_along(const double *xi, const double *xj, const double *c, double *out)
{
    double n[3] = {xj[0] - xi[0], xj[1] - xi[1], xj[2] - xi[2]};
    const double norm = sqrt(n[0]*n[0] + n[1]*n[1] + n[2]*n[2]);
    const double inv = (norm == 0.) ? 0. : 1. / norm;
    n[0] *= inv; n[1] *= inv; n[2] *= inv;
    const double mag = c[0]*n[0] + c[1]*n[1] + c[2]*n[2];
    out[0] = mag * n[0]; out[1] = mag * n[1]; out[2] = mag * n[2];
}

static int pgl_ncols(unsigned keys)
{
    static const int width[13] = {6, 6, 3, 3, 3, 3, 3, 3, 3, 3, 1, 1, 3};
    int n = 0;
    for (int b = 0; b < 13; b++) if (keys & (1u << b)) n += width[b];
    return n;
}

/* compute pair/gran/local (src/compute_pair_gran_local.cpp add_pair,
   :417-609, fed by PairGran::compute_pgl, src/pair_gran.cpp:676-707:
   computeflag 0, shearupdate 0, add_pair for every touching pair, newton
   off: a pair with a ghost is kept only when tag_i > tag_j).  Columns in
   add_pair's order for the keyword bits set in keys.  Returns the row count. */
int orc_pair_gran_local(orc_sim *s, unsigned keys, int cap, double *rows)
{
    const int nc = pgl_ncols(keys);
    int k = 0;
    for (int i = 0; i < s->nlocal; i++) {
        const double xtmp = s->x[3*i], ytmp = s->x[3*i+1], ztmp = s->x[3*i+2];
        const double radi = s->radius[i];
        for (int jj = 0; jj < s->nnum[i]; jj++) {
            const int e = s->nstart[i] + jj;
            const int j = s->nbr[e];
            const double delx = xtmp - s->x[3*j], dely = ytmp - s->x[3*j+1], delz = ztmp - s->x[3*j+2];
            const double rsq = delx * delx + dely * dely + delz * delz;
            const double radj = s->radius[j];
            const double radsum = radi + radj;
            if (!(rsq < radsum * radsum)) continue;
            if (j >= s->nlocal && s->tag[i] <= s->tag[j]) continue;
            sidata_t sd; memset(&sd, 0, sizeof sd);
            force_t fi, fj; memset(&fi, 0, sizeof fi); memset(&fj, 0, sizeof fj);
            int flag = s->flag[e];
            double hist[3] = {s->hist[3*e], s->hist[3*e+1], s->hist[3*e+2]};
            sd.is_wall = 0;
            sd.radi = radi; sd.radj = radj; sd.radsum = radsum; sd.rsq = rsq;
            sd.delta[0] = delx; sd.delta[1] = dely; sd.delta[2] = delz;
            sd.contact_flags = &flag;
            sd.contact_history = hist;
            sd.v_i = &s->v[3*i]; sd.v_j = &s->v[3*j];
            sd.itype = s->type[i]; sd.jtype = s->type[j];
            sd.computeflag = 0; sd.shearupdate = 0;
            const double r = sqrt(rsq);
            const double rinv = 1.0 / r;
            const double mi = s->rmass[i], mj = s->rmass[j];
            const double meff = mi * mj / (mi + mj);
            sd.r = r; sd.rinv = rinv; sd.meff = meff; sd.mi = mi; sd.mj = mj;
            sd.en[0] = delx * rinv; sd.en[1] = dely * rinv; sd.en[2] = delz * rinv;
            sd.omega_i = &s->omega[3*i]; sd.omega_j = &s->omega[3*j];
            contact_chain(s, &sd, &fi, &fj, s->p.rolling_cdt);
            if (rows && k < cap) {
                double *row = rows + (size_t)nc * k;
                const double *xi = &s->x[3*i], *xj = &s->x[3*j];
                int n = 0;
                if (keys & 0x1u) {
                    for (int d = 0; d < 3; d++) row[n++] = pgl_remap(s, d, xi[d]);
                    for (int d = 0; d < 3; d++) row[n++] = pgl_remap(s, d, xj[d]);
                }
                if (keys & 0x2u) {
                    for (int d = 0; d < 3; d++) row[n++] = s->v[3*i+d];
                    for (int d = 0; d < 3; d++) row[n++] = s->v[3*j+d];
                }
                if (keys & 0x4u) {
                    row[n++] = (double)s->tag[i];
                    row[n++] = (double)s->tag[j];
                    row[n++] = j < s->nlocal ? 0. : 1.;
                }
                if (keys & 0x8u) for (int d = 0; d < 3; d++) row[n++] = fi.F[d];
                double fn[3], tn[3];
                pgl_along(xi, xj, fi.F, fn);
                pgl_along(xi, xj, fi.T, tn);
                if (keys & 0x10u) for (int d = 0; d < 3; d++) row[n++] = fn[d];
                if (keys & 0x20u) for (int d = 0; d < 3; d++) row[n++] = fi.F[d] - fn[d];
                if (keys & 0x40u) for (int d = 0; d < 3; d++) row[n++] = fi.T[d];
                if (keys & 0x80u) for (int d = 0; d < 3; d++) row[n++] = tn[d];
                if (keys & 0x100u) for (int d = 0; d < 3; d++) row[n++] = fi.T[d] - tn[d];
                if (keys & 0x200u) for (int d = 0; d < 3; d++) row[n++] = hist[d];
                if (keys & 0xc00u) {
                    double del[3] = {xi[0] - xj[0], xi[1] - xj[1], xi[2] - xj[2]};
                    const double rs = del[0]*del[0] + del[1]*del[1] + del[2]*del[2];
                    const double rr = sqrt(rs);
                    if (keys & 0x400u)
                        row[n++] = - M_PI/4 * ((rr-radi-radj)*(rr+radi-radj)*(rr-radi+radj)*(rr+radi+radj)) / rs;
                    if (keys & 0x800u) row[n++] = radi + radj - rr;
                }
                if (keys & 0x1000u)
                    for (int d = 0; d < 3; d++) row[n++] = (xi[d]*radj + xj[d]*radi) / (radi + radj);
            }
            k++;
        }
    }
    return k;
}

/* fix mesh/surface/stress on mesh wall fix ifix with reference point p_ref */
int orc_add_mesh_stress(orc_sim *s, int ifix, double px, double py, double pz)
{
    if (ifix < 0 || ifix >= s->nfix || !s->fix[ifix].wm) return -1;
    wall_mesh *m = s->fix[ifix].wm;
    m->stress = 1;
    m->p_ref[0] = px; m->p_ref[1] = py; m->p_ref[2] = pz;
    m->tri_f = calloc((size_t)(m->ntri > 0 ? m->ntri : 1), sizeof(double)*3);
    m->area_ev = calloc((size_t)(m->ntri > 0 ? m->ntri : 1), sizeof(double)*6);
    m->area_el = calloc((size_t)(m->ntri > 0 ? m->ntri : 1), sizeof(double)*2);
    for (int t = 0; t < m->ntri; t++) {   /* added before setup: the elements as created */
        memcpy(m->area_ev[t][0], m->edgevec[t][0], sizeof(double)*3);
        memcpy(m->area_ev[t][1], m->edgevec[t][1], sizeof(double)*3);
        m->area_el[t][0] = m->edgelen[t][0]; m->area_el[t][1] = m->edgelen[t][1];
    }
    return 0;
}

/* per-element force of the last step (3 per triangle) and f_total, torque_total */
int orc_get_mesh_stress(orc_sim *s, int ifix, double *tri_f, double *tot6)
{
    if (ifix < 0 || ifix >= s->nfix || !s->fix[ifix].wm || !s->fix[ifix].wm->stress) return -1;
    wall_mesh *m = s->fix[ifix].wm;
    if (tri_f) memcpy(tri_f, m->tri_f, sizeof(double)*3*m->ntri);
    if (tot6) { memcpy(tot6, m->f_total, sizeof(double)*3); memcpy(tot6 + 3, m->torque_total, sizeof(double)*3); }
    return m->ntri;
}

/* MeshModuleStress::calc_total_force src/mesh_module_stress.cpp:335-375 with
   TriMesh::calcArea src/tri_mesh_I.h:305 of the element as created */
int orc_get_mesh_sigma(orc_sim *s, int ifix, double *sigma_n, double *sigma_t)
{
    if (ifix < 0 || ifix >= s->nfix || !s->fix[ifix].wm || !s->fix[ifix].wm->stress) return -1;
    wall_mesh *m = s->fix[ifix].wm;
    for (int i = 0; i < m->ntri; i++) {
        const double *e0 = m->area_ev[i][0], *e1 = m->area_ev[i][1];
        double cr[3] = {e0[1]*e1[2] - e0[2]*e1[1], e0[2]*e1[0] - e0[0]*e1[2], e0[0]*e1[1] - e0[1]*e1[0]};
        double area = 0.5*sqrt(cr[0]*cr[0] + cr[1]*cr[1] + cr[2]*cr[2]) * m->area_el[i][0] * m->area_el[i][1];
        double invSurfArea = 1./area;
        const double *sn = m->surfnorm[i];
        const double *f = m->tri_f[i];
        double sgn = f[0]*sn[0] + f[1]*sn[1] + f[2]*sn[2];
        double tmp[3] = {sn[0]*sgn, sn[1]*sgn, sn[2]*sgn};
        tmp[0] = f[0] - tmp[0]; tmp[1] = f[1] - tmp[1]; tmp[2] = f[2] - tmp[2];
        double sgt = sqrt(tmp[0]*tmp[0] + tmp[1]*tmp[1] + tmp[2]*tmp[2]);
        sgn = fabs(sgn); sgt = fabs(sgt);
        sigma_n[i] = sgn * invSurfArea;
        sigma_t[i] = sgt * invSurfArea;
    }
    return m->ntri;
}

/* restart: FixContactHistory::unpack_restart (src/fix_contact_history.cpp:608)
   for the atoms as added (before setup; computeflag 0 so setup keeps them) */
int orc_upload_history(orc_sim *s, int n, const int *npartner, const int *ptag, const double *hist)
{
    if (n != s->nlocal) { fail(s, "history for %d atoms, %d added", n, s->nlocal); return -1; }
    size_t off = 0;
    for (int i = 0; i < n; i++) {
        free(s->partner[i]); free(s->phist[i]);
        s->npartner[i] = npartner[i];
        s->partner[i] = malloc(sizeof(int)*(npartner[i] > 0 ? npartner[i] : 1));
        s->phist[i] = malloc(sizeof(double)*3*(npartner[i] > 0 ? npartner[i] : 1));
        for (int m = 0; m < npartner[i]; m++, off++) {
            s->partner[i][m] = ptag[off];
            for (int d = 0; d < 3; d++) s->phist[i][3*m+d] = hist[3*off+d];
        }
    }
    s->computeflag = 0;
    return 0;
}

/* pack_restart after FixContactHistory::pre_exchange: per owned atom (atom
   order) its partners; returns the partner total (arrays may be NULL) */
int orc_get_history(orc_sim *s, int *npartner, int *ptag, double *hist)
{
    history_pre_exchange(s);
    s->computeflag = 1;   /* the pair keeps computing; the next build rebuilds the arrays */
    int tot = 0;
    for (int i = 0; i < s->nlocal; i++) {
        if (npartner) npartner[i] = s->npartner[i];
        for (int m = 0; m < s->npartner[i]; m++, tot++) {
            if (ptag) ptag[tot] = s->partner[i][m];
            if (hist) for (int d = 0; d < 3; d++) hist[3*tot+d] = s->phist[i][3*m+d];
        }
    }
    return tot;
}

/* FixWallGran restart data: per-atom wall shear history, before setup */
int orc_upload_wall_hist(orc_sim *s, int ifix, int n, const double *hist)
{
    if (ifix < 0 || ifix >= s->nfix || !s->fix[ifix].wp || n != s->nlocal) return -1;
    memcpy(s->fix[ifix].wp->hist, hist, sizeof(double)*3*n);
    return 0;
}

/* ComputeContactAtom::compute_peratom with skin 0 (src/compute_contact_atom.cpp:
   contact if rsq <= (radi + radj)^2 over the half list, tallied for i and j;
   newton off, so ghost tallies are dropped): per owned atom, in atom order */
int orc_contact_atom(orc_sim *s, double *out)
{
    const int nall = s->nlocal + s->nghost;
    double *contact = calloc((size_t)(nall > 0 ? nall : 1), sizeof(double));
    for (int i = 0; i < s->nlocal; i++) {
        const double xtmp = s->x[3*i], ytmp = s->x[3*i+1], ztmp = s->x[3*i+2], radi = s->radius[i];
        for (int jj = 0; jj < s->nnum[i]; jj++) {
            const int j = s->nbr[s->nstart[i] + jj];
            const double delx = xtmp - s->x[3*j], dely = ytmp - s->x[3*j+1], delz = ztmp - s->x[3*j+2];
            const double rsq = delx*delx + dely*dely + delz*delz;
            const double radsum = radi + s->radius[j] + 0.0;
            const double radsumsq = radsum*radsum;
            if (rsq <= radsumsq) {
                contact[i] += 1.0;
                contact[j] += 1.0;
            }
        }
    }
    memcpy(out, contact, sizeof(double)*s->nlocal);
    free(contact);
    return s->nlocal;
}

int orc_get_wall_hist(orc_sim *s, int ifix, double *hist)
{
    if (ifix < 0 || ifix >= s->nfix || !s->fix[ifix].wp) return -1;
    memcpy(hist, s->fix[ifix].wp->hist, sizeof(double)*3*s->nlocal);
    return s->nlocal;
}

/* wear finnie on a mesh with mesh/surface/stress: k_finnie ntypes x ntypes, row of the wall type */
int orc_add_mesh_wear(orc_sim *s, int ifix, const double *k_finnie)
{
    if (ifix < 0 || ifix >= s->nfix || !s->fix[ifix].wm || !s->fix[ifix].wm->stress) return -1;
    wall_mesh *m = s->fix[ifix].wm;
    const int nt = s->ntypes;
    m->wear = calloc(m->ntri > 0 ? m->ntri : 1, sizeof(double));
    m->kfin = calloc(nt + 1, sizeof(double));
    for (int j = 1; j <= nt; j++) m->kfin[j] = k_finnie[(m->wtype-1)*nt + (j-1)];
    return 0;
}

int orc_get_mesh_wear(orc_sim *s, int ifix, double *wear)
{
    if (ifix < 0 || ifix >= s->nfix || !s->fix[ifix].wm || !s->fix[ifix].wm->wear) return -1;
    memcpy(wear, s->fix[ifix].wm->wear, sizeof(double)*s->fix[ifix].wm->ntri);
    return 0;
}

/* FixContactHistoryMesh::write_restart (sort_contacts, src/fix_contact_history_mesh.cpp:
   375-405, 653-658) then FixContactHistory::pack_restart (src/fix_contact_history.cpp:
   588-604): per owned atom its partner count, per partner the triangle id and 3 shear
   values.  Returns the partner total; npartner / tri / hist may be NULL. */
int orc_get_mesh_history(orc_sim *s, int ifix, int cap, int *npartner, int *tri, double *hist)
{
    if (ifix < 0 || ifix >= s->nfix || !s->fix[ifix].wm) return -1;
    wall_mesh *m = s->fix[ifix].wm;
    mesh_sort_contacts(s, m);
    int k = 0;
    for (int i = 0; i < s->nlocal; i++) {
        if (npartner) npartner[i] = m->npartner[i];
        for (int q = 0; q < m->npartner[i]; q++, k++)
            if (k < cap) {
                if (tri) tri[k] = m->partner[i][q];
                if (hist) memcpy(&hist[3*k], &m->chist[i][3*q], sizeof(double)*3);
            }
    }
    return k;
}

/* FixContactHistoryMesh::unpack_restart src/fix_contact_history_mesh.cpp:613-650 */
int orc_upload_mesh_hist(orc_sim *s, int ifix, int n, const int *npartner, const int *tri, const double *hist)
{
    if (ifix < 0 || ifix >= s->nfix || !s->fix[ifix].wm || n != s->nlocal) return -1;
    wall_mesh *m = s->fix[ifix].wm;
    int k = 0;
    for (int i = 0; i < n; i++) {
        int np = npartner[i];
        free(m->partner[i]); free(m->chist[i]); free(m->keep[i]); free(m->isect[i]);
        m->partner[i] = malloc(sizeof(int)*(np > 0 ? np : 1));
        m->chist[i] = calloc((size_t)3*(np > 0 ? np : 1), sizeof(double));
        m->keep[i] = calloc(np > 0 ? np : 1, 1);
        m->isect[i] = calloc(np > 0 ? np : 1, 1);
        for (int q = 0; q < np; q++, k++) {
            m->partner[i][q] = tri[k];
            memcpy(&m->chist[i][3*q], &hist[3*k], sizeof(double)*3);
        }
        m->npartner[i] = np;
        m->nneighs[i] = np;
    }
    return 0;
}

int orc_get_mesh_contacts(orc_sim *s, int ifix, int cap, int *tag, int *tri, double *hist)
{
    if (ifix < 0 || ifix >= s->nfix || !s->fix[ifix].wm) return -1;
    wall_mesh *m = s->fix[ifix].wm;
    int k = 0;
    for (int i = 0; i < s->nlocal; i++)
        for (int j = 0; j < m->nneighs[i]; j++) {
            if (!m->partner[i] || m->partner[i][j] < 0) continue;
            if (k < cap) {
                if (tag) tag[k] = s->tag[i];
                if (tri) tri[k] = m->partner[i][j];
                if (hist) memcpy(&hist[3*k], &m->chist[i][3*j], sizeof(double)*3);
            }
            k++;
        }
    return k;
}

int orc_get_mesh_nneighs(orc_sim *s, int ifix, int *nneighs)
{
    if (ifix < 0 || ifix >= s->nfix || !s->fix[ifix].wm) return -1;
    memcpy(nneighs, s->fix[ifix].wm->nneighs, sizeof(int)*s->nlocal);
    return s->nlocal;
}
