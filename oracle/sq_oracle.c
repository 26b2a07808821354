/*
 * sq_oracle.c -- CPU oracle for superquadric contact and integration.
 * TEST INFRASTRUCTURE ONLY (see sq_oracle.h for scope, parity status and
 * the recorded deviations).  Each function cites the reference code it
 * restates.
 */
#include "sq_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define SQ_PHI_INV 0.61803398874989479   /* golden section, src/superquadric.cpp:48 */

/* ------------------------------------------------------------------ */
/* small helpers                                                        */

static double sq_dot3(const double *a, const double *b) { return a[0]*b[0] + a[1]*b[1] + a[2]*b[2]; }
static void sq_cross3(const double *a, const double *b, double *r)
{ r[0] = a[1]*b[2] - a[2]*b[1]; r[1] = a[2]*b[0] - a[0]*b[2]; r[2] = a[0]*b[1] - a[1]*b[0]; }

/* MathExtraLiggghtsNonspherical::quat_to_mat (src/math_extra_liggghts_nonspherical.h) */
static void sq_quat_to_mat(const double *q, double *m)
{
    const double w2 = q[0]*q[0], i2 = q[1]*q[1], j2 = q[2]*q[2], k2 = q[3]*q[3];
    const double twoij = 2.0*q[1]*q[2], twoik = 2.0*q[1]*q[3], twojk = 2.0*q[2]*q[3];
    const double twoiw = 2.0*q[1]*q[0], twojw = 2.0*q[2]*q[0], twokw = 2.0*q[3]*q[0];
    m[0] = w2+i2-j2-k2; m[1] = twoij-twokw; m[2] = twojw+twoik;
    m[3] = twoij+twokw; m[4] = w2-i2+j2-k2; m[5] = twojk-twoiw;
    m[6] = twoik-twojw; m[7] = twojk+twoiw; m[8] = w2-i2-j2+k2;
}
static void sq_matvec(const double *m, const double *v, double *r)
{
    r[0] = m[0]*v[0] + m[1]*v[1] + m[2]*v[2];
    r[1] = m[3]*v[0] + m[4]*v[1] + m[5]*v[2];
    r[2] = m[6]*v[0] + m[7]*v[1] + m[8]*v[2];
}
static void sq_tmatvec(const double *m, const double *v, double *r)
{
    r[0] = m[0]*v[0] + m[3]*v[1] + m[6]*v[2];
    r[1] = m[1]*v[0] + m[4]*v[1] + m[7]*v[2];
    r[2] = m[2]*v[0] + m[5]*v[1] + m[8]*v[2];
}

/* MathExtraLiggghtsNonspherical::pow_abs_int / pow_abs
   (src/math_extra_liggghts_nonspherical.h:137-221): |a|^b by repeated
   products for the integer part, sqrt or pow for the fractional part */
static double sq_pow_abs_int(double a, int b)
{
    a = fabs(a);
    switch (b) {
    case 0: return 1.0;
    case 1: return a;
    case 2: return a*a;
    case 3: return a*a*a;
    case 4: { double a2 = a*a; return a2*a2; }
    case 5: { double a2 = a*a; return a2*a2*a; }
    case 6: { double a3 = a*a*a; return a3*a3; }
    case 7: { double a2 = a*a; double a3 = a2*a; return a2*a2*a3; }
    case 8: { double a2 = a*a; double a4 = a2*a2; return a4*a4; }
    case 9: { double a3 = a*a*a; return a3*a3*a3; }
    default: { double r = a; for (int i = 0; i < b - 1; i++) r *= a; return r; }
    }
}
static double sq_pow_abs(double base, double e)
{
    base = fabs(base);
    const double tol = 1e-12;
    if (fabs(e) < tol || fabs(base - 1.0) < tol) return 1.0;
    if (fabs(base) < tol) return 0.0;
    const double n = floor(fabs(e));
    double r = sq_pow_abs_int(base, (int)n);
    const double nd = fabs(e) - n;
    if (nd > 0.0) {
        if (fabs(2.0*nd - 1.0) < 2.0*tol) r *= sqrt(base);
        else r *= pow(base, nd);
    }
    return e > 0.0 ? r : 1.0/r;
}
static double sq_sign(double v) { return v > 0.0 ? 1.0 : (v < 0.0 ? -1.0 : 0.0); }
/* MathExtraLiggghts::compDouble */
static int sq_comp_double(double a, double b, double prec)
{
    if (a == b) return 1;
    if (fabs(a - b) < prec) return 1;
    return 0;
}
/* MathExtraLiggghtsNonspherical::isInteger */
static int sq_is_integer(double x) { return sq_comp_double(x, floor(x + 1e-2), 1e-2); }

/* ------------------------------------------------------------------ */
/* Superquadric (src/superquadric.cpp) with n1 = n2 = n                 */

typedef struct {
    const orc_sq_particle *p;
    double rot[9];           /* rotation_matrix (local -> global) */
    double shape[3], shape_inv[3];
    double n;
    double koef;             /* calc_koef :701 */
    int use_int;             /* useIntBlockiness */
} sq_body;

static void sq_body_set(sq_body *b, const orc_sq_particle *p, const double *shape, double n)
{
    b->p = p;
    sq_quat_to_mat(p->quat, b->rot);
    for (int d = 0; d < 3; d++) { b->shape[d] = shape[d]; b->shape_inv[d] = 1.0/shape[d]; }
    b->n = n;
    b->koef = sq_pow_abs(0.5, n - 2.0);
    const int ell = sq_comp_double(n, 2.0, 1e-2);
    b->use_int = ell ? 1 : sq_is_integer(n);
}

static void sq_global2local(const sq_body *b, const double *x, double *xl)
{
    double t[3] = {x[0] - b->p->center[0], x[1] - b->p->center[1], x[2] - b->p->center[2]};
    sq_tmatvec(b->rot, t, xl);
}

/* Superquadric::shape_function_local (:111) */
static double sq_f_local(const sq_body *b, const double *xl)
{
    double f;
    if (b->use_int) {
        const int ni = (int)floor(b->n + 1e-2);
        f = sq_pow_abs_int(xl[0]*b->shape_inv[0], ni) + sq_pow_abs_int(xl[1]*b->shape_inv[1], ni) +
            sq_pow_abs_int(xl[2]*b->shape_inv[2], ni) - 1.0;
    } else {
        f = (sq_pow_abs(sq_pow_abs(xl[0]*b->shape_inv[0], b->n) + sq_pow_abs(xl[1]*b->shape_inv[1], b->n), 1.0) +
             sq_pow_abs(xl[2]*b->shape_inv[2], b->n) - 1.0);
    }
    return b->koef*f;
}

/* Superquadric::shape_function_gradient_local (:141), n1 = n2 branch */
static void sq_grad_local(const sq_body *b, const double *xl, double *g)
{
    const double a = b->shape_inv[0], bb = b->shape_inv[1], c = b->shape_inv[2], n = b->n;
    const double xa = xl[0]*a, yb = xl[1]*bb, zc = xl[2]*c;
    double xan21, ybn21, zcn11;
    if (b->use_int) {
        const int ni = (int)floor(n + 1e-2);
        xan21 = sq_pow_abs_int(xa, ni - 1); ybn21 = sq_pow_abs_int(yb, ni - 1); zcn11 = sq_pow_abs_int(zc, ni - 1);
    } else {
        xan21 = sq_pow_abs(xa, n - 1.0); ybn21 = sq_pow_abs(yb, n - 1.0); zcn11 = sq_pow_abs(zc, n - 1.0);
    }
    g[0] = n*(b->koef*a)*sq_sign(xa)*xan21;
    g[1] = n*(b->koef*bb)*sq_sign(yb)*ybn21;
    g[2] = n*(b->koef*c)*sq_sign(zc)*zcn11;
}

/* Superquadric::shape_function_props_local (:237), n1 = n2 branch */
static void sq_props_local(const sq_body *b, const double *xl, double *f, double *g, double *h)
{
    const double a = b->shape_inv[0], bb = b->shape_inv[1], c = b->shape_inv[2], n = b->n, k = b->koef;
    const double xa = xl[0]*a, yb = xl[1]*bb, zc = xl[2]*c;
    double xan22, ybn22, zcn12;
    if (b->use_int) {
        const int ni = (int)floor(n + 1e-2);
        xan22 = sq_pow_abs_int(xa, ni - 2); ybn22 = sq_pow_abs_int(yb, ni - 2); zcn12 = sq_pow_abs_int(zc, ni - 2);
    } else {
        xan22 = sq_pow_abs(xa, n - 2.0); ybn22 = sq_pow_abs(yb, n - 2.0); zcn12 = sq_pow_abs(zc, n - 2.0);
    }
    const double xan21 = xan22*fabs(xa), ybn21 = ybn22*fabs(yb), zcn11 = zcn12*fabs(zc);
    const double xan2 = xan21*fabs(xa), ybn2 = ybn21*fabs(yb), zcn1 = zcn11*fabs(zc);
    *f = k*(xan2 + ybn2 + zcn1 - 1.0);
    g[0] = k*a*n*sq_sign(xa)*xan21;
    g[1] = k*bb*n*sq_sign(yb)*ybn21;
    g[2] = k*c*n*sq_sign(zc)*zcn11;
    if (h) {
        h[0] = (k*a)*(n*(n - 1.0)*xan22)*a;
        h[4] = (k*bb)*(n*(n - 1.0)*ybn22)*bb;
        h[8] = (k*c)*(n*(n - 1.0)*zcn12)*c;
        h[1] = h[3] = h[2] = h[6] = h[5] = h[7] = 0.0;
    }
}

/* shape_function_props_global (:316): local props, gradient rotated to
   the global frame, Hessian A H A^T (tensor_quat_rotate) */
static void sq_props_global(const sq_body *b, const double *x, double *f, double *g, double *h)
{
    double xl[3], gl[3], hl[9];
    sq_global2local(b, x, xl);
    sq_props_local(b, xl, f, gl, h ? hl : NULL);
    sq_matvec(b->rot, gl, g);
    if (h) {
        const double *A = b->rot;
        double t[9];
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
                t[3*i + j] = A[3*i + 0]*hl[0*3 + j] + A[3*i + 1]*hl[1*3 + j] + A[3*i + 2]*hl[2*3 + j];
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
                h[3*i + j] = t[3*i + 0]*A[3*j + 0] + t[3*i + 1]*A[3*j + 1] + t[3*i + 2]*A[3*j + 2];
    }
}

void orc_sq_shape_props(const orc_sq_particle *P, const double x[3], double *f, double grad[3], double hess[9])
{
    sq_body b;
    sq_body_set(&b, P, P->shape, P->n);
    sq_props_global(&b, x, f, grad, hess);
}

double orc_sq_bounding_radius(const double shape[3], double n)
{
    /* bounding_sphere_radius_superquadric with n1 = n2 = n, times scale_koef
       1.0001 (src/math_extra_liggghts_nonspherical.h:60) */
    if (sq_comp_double(n, 2.0, 1e-13)) return fmax(fmax(shape[0], shape[1]), shape[2])*1.0001;
    const double a = fmax(shape[0], shape[1]), b = fmin(shape[0], shape[1]), c = shape[2];
    const double n1 = fmax(2.1, n), n2 = fmax(2.1, n);
    const double alpha = sq_pow_abs(b/a, 2.0/(n2 - 2.0));
    const double gamma = sq_pow_abs(1.0 + sq_pow_abs(alpha, n2), n1/n2 - 1.0);
    const double beta = sq_pow_abs(c*c/(a*a)*gamma, 1.0/(n1 - 2.0));
    const double x0 = 1.0/sq_pow_abs(sq_pow_abs(1.0 + sq_pow_abs(alpha, n2), n1/n2) + sq_pow_abs(beta, n1), 1.0/n1);
    const double xt = x0*a, yt = alpha*x0*b, zt = beta*x0*c;
    return sqrt(xt*xt + yt*yt + zt*zt)*1.0001;
}

/* ------------------------------------------------------------------ */
/* contact point: calc_F and the Newton solve                          */

/* calc_F with mu given (src/math_extra_liggghts_superquadric.cpp:619) */
static double sq_calc_F_mu(const sq_body *A, const sq_body *B, double *f1, double *f2, double *gA, double *gB,
                           const double *pt, double mu, double *F, double *merit)
{
    sq_props_global(A, pt, f1, gA, NULL);
    sq_props_global(B, pt, f2, gB, NULL);
    const double mu_sq = mu*mu;
    F[0] = gA[0] + mu_sq*gB[0];
    F[1] = gA[1] + mu_sq*gB[1];
    F[2] = gA[2] + mu_sq*gB[2];
    F[3] = *f1 - *f2;
    double v[3];
    sq_cross3(gA, gB, v);
    const double sine = fabs(sq_dot3(v, v)/(sq_dot3(gA, gA)*sq_dot3(gB, gB)));
    const double aaa = fabs(*f1 - *f2)/(fmax(fabs(*f1), fabs(*f2)) + 1e-16);
    *merit = fmax(sine, aaa*aaa);
    return F[0]*F[0] + F[1]*F[1] + F[2]*F[2] + F[3]*F[3];
}

/* calc_F with mu from the gradients (:645): mu^2 = -gA.gB / |gB|^2 */
static double sq_calc_F(const sq_body *A, const sq_body *B, double *f1, double *f2, double *gA, double *gB,
                        const double *pt, double *mu, double *F, double *merit)
{
    sq_props_global(A, pt, f1, gA, NULL);
    sq_props_global(B, pt, f2, gB, NULL);
    const double mu_sq = -sq_dot3(gA, gB)/sq_dot3(gB, gB);
    *mu = sqrt(fabs(mu_sq));
    F[0] = gA[0] + mu_sq*gB[0];
    F[1] = gA[1] + mu_sq*gB[1];
    F[2] = gA[2] + mu_sq*gB[2];
    F[3] = *f1 - *f2;
    double v[3];
    sq_cross3(gA, gB, v);
    const double sine = fabs(sq_dot3(v, v)/(sq_dot3(gA, gA)*sq_dot3(gB, gB)));
    const double aaa = fabs(*f1 - *f2)/(fmax(fabs(*f1), fabs(*f2)) + 1e-16);
    *merit = fmax(sine, aaa*aaa);
    return F[0]*F[0] + F[1]*F[1] + F[2]*F[2] + F[3]*F[3];
}

/* 4x4 linear solve J x = F, Gaussian elimination with partial pivoting;
   returns 0 if singular */
static int sq_solve4(const double *J, const double *F, double *x)
{
    double a[4][5];
    for (int i = 0; i < 4; i++) {
        for (int j = 0; j < 4; j++) a[i][j] = J[4*i + j];
        a[i][4] = F[i];
    }
    for (int c = 0; c < 4; c++) {
        int p = c;
        for (int r = c + 1; r < 4; r++) if (fabs(a[r][c]) > fabs(a[p][c])) p = r;
        if (a[p][c] == 0.0) return 0;
        if (p != c) for (int j = 0; j < 5; j++) { double t = a[c][j]; a[c][j] = a[p][j]; a[p][j] = t; }
        for (int r = c + 1; r < 4; r++) {
            const double m = a[r][c]/a[c][c];
            for (int j = c; j < 5; j++) a[r][j] -= m*a[c][j];
        }
    }
    for (int i = 3; i >= 0; i--) {
        double s = a[i][4];
        for (int j = i + 1; j < 4; j++) s -= a[i][j]*x[j];
        x[i] = s/a[i][i];
    }
    return 1;
}

/* MathExtraLiggghtsNonspherical::calc_contact_point (:778-1020): Newton on
   F(x, mu) = (gA + mu^2 gB, fA - fB) = 0 from the better of the given
   point and the sphere solution; a rejected Newton step falls back to a
   golden-section search along it.  Converged when the merit is below 1e-10,
   the step below 1e-12 x the smallest half-axis, or the residual stalls
   (relative change < 1e-3). */
typedef struct {
    double point[3], mu, fi, fj, gA[3], gB[3], merit;
    int iters, fail;
} sq_newton;

static void sq_newton_solve(const sq_body *A, const sq_body *B, double ratio, const double *init1,
                            int have_mu, double mu_init, sq_newton *o)
{
    const double tol1 = 1e-10, tol2 = 1e-12;
    o->fail = 0;
    o->iters = 0;
    double F[4], F1[4], F2[4], gA1[3], gB1[3], gA2[3], gB2[3];
    double fi1, fj1, fi2, fj2, mu1, mu2, merit01, merit02;
    double res01;
    if (have_mu) {
        mu1 = mu_init;
        res01 = sq_calc_F_mu(A, B, &fi1, &fj1, gA1, gB1, init1, mu1, F1, &merit01);
    } else {
        res01 = sq_calc_F(A, B, &fi1, &fj1, gA1, gB1, init1, &mu1, F1, &merit01);
    }
    if (merit01 < tol1) {
        memcpy(o->point, init1, sizeof(double)*3);
        memcpy(o->gA, gA1, sizeof gA1); memcpy(o->gB, gB1, sizeof gB1);
        o->fi = fi1; o->fj = fj1; o->mu = mu1; o->merit = merit01;
        return;
    }
    double init2[3];
    for (int k = 0; k < 3; k++) init2[k] = ratio*B->p->center[k] + (1.0 - ratio)*A->p->center[k];
    const double res02 = sq_calc_F(A, B, &fi2, &fj2, gA2, gB2, init2, &mu2, F2, &merit02);
    double point[3], gA[3], gB[3], mu, fi, fj, res0, merit0;
    if (res01 < res02) {
        res0 = res01; memcpy(gA, gA1, sizeof gA); memcpy(gB, gB1, sizeof gB); memcpy(point, init1, sizeof point);
        memcpy(F, F1, sizeof F); fi = fi1; fj = fj1; mu = mu1; merit0 = merit01;
    } else {
        res0 = res02; memcpy(gA, gA2, sizeof gA); memcpy(gB, gB2, sizeof gB); memcpy(point, init2, sizeof point);
        memcpy(F, F2, sizeof F); fi = fi2; fj = fj2; mu = mu2; merit0 = merit02;
    }
    if (merit0 < tol1) {
        memcpy(o->point, point, sizeof point); memcpy(o->gA, gA, sizeof gA); memcpy(o->gB, gB, sizeof gB);
        o->fi = fi; o->fj = fj; o->mu = mu; o->merit = merit0;
        return;
    }
    double merit1 = merit0, merit2 = merit0, res1 = res0, res2 = res0;
    const double size_i = fmin(fmin(A->shape[0], A->shape[1]), A->shape[2]);
    const double size_j = fmin(fmin(B->shape[0], B->shape[1]), B->shape[2]);
    const double size = fmin(size_i, size_j);
    const int Niter = 100000;
    for (int iter = 0; iter < Niter; iter++) {
        o->iters++;
        merit2 = merit1;
        res2 = res1;
        double f_, hA[9], hB[9], gtmp[3];
        sq_props_global(A, point, &f_, gtmp, hA);
        sq_props_global(B, point, &f_, gtmp, hB);
        const double mu_sq = mu*mu;
        double J[16];
        for (int i = 0; i < 3; i++) {
            for (int j = 0; j < 3; j++) J[4*i + j] = hA[3*i + j] + mu_sq*hB[3*i + j];
            J[3 + 4*i] = 2.0*mu*gB[i];
            J[i + 4*3] = gA[i] - gB[i];
        }
        J[15] = 0.0;
        double delta[4];
        int converged = 0, nan_found = 0;
        if (!sq_solve4(J, F, delta)) nan_found = 1;
        for (int i = 0; i < 4 && !nan_found; i++) if (isnan(delta[i])) nan_found = 1;
        if (nan_found) { o->fail = 1; break; }
        const double deltax = fmax(fmax(fabs(delta[0]), fabs(delta[1])), fabs(delta[2]));
        if (deltax == 0.0) {
            converged = 1;
        } else {
            double p_[3] = {point[0] - delta[0], point[1] - delta[1], point[2] - delta[2]};
            const double mu_ = mu - delta[3];
            double fi_, fj_, merit2_, gA_[3], gB_[3], F_[4];
            const double res2_ = sq_calc_F_mu(A, B, &fi_, &fj_, gA_, gB_, p_, mu_, F_, &merit2_);
            if (res2_ < res1 || merit2_ < tol1 || deltax < tol2*size) {
                merit2 = merit2_; res2 = res2_; mu = mu_; fi = fi_; fj = fj_;
                memcpy(point, p_, sizeof point); memcpy(gA, gA_, sizeof gA); memcpy(gB, gB_, sizeof gB);
                memcpy(F, F_, sizeof F);
                if (merit2 < tol1 || deltax < tol2*size) converged = 1;
            } else {   /* golden-section search along the Newton step */
                double a = 0.0, b = 1.0, eps = fabs(b - a);
                double res2a = 0, res2b = 0, merit2a = 0, merit2b = 0, pa[3], pb[3];
                while (eps > 1e-8) {
                    const double al1 = b - (b - a)*SQ_PHI_INV;
                    const double al2 = a + (b - a)*SQ_PHI_INV;
                    for (int k = 0; k < 3; k++) { pa[k] = point[k] - al1*delta[k]; pb[k] = point[k] - al2*delta[k]; }
                    mu1 = mu - al1*delta[3];
                    res2a = sq_calc_F_mu(A, B, &fi1, &fj1, gA1, gB1, pa, mu1, F1, &merit2a);
                    mu2 = mu - al2*delta[3];
                    res2b = sq_calc_F_mu(A, B, &fi2, &fj2, gA2, gB2, pb, mu2, F2, &merit2b);
                    if (fmin(res2a, res2b) < res1) {
                        if (res2a < res2b) {
                            res2 = res2a; memcpy(F, F1, sizeof F); mu = mu1; memcpy(gA, gA1, sizeof gA);
                            memcpy(gB, gB1, sizeof gB); memcpy(point, pa, sizeof point); fi = fi1; fj = fj1;
                            merit2 = merit2a;
                        } else {
                            res2 = res2b; memcpy(F, F2, sizeof F); mu = mu2; memcpy(gA, gA2, sizeof gA);
                            memcpy(gB, gB2, sizeof gB); memcpy(point, pb, sizeof point); fi = fi2; fj = fj2;
                            merit2 = merit2b;
                        }
                        if (merit2 < tol1) converged = 1;
                        eps = 0.0;
                    } else {
                        if (res2a > res2b) a = al1; else b = al2;
                        eps = fabs(b - a);
                    }
                }
                if (eps != 0.0) {
                    memcpy(F, F2, sizeof F); mu = mu2; memcpy(gA, gA2, sizeof gA); memcpy(gB, gB2, sizeof gB);
                    memcpy(point, pb, sizeof point); fi = fi2; fj = fj2;
                    res2 = res2b; merit2 = merit2b;
                    if (merit2 < tol1) converged = 1;
                }
            }
            if (fabs(res1 - res2)/fmax(res1, res2) < 1e-3) converged = 1;
        }
        merit1 = merit2;
        res1 = res2;
        if (iter >= Niter - 1) o->fail = 1;
        if (converged || o->fail) break;
    }
    memcpy(o->point, point, sizeof point); memcpy(o->gA, gA, sizeof gA); memcpy(o->gB, gB, sizeof gB);
    o->fi = fi; o->fj = fj; o->mu = mu; o->merit = merit1;
}

/* calc_contact_point_if_no_previous_point_avaialable (:1391-1435): from
   spheres of the volume-equivalent radius cbrt(abc) (blockiness 2) to the
   actual shapes in N = max((nmax - 2)/1 + 1, 10) + 1 stages, each stage's
   solution seeding the next */
static void sq_homotopy(const orc_sq_particle *PA, const orc_sq_particle *PB, sq_newton *o, int *iters, int *solves)
{
    const double ri = cbrt(PA->shape[0]*PA->shape[1]*PA->shape[2]);
    const double rj = cbrt(PB->shape[0]*PB->shape[1]*PB->shape[2]);
    const double ratio = ri/(ri + rj);
    const double nmax = fmax(PA->n, PB->n);
    const int N1 = (int)((nmax - 2.0)/1.0 + 1);
    const int N = N1 > 10 ? N1 : 10;
    const double N_inv = 1.0/(double)N;
    double cp[3];
    *iters = 0;
    *solves = 0;
    for (int i = 0; i <= N; i++) {
        const double t = (double)i*N_inv;
        double sa[3], sb[3];
        for (int d = 0; d < 3; d++) { sa[d] = ri + (PA->shape[d] - ri)*t; sb[d] = rj + (PB->shape[d] - rj)*t; }
        sq_body A, B;
        sq_body_set(&A, PA, sa, 2.0 + (PA->n - 2.0)*t);
        sq_body_set(&B, PB, sb, 2.0 + (PB->n - 2.0)*t);
        if (i == 0)
            for (int k = 0; k < 3; k++) cp[k] = ratio*PB->center[k] + (1.0 - ratio)*PA->center[k];
        double pre[3] = {cp[0], cp[1], cp[2]};
        sq_newton_solve(&A, &B, ratio, pre, 0, 0.0, o);
        memcpy(cp, o->point, sizeof cp);
        *iters += o->iters;
        (*solves)++;
    }
}

void orc_sq_contact_point(const orc_sq_particle *A, const orc_sq_particle *B, int mode, const double guess[3],
                          orc_sq_solution *out)
{
    sq_newton o;
    memset(out, 0, sizeof *out);
    if (mode == ORC_SQ_GUESS_HOMOTOPY) {
        sq_homotopy(A, B, &o, &out->iters, &out->solves);
    } else {
        sq_body a, b;
        sq_body_set(&a, A, A->shape, A->n);
        sq_body_set(&b, B, B->shape, B->n);
        const double ri = cbrt(A->shape[0]*A->shape[1]*A->shape[2]);
        const double rj = cbrt(B->shape[0]*B->shape[1]*B->shape[2]);
        sq_newton_solve(&a, &b, ri/(ri + rj), guess, 0, 0.0, &o);
        out->iters = o.iters;
        out->solves = 1;
    }
    memcpy(out->point, o.point, sizeof out->point);
    memcpy(out->gradi, o.gA, sizeof out->gradi);
    memcpy(out->gradj, o.gB, sizeof out->gradj);
    out->mu = o.mu;
    out->fi = o.fi;
    out->fj = o.fj;
    out->merit = o.merit;
    out->fail = o.fail;
}

/* ------------------------------------------------------------------ */
/* broad phase: oriented bounding boxes (obb_intersect :166, the 15
   separating axes of two boxes, half-axes scaled by 1.0001)             */

static int sq_obb_intersect(const sq_body *A, const sq_body *B)
{
    double T[3] = {A->p->center[0] - B->p->center[0], A->p->center[1] - B->p->center[1],
                   A->p->center[2] - B->p->center[2]};
    double a[3], b[3];
    for (int d = 0; d < 3; d++) { a[d] = A->shape[d]*1.0001; b[d] = B->shape[d]*1.0001; }
    /* axes: columns of the rotation matrices; C = A^T B */
    double C[9], AbsC[9], TA[3], TB[3];
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            C[3*i + j] = A->rot[0*3 + i]*B->rot[0*3 + j] + A->rot[1*3 + i]*B->rot[1*3 + j] + A->rot[2*3 + i]*B->rot[2*3 + j];
            AbsC[3*i + j] = fabs(C[3*i + j]);
        }
    sq_tmatvec(A->rot, T, TA);
    sq_tmatvec(B->rot, T, TB);
    for (int i = 0; i < 3; i++) {   /* axes of A */
        const double r = a[i], rb = b[0]*AbsC[3*i] + b[1]*AbsC[3*i + 1] + b[2]*AbsC[3*i + 2];
        if (fabs(TA[i]) > r + rb) return 0;
    }
    for (int j = 0; j < 3; j++) {   /* axes of B */
        const double ra = a[0]*AbsC[j] + a[1]*AbsC[3 + j] + a[2]*AbsC[6 + j];
        if (fabs(TB[j]) > ra + b[j]) return 0;
    }
    for (int i = 0; i < 3; i++)     /* A_i x B_j */
        for (int j = 0; j < 3; j++) {
            const int i1 = (i + 1)%3, i2 = (i + 2)%3, j1 = (j + 1)%3, j2 = (j + 2)%3;
            const double ra = a[i1]*AbsC[3*i2 + j] + a[i2]*AbsC[3*i1 + j];
            const double rb = b[j1]*AbsC[3*i + j2] + b[j2]*AbsC[3*i + j1];
            const double t = fabs(TA[i2]*C[3*i1 + j] - TA[i1]*C[3*i2 + j]);
            if (t > ra + rb) return 0;
        }
    return 1;
}

/* ------------------------------------------------------------------ */
/* overlap: Superquadric::surface_line_intersection (:712-818) and
   extended_overlap_algorithm (:1489)                                    */

static double sq_line_intersection(const sq_body *b, const double *start, const double *dir, double alpha_prev,
                                   double *result)
{
    const int max_iters = 20;
    double sl[3], dl[3], point[3], gl[3];
    sq_global2local(b, start, sl);
    sq_tmatvec(b->rot, dir, dl);
    double alpha = alpha_prev;
    const double eps0 = 1e-14;
    const int is_ell = sq_comp_double(b->n, 2.0, 1e-2);
    if (is_ell) {
        const double x0 = sl[0]*b->shape_inv[0], nx = dl[0]*b->shape_inv[0];
        const double y0 = sl[1]*b->shape_inv[1], ny = dl[1]*b->shape_inv[1];
        const double z0 = sl[2]*b->shape_inv[2], nz = dl[2]*b->shape_inv[2];
        const double qa = nx*nx + ny*ny + nz*nz, qb = 2.0*(x0*nx + y0*ny + z0*nz), qc = x0*x0 + y0*y0 + z0*z0 - 1.0;
        const double D = qb*qb - 4.0*qa*qc, tai = 0.5/qa;
        double a1, a2;
        if (D < 0) { a1 = -qb*tai; a2 = a1; }
        else { const double sD = sqrt(D); a1 = (-qb + sD)*tai; a2 = (-qb - sD)*tai; }
        if (a1 > -eps0 && a2 < -eps0) alpha = a1;
        else if (a1 < -eps0 && a2 > -eps0) alpha = a2;
        else if (a1 < -eps0 && a2 < -eps0) alpha = fmax(a1, a2);
        else alpha = fmin(a1, a2);
    } else {
        const double a = 0.5*fmin(fmin(b->shape[0], b->shape[1]), b->shape[2])/sqrt(sq_dot3(dir, dir));
        const double eps = 1e-16;
        alpha = alpha < -a ? -a : (alpha > a ? a : alpha);
        for (int k = 0; k < 3; k++) point[k] = sl[k] + alpha*dl[k];
        double f0 = sq_f_local(b, point);
        if (fabs(f0) < eps) {
            for (int k = 0; k < 3; k++) result[k] = start[k] + alpha*dir[k];
            return alpha;
        }
        for (int it = 0; it < max_iters; it++) {
            if (fabs(f0) < eps*b->koef) break;
            sq_grad_local(b, point, gl);
            const double f_der = sq_dot3(gl, dl);
            double delta;
            if (fabs(f_der) < 1e-10) {
                delta = 1e-10;
                double p_[3], g_[3];
                for (int k = 0; k < 3; k++) p_[k] = point[k] + delta*dl[k];
                sq_grad_local(b, p_, g_);
                if (sq_dot3(g_, dl) < 0.0) delta = -delta;
            } else {
                delta = -f0/f_der;
                delta = delta < -a ? -a : (delta > a ? a : delta);
            }
            if (fabs(delta) <= eps) {
                alpha += delta;
                for (int k = 0; k < 3; k++) point[k] = point[k] + delta*dl[k];
                break;
            }
            while (fabs(delta) > eps) {
                double p_[3];
                for (int k = 0; k < 3; k++) p_[k] = point[k] + delta*dl[k];
                const double f_ = sq_f_local(b, p_);
                if (fabs(f_) < fabs(f0) || fabs(f_) < eps*b->koef) {
                    f0 = f_;
                    alpha += delta;
                    memcpy(point, p_, sizeof point);
                    break;
                }
                delta *= 0.5;
            }
        }
    }
    for (int k = 0; k < 3; k++) result[k] = start[k] + alpha*dir[k];
    return alpha;
}

/* ------------------------------------------------------------------ */
/* a superquadric DEM run: Verlet steps with fix nve/asphere
   (integration_scheme 1), a bounding-sphere half list with skin, and
   pair gran hertz/history on superquadric surfaces                      */

enum { SQ_FAR = 0, SQ_CLOSE = 1, SQ_INTERSECT = 2 };   /* src/surface_model_superquadric.h:73 */

typedef struct {
    int j;
    int flag;              /* contact flag (CONTACT_NORMAL_MODEL | CONTACT_TANGENTIAL_MODEL) */
    int state;             /* particles_were_in_contact */
    double cp[3];          /* contact point of the previous step */
    double alpha[2];       /* line-intersection parameters (extended overlap) */
    double shear[3];
} sq_slot;

struct orc_sq {
    orc_sq_params p;
    int n;
    double *x, *v, *quat, *angmom, *omega, *f, *torque, *shape, *blk, *rmass, *inertia, *volume;
    double *rb;            /* bounding-sphere radius (neighbour list, broad phase) */
    double *xhold;
    int *start, *num;      /* half list per atom (j > i ascending) */
    sq_slot *slots;
    int nslots, capslots;
    double Yeff, Geff, betaeff, mu;
    long iters, solves, pairs_solved, nbuilds;
};

static void sq_build(orc_sq *s, int transfer)
{
    /* Neighbor::build with FixContactHistory transfer keyed by the pair:
       only flagged (touching) pairs keep their history */
    sq_slot *old = s->slots;
    int *ostart = NULL, *onum = NULL;
    if (transfer && old) {
        ostart = malloc(sizeof(int)*s->n); onum = malloc(sizeof(int)*s->n);
        memcpy(ostart, s->start, sizeof(int)*s->n); memcpy(onum, s->num, sizeof(int)*s->n);
    }
    s->slots = NULL;
    s->nslots = 0;
    s->capslots = 0;
    for (int i = 0; i < s->n; i++) {
        s->start[i] = s->nslots;
        for (int j = i + 1; j < s->n; j++) {
            double d[3] = {s->x[3*i] - s->x[3*j], s->x[3*i+1] - s->x[3*j+1], s->x[3*i+2] - s->x[3*j+2]};
            const double cut = s->rb[i] + s->rb[j] + s->p.skin;
            if (sq_dot3(d, d) > cut*cut) continue;
            if (s->nslots == s->capslots) {
                s->capslots = s->capslots ? 2*s->capslots : 1024;
                s->slots = realloc(s->slots, sizeof(sq_slot)*s->capslots);
            }
            sq_slot *sl = &s->slots[s->nslots++];
            memset(sl, 0, sizeof *sl);
            sl->j = j;
            if (ostart)
                for (int q = 0; q < onum[i]; q++) {
                    const sq_slot *o = &old[ostart[i] + q];
                    if (o->j == j) { if (o->flag) *sl = *o; break; }
                }
        }
        s->num[i] = s->nslots - s->start[i];
    }
    free(old); free(ostart); free(onum);
    memcpy(s->xhold, s->x, sizeof(double)*3*s->n);
    s->nbuilds++;
}

orc_sq *orc_sq_create(const orc_sq_params *p, int n, const double *x, const double *v, const double *quat,
                      const double *angmom, const double *shape, const double *blockiness,
                      const double *rmass, const double *inertia, const double *volume)
{
    orc_sq *s = calloc(1, sizeof(orc_sq));
    s->p = *p;
    s->n = n;
#define SQ_ARR(name, k, src) s->name = malloc(sizeof(double)*(k)*(n > 0 ? n : 1)); if (src) memcpy(s->name, src, sizeof(double)*(k)*n); else memset(s->name, 0, sizeof(double)*(k)*(n > 0 ? n : 1));
    SQ_ARR(x, 3, x) SQ_ARR(v, 3, v) SQ_ARR(quat, 4, quat) SQ_ARR(angmom, 3, angmom) SQ_ARR(omega, 3, NULL)
    SQ_ARR(f, 3, NULL) SQ_ARR(torque, 3, NULL) SQ_ARR(shape, 3, shape) SQ_ARR(blk, 1, blockiness)
    SQ_ARR(rmass, 1, rmass) SQ_ARR(inertia, 3, inertia) SQ_ARR(volume, 1, volume) SQ_ARR(rb, 1, NULL)
    SQ_ARR(xhold, 3, NULL)
#undef SQ_ARR
    s->start = calloc(n > 0 ? n : 1, sizeof(int));
    s->num = calloc(n > 0 ? n : 1, sizeof(int));
    for (int i = 0; i < n; i++) s->rb[i] = orc_sq_bounding_radius(&s->shape[3*i], s->blk[i]);
    /* material constants as in src/global_properties.cpp:432-540 (one type) */
    const double E = p->youngs, nu = p->poisson;
    s->Yeff = 1./((1.-pow(nu,2.))/E+(1.-pow(nu,2.))/E);
    s->Geff = 1./(2.*(2.-nu)*(1.+nu)/E+2.*(2.-nu)*(1.+nu)/E);
    const double lg = log(p->restitution);
    s->betaeff = lg / sqrt(pow(lg,2.)+pow(M_PI,2.));
    s->mu = p->friction;
    /* omega from angmom: body-frame angmom / inertia, rotated back */
    for (int i = 0; i < n; i++) {
        double R[9], mb[3], wb[3];
        sq_quat_to_mat(&s->quat[4*i], R);
        sq_tmatvec(R, &s->angmom[3*i], mb);
        for (int d = 0; d < 3; d++) wb[d] = mb[d]/s->inertia[3*i + d];
        sq_matvec(R, wb, &s->omega[3*i]);
    }
    return s;
}

void orc_sq_destroy(orc_sq *s)
{
    if (!s) return;
    free(s->x); free(s->v); free(s->quat); free(s->angmom); free(s->omega); free(s->f); free(s->torque);
    free(s->shape); free(s->blk); free(s->rmass); free(s->inertia); free(s->volume); free(s->rb); free(s->xhold);
    free(s->start); free(s->num); free(s->slots);
    free(s);
}

/* MathExtra::quatvec / invquatvec / qnormalize (src/math_extra.h:546-615) */
static void sq_quatvec(const double *a, const double *b, double *c)
{
    c[0] = -a[1]*b[0] - a[2]*b[1] - a[3]*b[2];
    c[1] = a[0]*b[0] + a[2]*b[2] - a[3]*b[1];
    c[2] = a[0]*b[1] + a[3]*b[0] - a[1]*b[2];
    c[3] = a[0]*b[2] + a[1]*b[1] - a[2]*b[0];
}
static void sq_invquatvec(const double *a, const double *b, double *c)
{
    c[0] = -a[1]*b[0] + a[0]*b[1] + a[3]*b[2] - a[2]*b[3];
    c[1] = -a[2]*b[0] - a[3]*b[1] + a[0]*b[2] + a[1]*b[3];
    c[2] = -a[3]*b[0] + a[2]*b[1] - a[1]*b[2] + a[0]*b[3];
}
static void sq_qnormalize(double *q)
{
    const double norm = 1.0/sqrt(q[0]*q[0] + q[1]*q[1] + q[2]*q[2] + q[3]*q[3]);
    q[0] *= norm; q[1] *= norm; q[2] *= norm; q[3] *= norm;
}
/* no_squish_rotate (src/math_extra_liggghts_nonspherical.cpp:175) */
static void sq_no_squish_rotate(int k, double *p, double *q, const double *inertia, double dt)
{
    double kp[4] = {0, 0, 0, 0}, kq[4] = {0, 0, 0, 0};
    if (k == 1) {
        kq[0] = -q[1]; kp[0] = -p[1]; kq[1] = q[0]; kp[1] = p[0];
        kq[2] = q[3]; kp[2] = p[3]; kq[3] = -q[2]; kp[3] = -p[2];
    } else if (k == 2) {
        kq[0] = -q[2]; kp[0] = -p[2]; kq[1] = -q[3]; kp[1] = -p[3];
        kq[2] = q[0]; kp[2] = p[0]; kq[3] = q[1]; kp[3] = p[1];
    } else if (k == 3) {
        kq[0] = -q[3]; kp[0] = -p[3]; kq[1] = q[2]; kp[1] = p[2];
        kq[2] = -q[1]; kp[2] = -p[1]; kq[3] = q[0]; kp[3] = p[0];
    }
    double phi = p[0]*kq[0] + p[1]*kq[1] + p[2]*kq[2] + p[3]*kq[3];
    phi /= 4.0*inertia[k-1];
    const double c_phi = cos(dt*phi), s_phi = sin(dt*phi);
    p[0] = c_phi*p[0] + s_phi*kp[0]; p[1] = c_phi*p[1] + s_phi*kp[1];
    p[2] = c_phi*p[2] + s_phi*kp[2]; p[3] = c_phi*p[3] + s_phi*kp[3];
    q[0] = c_phi*q[0] + s_phi*kq[0]; q[1] = c_phi*q[1] + s_phi*kq[1];
    q[2] = c_phi*q[2] + s_phi*kq[2]; q[3] = c_phi*q[3] + s_phi*kq[3];
}

/* FixNVEAsphereBase::initial_integrate, integration_scheme 1 (src/fix_nve_asphere_base.cpp:319-444) */
static void sq_initial_integrate(orc_sq *s)
{
    const double dtv = s->p.dt, dtf = 0.5*s->p.dt*1.0, dtf2 = 2.0*dtf, dtq = 0.5*dtv;
    for (int i = 0; i < s->n; i++) {
        double R[9], mbody[3], conjqm[4], tbody[3], fquat[4], wbody[3];
        double *q = &s->quat[4*i], *v = &s->v[3*i], *x = &s->x[3*i], *in = &s->inertia[3*i];
        sq_quat_to_mat(q, R);
        const double dtfm = dtf/s->rmass[i];
        v[0] += dtfm*s->f[3*i]; v[1] += dtfm*s->f[3*i+1]; v[2] += dtfm*s->f[3*i+2];
        x[0] += dtv*v[0]; x[1] += dtv*v[1]; x[2] += dtv*v[2];
        sq_tmatvec(R, &s->angmom[3*i], mbody);
        sq_quatvec(q, mbody, conjqm);
        for (int k = 0; k < 4; k++) conjqm[k] *= 2.0;
        sq_tmatvec(R, &s->torque[3*i], tbody);
        sq_quatvec(q, tbody, fquat);
        for (int k = 0; k < 4; k++) conjqm[k] += dtf2*fquat[k];
        sq_no_squish_rotate(3, conjqm, q, in, dtq);
        sq_no_squish_rotate(2, conjqm, q, in, dtq);
        sq_no_squish_rotate(1, conjqm, q, in, dtv);
        sq_no_squish_rotate(2, conjqm, q, in, dtq);
        sq_no_squish_rotate(3, conjqm, q, in, dtq);
        sq_qnormalize(q);
        sq_quat_to_mat(q, R);
        sq_invquatvec(q, conjqm, mbody);
        for (int d = 0; d < 3; d++) mbody[d] *= 0.5;
        for (int d = 0; d < 3; d++) wbody[d] = mbody[d]/in[d];
        sq_matvec(R, mbody, &s->angmom[3*i]);
        sq_matvec(R, wbody, &s->omega[3*i]);
    }
}

/* FixNVEAsphereBase::final_integrate, integration_scheme 1 (:523-620) */
static void sq_final_integrate(orc_sq *s)
{
    const double dtf = 0.5*s->p.dt*1.0, dtf2 = dtf*2.0;
    for (int i = 0; i < s->n; i++) {
        double R[9], tbody[3], mbody[3], conjqm[4], fquat[4], wbody[3];
        double *q = &s->quat[4*i], *v = &s->v[3*i], *in = &s->inertia[3*i];
        const double dtfm = dtf/s->rmass[i];
        sq_quat_to_mat(q, R);
        v[0] += dtfm*s->f[3*i]; v[1] += dtfm*s->f[3*i+1]; v[2] += dtfm*s->f[3*i+2];
        sq_tmatvec(R, &s->torque[3*i], tbody);
        sq_tmatvec(R, &s->angmom[3*i], mbody);
        sq_quatvec(q, mbody, conjqm);
        for (int k = 0; k < 4; k++) conjqm[k] *= 2.0;
        sq_quatvec(q, tbody, fquat);
        for (int k = 0; k < 4; k++) conjqm[k] += dtf2*fquat[k];
        sq_invquatvec(q, conjqm, mbody);
        for (int d = 0; d < 3; d++) mbody[d] *= 0.5;
        for (int d = 0; d < 3; d++) wbody[d] = mbody[d]/in[d];
        sq_matvec(R, mbody, &s->angmom[3*i]);
        sq_matvec(R, wbody, &s->omega[3*i]);
    }
}

/* SurfaceModel<SUPERQUADRIC>::checkSurfaceIntersect
   (src/surface_model_superquadric.h:108-205) for one half-list slot;
   returns 1 when the surfaces intersect, with the contact point, normal,
   overlap and the solver's gradients */
static int sq_check_intersect(orc_sq *s, int i, int j, sq_slot *sl, double *cp, double *en, double *deltan)
{
    orc_sq_particle PA, PB;
    memcpy(PA.center, &s->x[3*i], sizeof PA.center); memcpy(PA.quat, &s->quat[4*i], sizeof PA.quat);
    memcpy(PA.shape, &s->shape[3*i], sizeof PA.shape); PA.n = s->blk[i];
    memcpy(PB.center, &s->x[3*j], sizeof PB.center); memcpy(PB.quat, &s->quat[4*j], sizeof PB.quat);
    memcpy(PB.shape, &s->shape[3*j], sizeof PB.shape); PB.n = s->blk[j];
    sq_body A, B;
    sq_body_set(&A, &PA, PA.shape, PA.n);
    sq_body_set(&B, &PB, PB.shape, PB.n);
    int in_contact = 0;
    const int obb = sl->state == SQ_INTERSECT ? 1 : sq_obb_intersect(&A, &B);
    if (obb) {
        const double ri = cbrt(PA.shape[0]*PA.shape[1]*PA.shape[2]);
        const double rj = cbrt(PB.shape[0]*PB.shape[1]*PB.shape[2]);
        const double ratio = ri/(ri + rj);
        sq_newton o;
        int it = 0, sv = 0;
        if (sl->state == SQ_FAR) {
            sq_homotopy(&PA, &PB, &o, &it, &sv);
        } else {
            /* calc_contact_point_using_prev_step (:1438): the previous point
               advanced with the mass-weighted contact-point velocity */
            double xci[3], xcj[3], vri[3], vrj[3], est[3];
            for (int k = 0; k < 3; k++) { xci[k] = sl->cp[k] - PA.center[k]; xcj[k] = sl->cp[k] - PB.center[k]; }
            sq_cross3(&s->omega[3*i], xci, vri);
            sq_cross3(&s->omega[3*j], xcj, vrj);
            const double mi = s->rmass[i], mj = s->rmass[j];
            for (int k = 0; k < 3; k++) {
                const double vi = s->v[3*i + k] + vri[k], vj = s->v[3*j + k] + vrj[k];
                const double veff = (vi*mi + vj*mj)/(mi + mj);
                est[k] = sl->cp[k] + veff*s->p.dt;
            }
            sq_newton_solve(&A, &B, ratio, est, 0, 0.0, &o);
            it = o.iters;
            sv = 1;
        }
        s->iters += it;
        s->solves += sv;
        s->pairs_solved++;
        memcpy(cp, o.point, sizeof(double)*3);
        memcpy(sl->cp, o.point, sizeof sl->cp);
        in_contact = fmax(o.fi, o.fj) < 0.0;
        if (in_contact) {
            for (int k = 0; k < 3; k++) en[k] = o.gB[k] - o.gA[k];
            const double nrm = sqrt(en[0]*en[0] + en[1]*en[1] + en[2]*en[2]);
            const double inv = nrm == 0. ? 0. : 1./nrm;
            for (int k = 0; k < 3; k++) en[k] *= inv;
            /* extended_overlap_algorithm (:1489) */
            double ne[3] = {-en[0], -en[1], -en[2]}, cpa[3], cpb[3];
            sl->alpha[0] = sq_line_intersection(&A, cp, ne, sl->alpha[0], cpa);
            sl->alpha[1] = sq_line_intersection(&B, cp, en, sl->alpha[1], cpb);
            *deltan = fabs(sl->alpha[0]) + fabs(sl->alpha[1]);
            sl->state = SQ_INTERSECT;
        } else {
            sl->state = SQ_CLOSE;
        }
    } else {
        sl->state = SQ_FAR;
    }
    return in_contact;
}

/* PairGran::compute for superquadrics (src/pair_gran_base.h:255-430) with
   the non-spherical kinematics (src/math_extra_liggghts_nonspherical.h:536),
   Hertz (src/normal_model_hertz.h:202-393) and tangential history with
   contact-point lever arms (src/tangential_model_history.h:130-300) */
static void sq_pair_compute(orc_sq *s, int shearupdate)
{
    memset(s->f, 0, sizeof(double)*3*s->n);
    memset(s->torque, 0, sizeof(double)*3*s->n);
    const double dt = s->p.dt;
    for (int i = 0; i < s->n; i++) {
        const double radi = cbrt(0.75*s->volume[i]/M_PI);
        for (int q = 0; q < s->num[i]; q++) {
            sq_slot *sl = &s->slots[s->start[i] + q];
            const int j = sl->j;
            double d[3] = {s->x[3*i] - s->x[3*j], s->x[3*i+1] - s->x[3*j+1], s->x[3*i+2] - s->x[3*j+2]};
            const double rsq = sq_dot3(d, d), radsum = s->rb[i] + s->rb[j];
            if (!(rsq < radsum*radsum)) continue;
            double cp[3], en[3], deltan = 0.0;
            if (!sq_check_intersect(s, i, j, sl, cp, en, &deltan)) continue;
            const double radj = cbrt(0.75*s->volume[j]/M_PI);
            const double mi = s->rmass[i], mj = s->rmass[j], meff = mi*mj/(mi + mj);
            double xci[3], xcj[3], vri[3], vrj[3], vrel[3];
            for (int k = 0; k < 3; k++) { xci[k] = cp[k] - s->x[3*i + k]; xcj[k] = cp[k] - s->x[3*j + k]; }
            sq_cross3(&s->omega[3*i], xci, vri);
            sq_cross3(&s->omega[3*j], xcj, vrj);
            for (int k = 0; k < 3; k++) vrel[k] = s->v[3*i + k] - s->v[3*j + k] + (vri[k] - vrj[k]);
            const double vn = sq_dot3(vrel, en);
            const double vtr[3] = {vrel[0] - vn*en[0], vrel[1] - vn*en[1], vrel[2] - vn*en[2]};
            const double reff = radi*radj/(radi + radj);
            const double sqrtval = sqrt(reff*deltan);
            const double Sn = 2.*s->Yeff*sqrtval, St = 8.*s->Geff*sqrtval;
            const double kn = 4./3.*s->Yeff*sqrtval, kt = St;
            const double sqrtFiveOverSix = 0.91287092917527685576161630466800355658790782499663875;
            const double gamman = -2.*sqrtFiveOverSix*s->betaeff*sqrt(Sn*meff);
            const double gammat = -2.*sqrtFiveOverSix*s->betaeff*sqrt(St*meff);
            const double Fn = -gamman*vn + kn*deltan;
            double Fi[3] = {Fn*en[0], Fn*en[1], Fn*en[2]}, Ti[3], Tj[3];
            const double Fnj[3] = {-Fi[0], -Fi[1], -Fi[2]};
            sq_cross3(xci, Fi, Ti);
            sq_cross3(xcj, Fnj, Tj);
            sl->flag |= 5;
            double *sh = sl->shear;
            if (shearupdate) {
                for (int k = 0; k < 3; k++) sh[k] += vtr[k]*dt;
                const double rsht = sq_dot3(sh, en);
                for (int k = 0; k < 3; k++) sh[k] -= rsht*en[k];
            }
            const double shrmag = sqrt(sq_dot3(sh, sh));
            double Ft[3] = {-(kt*sh[0]), -(kt*sh[1]), -(kt*sh[2])};
            const double Ft_shear = kt*shrmag, Ft_friction = s->mu*fabs(Fn);
            if (Ft_shear > Ft_friction) {
                if (shrmag != 0.0) {
                    const double ratio = Ft_friction/Ft_shear;
                    for (int k = 0; k < 3; k++) Ft[k] *= ratio;
                    if (shearupdate) for (int k = 0; k < 3; k++) sh[k] = -Ft[k]/kt;
                } else {
                    Ft[0] = Ft[1] = Ft[2] = 0.0;
                }
            } else {
                for (int k = 0; k < 3; k++) Ft[k] -= gammat*vtr[k];
            }
            double ti[3], tj[3];
            const double Ftj[3] = {-Ft[0], -Ft[1], -Ft[2]};
            sq_cross3(xci, Ft, ti);
            sq_cross3(xcj, Ftj, tj);
            for (int k = 0; k < 3; k++) {
                s->f[3*i + k] += Fi[k] + Ft[k];
                s->f[3*j + k] += Fnj[k] + Ftj[k];
                s->torque[3*i + k] += Ti[k] + ti[k];
                s->torque[3*j + k] += Tj[k] + tj[k];
            }
        }
    }
}

static int sq_decide(orc_sq *s)
{
    const double trig = 0.25*s->p.skin*s->p.skin;
    for (int i = 0; i < s->n; i++) {
        double d[3] = {s->x[3*i] - s->xhold[3*i], s->x[3*i+1] - s->xhold[3*i+1], s->x[3*i+2] - s->xhold[3*i+2]};
        if (sq_dot3(d, d) > trig) return 1;
    }
    return 0;
}

int orc_sq_setup(orc_sq *s)
{
    sq_build(s, 0);
    sq_pair_compute(s, 0);
    return 0;
}

int orc_sq_run(orc_sq *s, int nsteps)
{
    for (int step = 0; step < nsteps; step++) {
        sq_initial_integrate(s);
        if (sq_decide(s)) sq_build(s, 1);
        sq_pair_compute(s, 1);
        sq_final_integrate(s);
    }
    return 0;
}

void orc_sq_get_atoms(orc_sq *s, double *x, double *v, double *quat, double *angmom, double *omega, double *f,
                      double *torque)
{
    const int n = s->n;
    if (x) memcpy(x, s->x, sizeof(double)*3*n);
    if (v) memcpy(v, s->v, sizeof(double)*3*n);
    if (quat) memcpy(quat, s->quat, sizeof(double)*4*n);
    if (angmom) memcpy(angmom, s->angmom, sizeof(double)*3*n);
    if (omega) memcpy(omega, s->omega, sizeof(double)*3*n);
    if (f) memcpy(f, s->f, sizeof(double)*3*n);
    if (torque) memcpy(torque, s->torque, sizeof(double)*3*n);
}

int orc_sq_get_pairs(orc_sq *s, int cap, int *tag_i, int *tag_j, int *state, double *cp, double *shear)
{
    int k = 0;
    for (int i = 0; i < s->n; i++)
        for (int q = 0; q < s->num[i]; q++) {
            const sq_slot *sl = &s->slots[s->start[i] + q];
            if (k < cap) {
                if (tag_i) tag_i[k] = i + 1;
                if (tag_j) tag_j[k] = sl->j + 1;
                if (state) state[k] = sl->state;
                if (cp) memcpy(&cp[3*k], sl->cp, sizeof(double)*3);
                if (shear) memcpy(&shear[3*k], sl->shear, sizeof(double)*3);
            }
            k++;
        }
    return k;
}

void orc_sq_counters(orc_sq *s, long *iters, long *solves, long *pairs_solved, long *nbuilds)
{
    if (iters) *iters = s->iters;
    if (solves) *solves = s->solves;
    if (pairs_solved) *pairs_solved = s->pairs_solved;
    if (nbuilds) *nbuilds = s->nbuilds;
}
