// gb2_sq.cuh -- device math of the superquadric contact path.
//
// Superquadric shape function |x/a|^n + |y/b|^n + |z/c|^n - 1 scaled by
// 0.5^(n-2) (one blockiness per particle, n1 = n2), its gradient and Hessian
// (src/superquadric.cpp:111-330), the 4-unknown Newton solve for the contact
// point with golden-section fallback (src/math_extra_liggghts_superquadric.cpp:778-1020),
// the sphere-to-shape homotopy for pairs without a previous point (:1391),
// the oriented-box pre-test (:166), the line-surface intersection that
// measures the overlap (src/superquadric.cpp:712-818, extended overlap :1489)
// and the asphere integrator (src/fix_nve_asphere_base.cpp:319-620,
// integration_scheme 1).  The arithmetic is FP64 throughout; pow() with a
// non-integer exponent comes from CUDA's math library, so results agree
// with the CPU restatement to the solver tolerance, not bit for bit.
#pragma once

#include <cuda_runtime.h>

namespace gb2 {
namespace sq {

constexpr double kPhiInv = 0.61803398874989479;   // golden section
enum : int { FAR = 0, CLOSE = 1, INTERSECT = 2 };   // src/surface_model_superquadric.h:73

__device__ __forceinline__ double dot3(const double *a, const double *b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
__device__ __forceinline__ void cross3(const double *a, const double *b, double *r)
{
    r[0] = a[1] * b[2] - a[2] * b[1];
    r[1] = a[2] * b[0] - a[0] * b[2];
    r[2] = a[0] * b[1] - a[1] * b[0];
}

__device__ __forceinline__ void quat_to_mat(const double *q, double *m)
{
    const double w2 = q[0] * q[0], i2 = q[1] * q[1], j2 = q[2] * q[2], k2 = q[3] * q[3];
    const double twoij = 2.0 * q[1] * q[2], twoik = 2.0 * q[1] * q[3], twojk = 2.0 * q[2] * q[3];
    const double twoiw = 2.0 * q[1] * q[0], twojw = 2.0 * q[2] * q[0], twokw = 2.0 * q[3] * q[0];
    m[0] = w2 + i2 - j2 - k2;
    m[1] = twoij - twokw;
    m[2] = twojw + twoik;
    m[3] = twoij + twokw;
    m[4] = w2 - i2 + j2 - k2;
    m[5] = twojk - twoiw;
    m[6] = twoik - twojw;
    m[7] = twojk + twoiw;
    m[8] = w2 - i2 - j2 + k2;
}
__device__ __forceinline__ void matvec(const double *m, const double *v, double *r)
{
    r[0] = m[0] * v[0] + m[1] * v[1] + m[2] * v[2];
    r[1] = m[3] * v[0] + m[4] * v[1] + m[5] * v[2];
    r[2] = m[6] * v[0] + m[7] * v[1] + m[8] * v[2];
}
__device__ __forceinline__ void tmatvec(const double *m, const double *v, double *r)
{
    r[0] = m[0] * v[0] + m[3] * v[1] + m[6] * v[2];
    r[1] = m[1] * v[0] + m[4] * v[1] + m[7] * v[2];
    r[2] = m[2] * v[0] + m[5] * v[1] + m[8] * v[2];
}

// |a|^b by products (MathExtraLiggghtsNonspherical::pow_abs_int)
__device__ __forceinline__ double pow_abs_int(double a, int b)
{
    a = fabs(a);
    switch (b) {
    case 0: return 1.0;
    case 1: return a;
    case 2: return a * a;
    case 3: return a * a * a;
    case 4: { const double a2 = a * a; return a2 * a2; }
    case 5: { const double a2 = a * a; return a2 * a2 * a; }
    case 6: { const double a3 = a * a * a; return a3 * a3; }
    case 7: { const double a2 = a * a, a3 = a2 * a; return a2 * a2 * a3; }
    case 8: { const double a2 = a * a, a4 = a2 * a2; return a4 * a4; }
    case 9: { const double a3 = a * a * a; return a3 * a3 * a3; }
    default: { double r = a; for (int i = 0; i < b - 1; i++) r *= a; return r; }
    }
}
// |base|^e: integer part by products, fractional part by sqrt or pow
// (MathExtraLiggghtsNonspherical::pow_abs)
__device__ __forceinline__ double pow_abs(double base, double e)
{
    base = fabs(base);
    const double tol = 1e-12;
    if (fabs(e) < tol || fabs(base - 1.0) < tol) return 1.0;
    if (fabs(base) < tol) return 0.0;
    const double n = floor(fabs(e));
    double r = pow_abs_int(base, (int)n);
    const double nd = fabs(e) - n;
    if (nd > 0.0) {
        if (fabs(2.0 * nd - 1.0) < 2.0 * tol) r *= sqrt(base);
        else r *= pow(base, nd);
    }
    return e > 0.0 ? r : 1.0 / r;
}
__device__ __forceinline__ double sgn(double v) { return v > 0.0 ? 1.0 : (v < 0.0 ? -1.0 : 0.0); }
__device__ __forceinline__ bool comp_double(double a, double b, double prec) { return a == b || fabs(a - b) < prec; }
__device__ __forceinline__ bool is_integer(double x) { return comp_double(x, floor(x + 1e-2), 1e-2); }

struct Body {
    double c[3];
    double rot[9];
    double shape[3], inv[3];
    double n, koef;
    int use_int;
};

__device__ __forceinline__ void body_set(Body &b, const double *center, const double *quat, const double *shape, double n)
{
    for (int d = 0; d < 3; d++) {
        b.c[d] = center[d];
        b.shape[d] = shape[d];
        b.inv[d] = 1.0 / shape[d];
    }
    quat_to_mat(quat, b.rot);
    b.n = n;
    b.koef = pow_abs(0.5, n - 2.0);
    b.use_int = comp_double(n, 2.0, 1e-2) ? 1 : (is_integer(n) ? 1 : 0);
}
__device__ __forceinline__ void body_shape(Body &b, const double *shape, double n)
{
    for (int d = 0; d < 3; d++) {
        b.shape[d] = shape[d];
        b.inv[d] = 1.0 / shape[d];
    }
    b.n = n;
    b.koef = pow_abs(0.5, n - 2.0);
    b.use_int = comp_double(n, 2.0, 1e-2) ? 1 : (is_integer(n) ? 1 : 0);
}

__device__ __forceinline__ void to_local(const Body &b, const double *x, double *xl)
{
    const double t[3] = {x[0] - b.c[0], x[1] - b.c[1], x[2] - b.c[2]};
    tmatvec(b.rot, t, xl);
}

// shape function value in the body frame (Superquadric::shape_function_local)
__device__ __forceinline__ double f_local(const Body &b, const double *xl)
{
    double f;
    if (b.use_int) {
        const int ni = (int)floor(b.n + 1e-2);
        f = pow_abs_int(xl[0] * b.inv[0], ni) + pow_abs_int(xl[1] * b.inv[1], ni) + pow_abs_int(xl[2] * b.inv[2], ni) -
            1.0;
    } else {
        f = (pow_abs(pow_abs(xl[0] * b.inv[0], b.n) + pow_abs(xl[1] * b.inv[1], b.n), 1.0) +
             pow_abs(xl[2] * b.inv[2], b.n) - 1.0);
    }
    return b.koef * f;
}

__device__ __forceinline__ void grad_local(const Body &b, const double *xl, double *g)
{
    const double a = b.inv[0], bb = b.inv[1], c = b.inv[2], n = b.n;
    const double xa = xl[0] * a, yb = xl[1] * bb, zc = xl[2] * c;
    double xan21, ybn21, zcn11;
    if (b.use_int) {
        const int ni = (int)floor(n + 1e-2);
        xan21 = pow_abs_int(xa, ni - 1);
        ybn21 = pow_abs_int(yb, ni - 1);
        zcn11 = pow_abs_int(zc, ni - 1);
    } else {
        xan21 = pow_abs(xa, n - 1.0);
        ybn21 = pow_abs(yb, n - 1.0);
        zcn11 = pow_abs(zc, n - 1.0);
    }
    g[0] = n * (b.koef * a) * sgn(xa) * xan21;
    g[1] = n * (b.koef * bb) * sgn(yb) * ybn21;
    g[2] = n * (b.koef * c) * sgn(zc) * zcn11;
}

// value, gradient and (optionally) Hessian in the global frame
// (shape_function_props_local / _global)
__device__ __forceinline__ void props_global(const Body &b, const double *x, double *f, double *g, double *h)
{
    double xl[3];
    to_local(b, x, xl);
    const double a = b.inv[0], bb = b.inv[1], c = b.inv[2], n = b.n, k = b.koef;
    const double xa = xl[0] * a, yb = xl[1] * bb, zc = xl[2] * c;
    double xan22, ybn22, zcn12;
    if (b.use_int) {
        const int ni = (int)floor(n + 1e-2);
        xan22 = pow_abs_int(xa, ni - 2);
        ybn22 = pow_abs_int(yb, ni - 2);
        zcn12 = pow_abs_int(zc, ni - 2);
    } else {
        xan22 = pow_abs(xa, n - 2.0);
        ybn22 = pow_abs(yb, n - 2.0);
        zcn12 = pow_abs(zc, n - 2.0);
    }
    const double xan21 = xan22 * fabs(xa), ybn21 = ybn22 * fabs(yb), zcn11 = zcn12 * fabs(zc);
    const double xan2 = xan21 * fabs(xa), ybn2 = ybn21 * fabs(yb), zcn1 = zcn11 * fabs(zc);
    *f = k * (xan2 + ybn2 + zcn1 - 1.0);
    const double gl[3] = {k * a * n * sgn(xa) * xan21, k * bb * n * sgn(yb) * ybn21, k * c * n * sgn(zc) * zcn11};
    matvec(b.rot, gl, g);
    if (h) {
        // diagonal local Hessian rotated: h = A diag(d) A^T
        const double d0 = (k * a) * (n * (n - 1.0) * xan22) * a;
        const double d1 = (k * bb) * (n * (n - 1.0) * ybn22) * bb;
        const double d2 = (k * c) * (n * (n - 1.0) * zcn12) * c;
        const double *A = b.rot;
        for (int i = 0; i < 3; i++)
            for (int j = 0; j < 3; j++)
                h[3 * i + j] = (A[3 * i + 0] * d0) * A[3 * j + 0] + (A[3 * i + 1] * d1) * A[3 * j + 1] +
                               (A[3 * i + 2] * d2) * A[3 * j + 2];
    }
}

// calc_F: residual of the contact conditions at (x, mu)
__device__ __forceinline__ double calc_F(const Body &A, const Body &B, const double *pt, double mu, bool mu_from_grad,
                                         double &f1, double &f2, double *gA, double *gB, double *F, double &merit,
                                         double &mu_out)
{
    props_global(A, pt, &f1, gA, nullptr);
    props_global(B, pt, &f2, gB, nullptr);
    double mu_sq;
    if (mu_from_grad) {
        mu_sq = -dot3(gA, gB) / dot3(gB, gB);
        mu_out = sqrt(fabs(mu_sq));
    } else {
        mu_sq = mu * mu;
        mu_out = mu;
    }
    F[0] = gA[0] + mu_sq * gB[0];
    F[1] = gA[1] + mu_sq * gB[1];
    F[2] = gA[2] + mu_sq * gB[2];
    F[3] = f1 - f2;
    double v[3];
    cross3(gA, gB, v);
    const double sine = fabs(dot3(v, v) / (dot3(gA, gA) * dot3(gB, gB)));
    const double aaa = fabs(f1 - f2) / (fmax(fabs(f1), fabs(f2)) + 1e-16);
    merit = fmax(sine, aaa * aaa);
    return F[0] * F[0] + F[1] * F[1] + F[2] * F[2] + F[3] * F[3];
}

// 4x4 solve by Gaussian elimination with partial pivoting; false if singular
__device__ __forceinline__ bool solve4(const double *J, const double *F, double *x)
{
    double a[4][5];
    for (int i = 0; i < 4; i++) {
        for (int j = 0; j < 4; j++) a[i][j] = J[4 * i + j];
        a[i][4] = F[i];
    }
    for (int c = 0; c < 4; c++) {
        int p = c;
        for (int r = c + 1; r < 4; r++)
            if (fabs(a[r][c]) > fabs(a[p][c])) p = r;
        if (a[p][c] == 0.0) return false;
        if (p != c)
            for (int j = 0; j < 5; j++) {
                const double t = a[c][j];
                a[c][j] = a[p][j];
                a[p][j] = t;
            }
        for (int r = c + 1; r < 4; r++) {
            const double m = a[r][c] / a[c][c];
            for (int j = c; j < 5; j++) a[r][j] -= m * a[c][j];
        }
    }
    for (int i = 3; i >= 0; i--) {
        double s = a[i][4];
        for (int j = i + 1; j < 4; j++) s -= a[i][j] * x[j];
        x[i] = s / a[i][i];
    }
    return true;
}

struct Newton {
    double point[3], mu, fi, fj, gA[3], gB[3], merit;
    int iters, fail;
};

constexpr int kMaxNewton = 1000;   // iteration bound on the device (the reference allows 100000)

// calc_contact_point: Newton from the better of `init1` and the sphere
// solution, golden-section search when a step does not reduce the residual
template <int MAXIT = kMaxNewton>
__device__ __noinline__ void newton_solve(const Body &A, const Body &B, double ratio, const double *init1,
                                          bool have_mu, double mu_init, Newton &o)
{
    const double tol1 = 1e-10, tol2 = 1e-12;
    o.fail = 0;
    o.iters = 0;
    double F[4], F1[4], F2[4], gA1[3], gB1[3], gA2[3], gB2[3];
    double fi1, fj1, fi2, fj2, mu1, mu2, merit01, merit02, res01, res02;
    res01 = calc_F(A, B, init1, mu_init, !have_mu, fi1, fj1, gA1, gB1, F1, merit01, mu1);
    if (merit01 < tol1) {
        for (int k = 0; k < 3; k++) {
            o.point[k] = init1[k];
            o.gA[k] = gA1[k];
            o.gB[k] = gB1[k];
        }
        o.fi = fi1;
        o.fj = fj1;
        o.mu = mu1;
        o.merit = merit01;
        return;
    }
    double init2[3];
    for (int k = 0; k < 3; k++) init2[k] = ratio * B.c[k] + (1.0 - ratio) * A.c[k];
    res02 = calc_F(A, B, init2, 0.0, true, fi2, fj2, gA2, gB2, F2, merit02, mu2);
    double point[3], gA[3], gB[3], mu, fi, fj, res0, merit0;
    const bool first = res01 < res02;
    for (int k = 0; k < 3; k++) {
        point[k] = first ? init1[k] : init2[k];
        gA[k] = first ? gA1[k] : gA2[k];
        gB[k] = first ? gB1[k] : gB2[k];
    }
    for (int k = 0; k < 4; k++) F[k] = first ? F1[k] : F2[k];
    fi = first ? fi1 : fi2;
    fj = first ? fj1 : fj2;
    mu = first ? mu1 : mu2;
    res0 = first ? res01 : res02;
    merit0 = first ? merit01 : merit02;
    double merit1 = merit0, merit2 = merit0, res1 = res0, res2 = res0;
    if (merit0 >= tol1) {
        const double size = fmin(fmin(fmin(A.shape[0], A.shape[1]), A.shape[2]), fmin(fmin(B.shape[0], B.shape[1]), B.shape[2]));
        for (int iter = 0; iter < MAXIT; iter++) {
            o.iters++;
            merit2 = merit1;
            res2 = res1;
            double hA[9], hB[9], gt[3], ft;
            props_global(A, point, &ft, gt, hA);
            props_global(B, point, &ft, gt, hB);
            const double mu_sq = mu * mu;
            double J[16];
            for (int i = 0; i < 3; i++) {
                for (int j = 0; j < 3; j++) J[4 * i + j] = hA[3 * i + j] + mu_sq * hB[3 * i + j];
                J[3 + 4 * i] = 2.0 * mu * gB[i];
                J[i + 4 * 3] = gA[i] - gB[i];
            }
            J[15] = 0.0;
            double delta[4];
            bool converged = false;
            bool bad = !solve4(J, F, delta);
            for (int i = 0; i < 4 && !bad; i++)
                if (isnan(delta[i])) bad = true;
            if (bad) {
                o.fail = 1;
                break;
            }
            const double deltax = fmax(fmax(fabs(delta[0]), fabs(delta[1])), fabs(delta[2]));
            if (deltax == 0.0) {
                converged = true;
            } else {
                const double p_[3] = {point[0] - delta[0], point[1] - delta[1], point[2] - delta[2]};
                const double mu_ = mu - delta[3];
                double fi_, fj_, merit2_, gA_[3], gB_[3], F_[4], mo;
                const double res2_ = calc_F(A, B, p_, mu_, false, fi_, fj_, gA_, gB_, F_, merit2_, mo);
                if (res2_ < res1 || merit2_ < tol1 || deltax < tol2 * size) {
                    merit2 = merit2_;
                    res2 = res2_;
                    mu = mu_;
                    fi = fi_;
                    fj = fj_;
                    for (int k = 0; k < 3; k++) {
                        point[k] = p_[k];
                        gA[k] = gA_[k];
                        gB[k] = gB_[k];
                    }
                    for (int k = 0; k < 4; k++) F[k] = F_[k];
                    if (merit2 < tol1 || deltax < tol2 * size) converged = true;
                } else {   // golden-section search along the Newton step
                    double a = 0.0, b = 1.0, eps = 1.0;
                    double res2a = 0, res2b = 0, merit2a = 0, merit2b = 0, pa[3], pb[3];
                    while (eps > 1e-8) {
                        const double al1 = b - (b - a) * kPhiInv;
                        const double al2 = a + (b - a) * kPhiInv;
                        for (int k = 0; k < 3; k++) {
                            pa[k] = point[k] - al1 * delta[k];
                            pb[k] = point[k] - al2 * delta[k];
                        }
                        mu1 = mu - al1 * delta[3];
                        res2a = calc_F(A, B, pa, mu1, false, fi1, fj1, gA1, gB1, F1, merit2a, mo);
                        mu2 = mu - al2 * delta[3];
                        res2b = calc_F(A, B, pb, mu2, false, fi2, fj2, gA2, gB2, F2, merit2b, mo);
                        if (fmin(res2a, res2b) < res1) {
                            const bool ua = res2a < res2b;
                            res2 = ua ? res2a : res2b;
                            for (int k = 0; k < 4; k++) F[k] = ua ? F1[k] : F2[k];
                            mu = ua ? mu1 : mu2;
                            for (int k = 0; k < 3; k++) {
                                gA[k] = ua ? gA1[k] : gA2[k];
                                gB[k] = ua ? gB1[k] : gB2[k];
                                point[k] = ua ? pa[k] : pb[k];
                            }
                            fi = ua ? fi1 : fi2;
                            fj = ua ? fj1 : fj2;
                            merit2 = ua ? merit2a : merit2b;
                            if (merit2 < tol1) converged = true;
                            eps = 0.0;
                        } else {
                            if (res2a > res2b) a = al1;
                            else b = al2;
                            eps = fabs(b - a);
                        }
                    }
                    if (eps != 0.0) {
                        for (int k = 0; k < 4; k++) F[k] = F2[k];
                        mu = mu2;
                        for (int k = 0; k < 3; k++) {
                            gA[k] = gA2[k];
                            gB[k] = gB2[k];
                            point[k] = pb[k];
                        }
                        fi = fi2;
                        fj = fj2;
                        res2 = res2b;
                        merit2 = merit2b;
                        if (merit2 < tol1) converged = true;
                    }
                }
                if (fabs(res1 - res2) / fmax(res1, res2) < 1e-3) converged = true;
            }
            merit1 = merit2;
            res1 = res2;
            if (iter >= MAXIT - 1) o.fail = 1;
            if (converged || o.fail) break;
        }
    }
    for (int k = 0; k < 3; k++) {
        o.point[k] = point[k];
        o.gA[k] = gA[k];
        o.gB[k] = gB[k];
    }
    o.fi = fi;
    o.fj = fj;
    o.mu = mu;
    o.merit = merit1;
}

// Contact-point solve of one pair in one of three ways:
//   mode 0: homotopy from spheres of radius cbrt(abc) to the actual shapes in
//           N = max(nmax - 1, 10) + 1 stages (first contact, no previous point);
//   mode 1: one solve from `guess` (previous point advanced, or a learned guess
//           with `guess_mu`).
// Returns the final stage's solution; iters/solves count all stages.
template <int MAXIT = kMaxNewton>
__device__ __forceinline__ void contact_point(const double *ca, const double *qa, const double *sa, double na,
                                              const double *cb, const double *qb, const double *sb, double nb,
                                              int mode, const double *guess, bool have_mu, double guess_mu,
                                              Newton &o, int &iters, int &solves)
{
    Body A, B;
    body_set(A, ca, qa, sa, na);
    body_set(B, cb, qb, sb, nb);
    const double ri = cbrt(sa[0] * sa[1] * sa[2]);
    const double rj = cbrt(sb[0] * sb[1] * sb[2]);
    const double ratio = ri / (ri + rj);
    iters = 0;
    solves = 0;
    int N = 0;
    if (mode == 0) {
        const double nmax = fmax(na, nb);
        const int N1 = (int)((nmax - 2.0) / 1.0 + 1);
        N = N1 > 10 ? N1 : 10;
    }
    const double N_inv = mode == 0 ? 1.0 / (double)N : 0.0;
    double cp[3];
    if (mode == 0)
        for (int k = 0; k < 3; k++) cp[k] = ratio * cb[k] + (1.0 - ratio) * ca[k];
    else
        for (int k = 0; k < 3; k++) cp[k] = guess[k];
    for (int i = 0; i <= N; i++) {
        if (mode == 0) {
            const double t = (double)i * N_inv;
            double xa[3], xb[3];
            for (int d = 0; d < 3; d++) {
                xa[d] = ri + (sa[d] - ri) * t;
                xb[d] = rj + (sb[d] - rj) * t;
            }
            body_shape(A, xa, 2.0 + (na - 2.0) * t);
            body_shape(B, xb, 2.0 + (nb - 2.0) * t);
        }
        const double pre[3] = {cp[0], cp[1], cp[2]};
        newton_solve<MAXIT>(A, B, ratio, pre, mode == 1 && have_mu, guess_mu, o);
        for (int k = 0; k < 3; k++) cp[k] = o.point[k];
        iters += o.iters;
        solves++;
    }
}

// oriented bounding boxes intersect (15 separating axes, half-axes x 1.0001)
__device__ __forceinline__ bool obb_intersect(const double *ca, const double *Ra, const double *sa, const double *cb,
                                              const double *Rb, const double *sb)
{
    const double T[3] = {ca[0] - cb[0], ca[1] - cb[1], ca[2] - cb[2]};
    double a[3], b[3], C[9], AC[9], TA[3], TB[3];
    for (int d = 0; d < 3; d++) {
        a[d] = sa[d] * 1.0001;
        b[d] = sb[d] * 1.0001;
    }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            C[3 * i + j] = Ra[0 * 3 + i] * Rb[0 * 3 + j] + Ra[1 * 3 + i] * Rb[1 * 3 + j] + Ra[2 * 3 + i] * Rb[2 * 3 + j];
            AC[3 * i + j] = fabs(C[3 * i + j]);
        }
    tmatvec(Ra, T, TA);
    tmatvec(Rb, T, TB);
    for (int i = 0; i < 3; i++)
        if (fabs(TA[i]) > a[i] + (b[0] * AC[3 * i] + b[1] * AC[3 * i + 1] + b[2] * AC[3 * i + 2])) return false;
    for (int j = 0; j < 3; j++)
        if (fabs(TB[j]) > (a[0] * AC[j] + a[1] * AC[3 + j] + a[2] * AC[6 + j]) + b[j]) return false;
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 3; j++) {
            const int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
            const double ra = a[i1] * AC[3 * i2 + j] + a[i2] * AC[3 * i1 + j];
            const double rb = b[j1] * AC[3 * i + j2] + b[j2] * AC[3 * i + j1];
            if (fabs(TA[i2] * C[3 * i1 + j] - TA[i1] * C[3 * i2 + j]) > ra + rb) return false;
        }
    return true;
}

// Superquadric::surface_line_intersection with 20 iterations: the parameter
// alpha where start + alpha * dir meets the surface (Newton with halving)
__device__ __forceinline__ double line_intersection(const Body &b, const double *start, const double *dir,
                                                    double alpha_prev, double *result)
{
    double sl[3], dl[3], point[3], gl[3];
    to_local(b, start, sl);
    tmatvec(b.rot, dir, dl);
    double alpha = alpha_prev;
    const double eps0 = 1e-14;
    if (comp_double(b.n, 2.0, 1e-2)) {
        const double x0 = sl[0] * b.inv[0], nx = dl[0] * b.inv[0];
        const double y0 = sl[1] * b.inv[1], ny = dl[1] * b.inv[1];
        const double z0 = sl[2] * b.inv[2], nz = dl[2] * b.inv[2];
        const double qa = nx * nx + ny * ny + nz * nz, qb = 2.0 * (x0 * nx + y0 * ny + z0 * nz);
        const double qc = x0 * x0 + y0 * y0 + z0 * z0 - 1.0;
        const double D = qb * qb - 4.0 * qa * qc, tai = 0.5 / qa;
        double a1, a2;
        if (D < 0) {
            a1 = -qb * tai;
            a2 = a1;
        } else {
            const double sD = sqrt(D);
            a1 = (-qb + sD) * tai;
            a2 = (-qb - sD) * tai;
        }
        if (a1 > -eps0 && a2 < -eps0) alpha = a1;
        else if (a1 < -eps0 && a2 > -eps0) alpha = a2;
        else if (a1 < -eps0 && a2 < -eps0) alpha = fmax(a1, a2);
        else alpha = fmin(a1, a2);
    } else {
        const double a = 0.5 * fmin(fmin(b.shape[0], b.shape[1]), b.shape[2]) / sqrt(dot3(dir, dir));
        const double eps = 1e-16;
        alpha = alpha < -a ? -a : (alpha > a ? a : alpha);
        for (int k = 0; k < 3; k++) point[k] = sl[k] + alpha * dl[k];
        double f0 = f_local(b, point);
        if (!(fabs(f0) < eps)) {
            for (int it = 0; it < 20; it++) {
                if (fabs(f0) < eps * b.koef) break;
                grad_local(b, point, gl);
                const double f_der = dot3(gl, dl);
                double delta;
                if (fabs(f_der) < 1e-10) {
                    delta = 1e-10;
                    double p_[3], g_[3];
                    for (int k = 0; k < 3; k++) p_[k] = point[k] + delta * dl[k];
                    grad_local(b, p_, g_);
                    if (dot3(g_, dl) < 0.0) delta = -delta;
                } else {
                    delta = -f0 / f_der;
                    delta = delta < -a ? -a : (delta > a ? a : delta);
                }
                if (fabs(delta) <= eps) {
                    alpha += delta;
                    for (int k = 0; k < 3; k++) point[k] = point[k] + delta * dl[k];
                    break;
                }
                int halvings = 0;
                while (fabs(delta) > eps && halvings < 80) {
                    double p_[3];
                    for (int k = 0; k < 3; k++) p_[k] = point[k] + delta * dl[k];
                    const double f_ = f_local(b, p_);
                    if (fabs(f_) < fabs(f0) || fabs(f_) < eps * b.koef) {
                        f0 = f_;
                        alpha += delta;
                        for (int k = 0; k < 3; k++) point[k] = p_[k];
                        break;
                    }
                    delta *= 0.5;
                    halvings++;
                }
            }
        }
    }
    for (int k = 0; k < 3; k++) result[k] = start[k] + alpha * dir[k];
    return alpha;
}

// FixNVEAsphereBase, integration_scheme 1 helpers (src/math_extra.h, src/math_extra_liggghts_nonspherical.cpp:175)
__device__ __forceinline__ void quatvec(const double *a, const double *b, double *c)
{
    c[0] = -a[1] * b[0] - a[2] * b[1] - a[3] * b[2];
    c[1] = a[0] * b[0] + a[2] * b[2] - a[3] * b[1];
    c[2] = a[0] * b[1] + a[3] * b[0] - a[1] * b[2];
    c[3] = a[0] * b[2] + a[1] * b[1] - a[2] * b[0];
}
__device__ __forceinline__ void invquatvec(const double *a, const double *b, double *c)
{
    c[0] = -a[1] * b[0] + a[0] * b[1] + a[3] * b[2] - a[2] * b[3];
    c[1] = -a[2] * b[0] - a[3] * b[1] + a[0] * b[2] + a[1] * b[3];
    c[2] = -a[3] * b[0] + a[2] * b[1] - a[1] * b[2] + a[0] * b[3];
}
__device__ __forceinline__ void no_squish_rotate(int k, double *p, double *q, const double *inertia, double dt)
{
    double kp[4] = {0, 0, 0, 0}, kq[4] = {0, 0, 0, 0};
    if (k == 1) {
        kq[0] = -q[1]; kp[0] = -p[1]; kq[1] = q[0]; kp[1] = p[0];
        kq[2] = q[3]; kp[2] = p[3]; kq[3] = -q[2]; kp[3] = -p[2];
    } else if (k == 2) {
        kq[0] = -q[2]; kp[0] = -p[2]; kq[1] = -q[3]; kp[1] = -p[3];
        kq[2] = q[0]; kp[2] = p[0]; kq[3] = q[1]; kp[3] = p[1];
    } else {
        kq[0] = -q[3]; kp[0] = -p[3]; kq[1] = q[2]; kp[1] = p[2];
        kq[2] = -q[1]; kp[2] = -p[1]; kq[3] = q[0]; kp[3] = p[0];
    }
    double phi = p[0] * kq[0] + p[1] * kq[1] + p[2] * kq[2] + p[3] * kq[3];
    phi /= 4.0 * inertia[k - 1];
    double s_phi, c_phi;
    sincos(dt * phi, &s_phi, &c_phi);
    for (int m = 0; m < 4; m++) {
        const double pm = c_phi * p[m] + s_phi * kp[m];
        const double qm = c_phi * q[m] + s_phi * kq[m];
        p[m] = pm;
        q[m] = qm;
    }
}

}  // namespace sq
}  // namespace gb2
