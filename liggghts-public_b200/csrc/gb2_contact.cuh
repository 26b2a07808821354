// gb2_contact.cuh -- device contact models of the granular hot path.
//
// Hertz normal force, tangential history (Coulomb-capped shear spring) and
// CDT rolling friction for sphere pairs and sphere-wall contacts.  The
// statement order follows the reference model chain
// surface -> normal -> tangential -> rolling (src/contact_models.h:228-238):
//   surface default   src/surface_model_default.h:150-204
//   normal hertz      src/normal_model_hertz.h:202-393
//   tangential history src/tangential_model_history.h:130-339
//   rolling cdt       src/rolling_model_cdt.h:89-159
// Kernels that include this file are compiled with --fmad=false in the FP64
// path so every product and sum is rounded exactly as the reference CPU
// code rounds it.
#pragma once

#include <cuda_runtime.h>

namespace gb2 {

// per type-pair material constants, resolved on the host exactly as
// MODEL_PARAMS::createYeff/createGeff/createBetaEff do
struct MatPair {
    double Yeff, Geff, betaeff, mu, mur;
};

struct ContactOut {
    double F[3];
    double T[3];
};

#ifdef __CUDACC__   // device code; host-only units see the structs

// sqrt(5/6) as written in src/normal_model_hertz.h:235
#define GB2_SQRT_FIVE_OVER_SIX 0.91287092917527685576161630466800355658790782499663875

// One sphere-sphere contact seen from particle "i" (the half-list owner in
// the reference, or the j-particle when a reverse entry is evaluated from
// its own side with negated shear -- bit-identical to the reference's
// j_forces, see the engine notes).  Adds i's force and torque to `out`
// in the reference's accumulation order and updates `shear` in place when
// update_history is set.  Returns nothing; the caller applies the
// rsq < radsum^2 broad phase.
template <bool ACCUM = true>
__device__ __forceinline__ void pair_contact(const MatPair &M, double delx, double dely, double delz, double rsq,
                                             double radi, double radj, const double vi[3], const double vj[3],
                                             const double wi[3], const double wj[3], double mi, double mj,
                                             double shear[3], bool update_history, double dt, bool rolling,
                                             bool tdamp, ContactOut &out)
{
    const double radsum = radi + radj;
    const double r = sqrt(rsq);
    const double rinv = 1.0 / r;
    const double enx = delx * rinv;
    const double eny = dely * rinv;
    const double enz = delz * rinv;
    const double meff = mi * mj / (mi + mj);

    // ---- surface model (sphere kinematics)
    const double vr1 = vi[0] - vj[0];
    const double vr2 = vi[1] - vj[1];
    const double vr3 = vi[2] - vj[2];
    const double vn = vr1 * enx + vr2 * eny + vr3 * enz;
    const double vn1 = vn * enx;
    const double vn2 = vn * eny;
    const double vn3 = vn * enz;
    const double vt1 = vr1 - vn1;
    const double vt2 = vr2 - vn2;
    const double vt3 = vr3 - vn3;
    const double deltan = radsum - r;
    const double cri = radi - 0.5 * deltan;
    const double crj = radj - 0.5 * deltan;
    const double wr1 = (cri * wi[0] + crj * wj[0]) * rinv;
    const double wr2 = (cri * wi[1] + crj * wj[1]) * rinv;
    const double wr3 = (cri * wi[2] + crj * wj[2]) * rinv;
    const double vtr1 = vt1 - (delz * wr2 - dely * wr3);
    const double vtr2 = vt2 - (delx * wr3 - delz * wr1);
    const double vtr3 = vt3 - (dely * wr1 - delx * wr2);

    // ---- normal model (Hertz)
    const double reff = radi * radj / (radi + radj);
    const double sqrtval = sqrt(reff * deltan);
    const double Sn = 2. * M.Yeff * sqrtval;
    const double St = 8. * M.Geff * sqrtval;
    double kn = 4. / 3. * M.Yeff * sqrtval;
    double kt = St;
    const double gamman = -2. * GB2_SQRT_FIVE_OVER_SIX * M.betaeff * sqrt(Sn * meff);
    const double gammat = tdamp ? -2. * GB2_SQRT_FIVE_OVER_SIX * M.betaeff * sqrt(St * meff) : 0.0;
    kn /= 1.0;   // force->nktv2p = 1 (si)
    kt /= 1.0;
    const double Fn_damping = -gamman * vn;
    const double Fn_contact = kn * deltan;
    const double Fn = Fn_damping + Fn_contact;
    double F0 = 0.0, F1 = 0.0, F2 = 0.0;
    F0 += Fn * enx;
    F1 += Fn * eny;
    F2 += Fn * enz;

    // ---- tangential model (history)
    if (update_history) {
        shear[0] += vtr1 * dt;
        shear[1] += vtr2 * dt;
        shear[2] += vtr3 * dt;
        const double rsht = shear[0] * enx + shear[1] * eny + shear[2] * enz;
        shear[0] -= rsht * enx;
        shear[1] -= rsht * eny;
        shear[2] -= rsht * enz;
    }
    const double shrmag = sqrt(shear[0] * shear[0] + shear[1] * shear[1] + shear[2] * shear[2]);
    double Ft1 = -(kt * shear[0]);
    double Ft2 = -(kt * shear[1]);
    double Ft3 = -(kt * shear[2]);
    const double Ft_shear = kt * shrmag;
    const double Ft_friction = M.mu * fabs(Fn);
    if (Ft_shear > Ft_friction) {
        if (shrmag != 0.0) {
            const double ratio = Ft_friction / Ft_shear;
            Ft1 *= ratio;
            Ft2 *= ratio;
            Ft3 *= ratio;
            if (update_history) {
                shear[0] = -Ft1 / kt;
                shear[1] = -Ft2 / kt;
                shear[2] = -Ft3 / kt;
            }
        } else {
            Ft1 = Ft2 = Ft3 = 0.0;
        }
    } else {
        Ft1 -= (gammat * vtr1);
        Ft2 -= (gammat * vtr2);
        Ft3 -= (gammat * vtr3);
    }
    const double tor1 = eny * Ft3 - enz * Ft2;
    const double tor2 = enz * Ft1 - enx * Ft3;
    const double tor3 = enx * Ft2 - eny * Ft1;
    double T0 = 0.0, T1 = 0.0, T2 = 0.0;
    F0 += Ft1;
    F1 += Ft2;
    F2 += Ft3;
    T0 += -cri * tor1;
    T1 += -cri * tor2;
    T2 += -cri * tor3;

    // ---- rolling model (CDT, torsion torque off)
    if (rolling) {
        double rt0 = 0., rt1 = 0., rt2 = 0.;
        const double wrr0 = wi[0] - wj[0];
        const double wrr1 = wi[1] - wj[1];
        const double wrr2 = wi[2] - wj[2];
        const double wrmag = sqrt(wrr0 * wrr0 + wrr1 * wrr1 + wrr2 * wrr2);
        if (wrmag > 0.) {
            const double sc = M.mur * kn * deltan * reff / wrmag;
            rt0 = sc * wrr0;
            rt1 = sc * wrr1;
            rt2 = sc * wrr2;
            const double d = rt0 * enx + rt1 * eny + rt2 * enz;
            const double rn0 = enx * d, rn1 = eny * d, rn2 = enz * d;
            rt0 = rt0 - rn0;
            rt1 = rt1 - rn1;
            rt2 = rt2 - rn2;
        }
        T0 -= rt0;
        T1 -= rt1;
        T2 -= rt2;
    }
    if (ACCUM) {
        out.F[0] += F0;
        out.F[1] += F1;
        out.F[2] += F2;
        out.T[0] += T0;
        out.T[1] += T1;
        out.T[2] += T2;
    } else {   // the pair's own contribution, for a later in-order sum
        out.F[0] = F0;
        out.F[1] = F1;
        out.F[2] = F2;
        out.T[0] = T0;
        out.T[1] = T1;
        out.T[2] = T2;
    }
}

struct ContactOutF {
    float F[3];
    float T[3];
};

// Split-precision form of pair_contact: the same model chain (surface
// default -> Hertz -> tangential history -> CDT rolling), evaluated in FP32
// on operands the caller prepares in FP64 -- the relative position
// del = x_i - x_j, its length r and the overlap deltan = radsum - r are
// differenced in FP64 and only then rounded, so the near-touching overlap
// (a difference of two nearly equal FP64 lengths) keeps its accuracy.  The
// pair's own contribution is returned in `out` (for an in-order Kahan sum
// by the caller); `shear` is updated in place when update_history is set.
__device__ __forceinline__ void pair_contact_f32(const MatPair &M, float delx, float dely, float delz, float r,
                                                 float deltan, float radi, float radj, const float vi[3],
                                                 const float vj[3], const float wi[3], const float wj[3], float mi,
                                                 float mj, float shear[3], bool update_history, float dt,
                                                 bool rolling, bool tdamp, ContactOutF &out)
{
    const float rinv = 1.0f / r;
    const float enx = delx * rinv;
    const float eny = dely * rinv;
    const float enz = delz * rinv;
    const float meff = mi * mj / (mi + mj);

    // surface model
    const float vr1 = vi[0] - vj[0];
    const float vr2 = vi[1] - vj[1];
    const float vr3 = vi[2] - vj[2];
    const float vn = vr1 * enx + vr2 * eny + vr3 * enz;
    const float vt1 = vr1 - vn * enx;
    const float vt2 = vr2 - vn * eny;
    const float vt3 = vr3 - vn * enz;
    const float cri = radi - 0.5f * deltan;
    const float crj = radj - 0.5f * deltan;
    const float wr1 = (cri * wi[0] + crj * wj[0]) * rinv;
    const float wr2 = (cri * wi[1] + crj * wj[1]) * rinv;
    const float wr3 = (cri * wi[2] + crj * wj[2]) * rinv;
    const float vtr1 = vt1 - (delz * wr2 - dely * wr3);
    const float vtr2 = vt2 - (delx * wr3 - delz * wr1);
    const float vtr3 = vt3 - (dely * wr1 - delx * wr2);

    // normal model (Hertz)
    const float Yeff = (float)M.Yeff, Geff = (float)M.Geff, beta = (float)M.betaeff;
    const float reff = radi * radj / (radi + radj);
    const float sqrtval = sqrtf(reff * deltan);
    const float Sn = 2.f * Yeff * sqrtval;
    const float St = 8.f * Geff * sqrtval;
    const float kn = (4.f / 3.f) * Yeff * sqrtval;
    const float kt = St;
    const float c56 = (float)GB2_SQRT_FIVE_OVER_SIX;
    const float gamman = -2.f * c56 * beta * sqrtf(Sn * meff);
    const float gammat = tdamp ? -2.f * c56 * beta * sqrtf(St * meff) : 0.f;
    const float Fn = -gamman * vn + kn * deltan;
    float F0 = Fn * enx, F1 = Fn * eny, F2 = Fn * enz;

    // tangential model (history)
    if (update_history) {
        shear[0] += vtr1 * dt;
        shear[1] += vtr2 * dt;
        shear[2] += vtr3 * dt;
        const float rsht = shear[0] * enx + shear[1] * eny + shear[2] * enz;
        shear[0] -= rsht * enx;
        shear[1] -= rsht * eny;
        shear[2] -= rsht * enz;
    }
    const float shrmag = sqrtf(shear[0] * shear[0] + shear[1] * shear[1] + shear[2] * shear[2]);
    float Ft1 = -(kt * shear[0]);
    float Ft2 = -(kt * shear[1]);
    float Ft3 = -(kt * shear[2]);
    const float Ft_shear = kt * shrmag;
    const float Ft_friction = (float)M.mu * fabsf(Fn);
    if (Ft_shear > Ft_friction) {
        if (shrmag != 0.f) {
            const float ratio = Ft_friction / Ft_shear;
            Ft1 *= ratio;
            Ft2 *= ratio;
            Ft3 *= ratio;
            if (update_history) {
                const float ktinv = 1.0f / kt;
                shear[0] = -Ft1 * ktinv;
                shear[1] = -Ft2 * ktinv;
                shear[2] = -Ft3 * ktinv;
            }
        } else {
            Ft1 = Ft2 = Ft3 = 0.f;
        }
    } else {
        Ft1 -= gammat * vtr1;
        Ft2 -= gammat * vtr2;
        Ft3 -= gammat * vtr3;
    }
    F0 += Ft1;
    F1 += Ft2;
    F2 += Ft3;
    float T0 = -cri * (eny * Ft3 - enz * Ft2);
    float T1 = -cri * (enz * Ft1 - enx * Ft3);
    float T2 = -cri * (enx * Ft2 - eny * Ft1);

    // rolling model (CDT)
    if (rolling) {
        const float wrr0 = wi[0] - wj[0];
        const float wrr1 = wi[1] - wj[1];
        const float wrr2 = wi[2] - wj[2];
        const float wr2sum = wrr0 * wrr0 + wrr1 * wrr1 + wrr2 * wrr2;
        if (wr2sum > 0.f) {
            const float sc = (float)M.mur * kn * deltan * reff * rsqrtf(wr2sum);
            float rt0 = sc * wrr0, rt1 = sc * wrr1, rt2 = sc * wrr2;
            const float d = rt0 * enx + rt1 * eny + rt2 * enz;
            rt0 -= enx * d;
            rt1 -= eny * d;
            rt2 -= enz * d;
            T0 -= rt0;
            T1 -= rt1;
            T2 -= rt2;
        }
    }
    out.F[0] = F0;
    out.F[1] = F1;
    out.F[2] = F2;
    out.T[0] = T0;
    out.T[1] = T1;
    out.T[2] = T2;
}

// Sphere-wall contact (primitive plane or mesh triangle), following
// Walls::Granular::compute_force (src/fix_wall_gran_base.h:148-306) and the
// is_wall branches of the model chain.  `d` is the vector from the wall
// contact point to the sphere centre (the negated resolveContact delta),
// `overlap` the positive overlap (-deltan).  vwall is the wall velocity at
// the contact point.
__device__ __forceinline__ void wall_contact(const MatPair &M, const double d[3], double overlap, double radi,
                                             const double vi[3], const double wi[3], const double vwall[3],
                                             double mass, double shear[3], bool update_history, double dt,
                                             bool rolling, bool tdamp, ContactOut &out)
{
    const double r = radi - overlap;
    const double rinv = 1.0 / r;
    const double enx = d[0] * rinv;
    const double eny = d[1] * rinv;
    const double enz = d[2] * rinv;
    const double radsum = radi;

    // ---- surface model, wall branch
    const double vr1 = vi[0] - vwall[0];
    const double vr2 = vi[1] - vwall[1];
    const double vr3 = vi[2] - vwall[2];
    const double vn = vr1 * enx + vr2 * eny + vr3 * enz;
    const double vn1 = vn * enx;
    const double vn2 = vn * eny;
    const double vn3 = vn * enz;
    const double vt1 = vr1 - vn1;
    const double vt2 = vr2 - vn2;
    const double vt3 = vr3 - vn3;
    const double deltan = radsum - r;       // recomputed overlap, stored back as sidata.deltan
    const double cr = radi - 0.5 * overlap; // uses the overlap handed in
    const double wr1 = cr * wi[0] * rinv;
    const double wr2 = cr * wi[1] * rinv;
    const double wr3 = cr * wi[2] * rinv;
    const double vtr1 = vt1 - (d[2] * wr2 - d[1] * wr3);
    const double vtr2 = vt2 - (d[0] * wr3 - d[2] * wr1);
    const double vtr3 = vt3 - (d[1] * wr1 - d[0] * wr2);

    // ---- normal model, wall branch (reff = radi, meff = particle mass)
    const double reff = radi;
    const double sqrtval = sqrt(reff * deltan);
    const double Sn = 2. * M.Yeff * sqrtval;
    const double St = 8. * M.Geff * sqrtval;
    double kn = 4. / 3. * M.Yeff * sqrtval;
    double kt = St;
    const double gamman = -2. * GB2_SQRT_FIVE_OVER_SIX * M.betaeff * sqrt(Sn * mass);
    const double gammat = tdamp ? -2. * GB2_SQRT_FIVE_OVER_SIX * M.betaeff * sqrt(St * mass) : 0.0;
    kn /= 1.0;
    kt /= 1.0;
    const double Fn_damping = -gamman * vn;
    const double Fn_contact = kn * deltan;
    const double Fn = Fn_damping + Fn_contact;
    double F0 = 0.0, F1 = 0.0, F2 = 0.0;
    const double Fn_ = Fn * 1.0;   // area_ratio
    F0 += Fn_ * enx;
    F1 += Fn_ * eny;
    F2 += Fn_ * enz;

    // ---- tangential model
    if (update_history) {
        shear[0] += vtr1 * dt;
        shear[1] += vtr2 * dt;
        shear[2] += vtr3 * dt;
        const double rsht = shear[0] * enx + shear[1] * eny + shear[2] * enz;
        shear[0] -= rsht * enx;
        shear[1] -= rsht * eny;
        shear[2] -= rsht * enz;
    }
    const double shrmag = sqrt(shear[0] * shear[0] + shear[1] * shear[1] + shear[2] * shear[2]);
    double Ft1 = -(kt * shear[0]);
    double Ft2 = -(kt * shear[1]);
    double Ft3 = -(kt * shear[2]);
    const double Ft_shear = kt * shrmag;
    const double Ft_friction = M.mu * fabs(Fn);
    if (Ft_shear > Ft_friction) {
        if (shrmag != 0.0) {
            const double ratio = Ft_friction / Ft_shear;
            Ft1 *= ratio;
            Ft2 *= ratio;
            Ft3 *= ratio;
            if (update_history) {
                shear[0] = -Ft1 / kt;
                shear[1] = -Ft2 / kt;
                shear[2] = -Ft3 / kt;
            }
        } else {
            Ft1 = Ft2 = Ft3 = 0.0;
        }
    } else {
        Ft1 -= (gammat * vtr1);
        Ft2 -= (gammat * vtr2);
        Ft3 -= (gammat * vtr3);
    }
    const double tor1 = eny * Ft3 - enz * Ft2;
    const double tor2 = enz * Ft1 - enx * Ft3;
    const double tor3 = enx * Ft2 - eny * Ft1;
    double T0 = 0.0, T1 = 0.0, T2 = 0.0;
    F0 += Ft1 * 1.0;
    F1 += Ft2 * 1.0;
    F2 += Ft3 * 1.0;
    T0 += (-cr * tor1) * 1.0;
    T1 += (-cr * tor2) * 1.0;
    T2 += (-cr * tor3) * 1.0;

    // ---- rolling model, wall branch
    if (rolling) {
        double rt0 = 0., rt1 = 0., rt2 = 0.;
        const double wrmag = sqrt(wr1 * wr1 + wr2 * wr2 + wr3 * wr3);
        if (wrmag > 0.) {
            const double Fnr = deltan * kn;
            rt0 = M.mur * Fnr * wr1 / wrmag * reff;
            rt1 = M.mur * Fnr * wr2 / wrmag * reff;
            rt2 = M.mur * Fnr * wr3 / wrmag * reff;
            const double dd = rt0 * enx + rt1 * eny + rt2 * enz;
            const double rn0 = enx * dd, rn1 = eny * dd, rn2 = enz * dd;
            rt0 = rt0 - rn0;
            rt1 = rt1 - rn1;
            rt2 = rt2 - rn2;
        }
        T0 -= rt0;
        T1 -= rt1;
        T2 -= rt2;
    }
    // force_update of the wall style: f += delta_F, torque += delta_torque
    out.F[0] += F0;
    out.F[1] += F1;
    out.F[2] += F2;
    out.T[0] += T0;
    out.T[1] += T1;
    out.T[2] += T2;
}

#endif  // __CUDACC__

}  // namespace gb2
