// gb2_sq_kernels.cuh -- kernels of the superquadric time step.
//
// Layout (structure of arrays, 32-byte records):
//   per atom: x {x, y, z, rbound}, v {vx, vy, vz, m}, q {w, i, j, k},
//             L {angmom, -}, w {omega, -}, f, t, shape {a, b, c, n},
//             inert {Ixx, Iyy, Izz, rvol}, xhold
//   half list in CSR form by owner i (neighbours j > i, ascending):
//             start[i] .. start[i+1], nbr[s]; per slot s the contact history
//             flag, state (far/close/intersect), cp {contact point, -},
//             alpha {alphaA, alphaB}, shear {s0, s1, s2, -}
//   per slot results of the pair pass: fi (force on i), ti, tj (torques)
//   reverse CSR by j: rstart[j] .. rstart[j+1], rslot[r] = slot index (ascending i)
#pragma once

#include "gb2_sq.cuh"
#include "gb2_internal.h"
#include "gb2_mma.cuh"

namespace gb2 {
namespace sq {

struct SqDev {
    int n;
    dbl4 *x, *v, *q, *L, *w, *f, *t, *shape, *inert, *xhold;
    // list
    int *start, *nbr, *flag, *state;
    dbl4 *cp, *shear;
    double2 *alpha;
    dbl4 *pfi, *pti, *ptj;
    int *rstart, *rslot;
    // physics
    double dt, skin, triggersq;
    double Yeff, Geff, betaeff, mu;
    // counters: iterations, solves, pairs solved, learned guesses used, learned guesses rejected
    unsigned long long *cnt;
    int *dflag;
    // learned initial guess (null when off)
    const float *mlp;
};

// FixNVEAsphereBase::initial_integrate, integration_scheme 1
// (src/fix_nve_asphere_base.cpp:319-444), and Neighbor::check_distance
__global__ void k_sq_initial(SqDev D, int check)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.n) return;
    const double dtv = D.dt, dtf = 0.5 * D.dt * 1.0, dtf2 = 2.0 * dtf, dtq = 0.5 * dtv;
    dbl4 x = D.x[i], v = D.v[i], q4 = D.q[i];
    const dbl4 f = D.f[i], tq = D.t[i], in4 = D.inert[i], L4 = D.L[i];
    double q[4] = {q4.x, q4.y, q4.z, q4.w};
    const double in[3] = {in4.x, in4.y, in4.z};
    double R[9], mbody[3], conjqm[4], tbody[3], fquat[4], wbody[3];
    quat_to_mat(q, R);
    const double dtfm = dtf / v.w;
    v.x += dtfm * f.x;
    v.y += dtfm * f.y;
    v.z += dtfm * f.z;
    x.x += dtv * v.x;
    x.y += dtv * v.y;
    x.z += dtv * v.z;
    const double Lv[3] = {L4.x, L4.y, L4.z}, Tv[3] = {tq.x, tq.y, tq.z};
    tmatvec(R, Lv, mbody);
    quatvec(q, mbody, conjqm);
    for (int k = 0; k < 4; k++) conjqm[k] *= 2.0;
    tmatvec(R, Tv, tbody);
    quatvec(q, tbody, fquat);
    for (int k = 0; k < 4; k++) conjqm[k] += dtf2 * fquat[k];
    no_squish_rotate(3, conjqm, q, in, dtq);
    no_squish_rotate(2, conjqm, q, in, dtq);
    no_squish_rotate(1, conjqm, q, in, dtv);
    no_squish_rotate(2, conjqm, q, in, dtq);
    no_squish_rotate(3, conjqm, q, in, dtq);
    const double norm = 1.0 / sqrt(q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3]);
    for (int k = 0; k < 4; k++) q[k] *= norm;
    quat_to_mat(q, R);
    invquatvec(q, conjqm, mbody);
    for (int d = 0; d < 3; d++) mbody[d] *= 0.5;
    for (int d = 0; d < 3; d++) wbody[d] = mbody[d] / in[d];
    double Lo[3], wo[3];
    matvec(R, mbody, Lo);
    matvec(R, wbody, wo);
    D.x[i] = x;
    D.v[i] = v;
    D.q[i] = dbl4{q[0], q[1], q[2], q[3]};
    D.L[i] = dbl4{Lo[0], Lo[1], Lo[2], 0.0};
    D.w[i] = dbl4{wo[0], wo[1], wo[2], 0.0};
    if (check) {
        const dbl4 h = D.xhold[i];
        const double dx = x.x - h.x, dy = x.y - h.y, dz = x.z - h.z;
        if (dx * dx + dy * dy + dz * dz > D.triggersq) *D.dflag = 1;
    }
}

// FixNVEAsphereBase::final_integrate, integration_scheme 1 (:523-620)
__global__ void k_sq_final(SqDev D)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.n) return;
    const double dtf = 0.5 * D.dt * 1.0, dtf2 = dtf * 2.0;
    dbl4 v = D.v[i];
    const dbl4 q4 = D.q[i], f = D.f[i], tq = D.t[i], in4 = D.inert[i], L4 = D.L[i];
    const double q[4] = {q4.x, q4.y, q4.z, q4.w};
    const double in[3] = {in4.x, in4.y, in4.z};
    double R[9], tbody[3], mbody[3], conjqm[4], fquat[4], wbody[3];
    const double dtfm = dtf / v.w;
    quat_to_mat(q, R);
    v.x += dtfm * f.x;
    v.y += dtfm * f.y;
    v.z += dtfm * f.z;
    const double Tv[3] = {tq.x, tq.y, tq.z}, Lv[3] = {L4.x, L4.y, L4.z};
    tmatvec(R, Tv, tbody);
    tmatvec(R, Lv, mbody);
    quatvec(q, mbody, conjqm);
    for (int k = 0; k < 4; k++) conjqm[k] *= 2.0;
    quatvec(q, tbody, fquat);
    for (int k = 0; k < 4; k++) conjqm[k] += dtf2 * fquat[k];
    invquatvec(q, conjqm, mbody);
    for (int d = 0; d < 3; d++) mbody[d] *= 0.5;
    for (int d = 0; d < 3; d++) wbody[d] = mbody[d] / in[d];
    double Lo[3], wo[3];
    matvec(R, mbody, Lo);
    matvec(R, wbody, wo);
    D.v[i] = v;
    D.L[i] = dbl4{Lo[0], Lo[1], Lo[2], 0.0};
    D.w[i] = dbl4{wo[0], wo[1], wo[2], 0.0};
}

// omega from angular momentum (set-up)
__global__ void k_sq_omega(SqDev D)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= D.n) return;
    const dbl4 q4 = D.q[i], L4 = D.L[i], in4 = D.inert[i];
    const double q[4] = {q4.x, q4.y, q4.z, q4.w}, Lv[3] = {L4.x, L4.y, L4.z};
    double R[9], mb[3], wb[3], wo[3];
    quat_to_mat(q, R);
    tmatvec(R, Lv, mb);
    wb[0] = mb[0] / in4.x;
    wb[1] = mb[1] / in4.y;
    wb[2] = mb[2] / in4.z;
    matvec(R, wb, wo);
    D.w[i] = dbl4{wo[0], wo[1], wo[2], 0.0};
}

// ------------------------------------------------------------------
// learned initial guess: MLP 14 -> 64 -> 64 -> 64 -> 4 (ReLU), BF16 weights
// and activations with FP32 accumulation, parameters packed as
//   in_mean[14] in_std[14] out_mean[4] out_std[4]
//   W1[64][14] b1[64] W2[64][64] b2[64] W3[64][64] b3[64] W4[4][64] b4[4]
constexpr int kMlpIn = 14, kMlpH = 64, kMlpOut = 4;
constexpr int kMlpOffW1 = 36, kMlpOffB1 = kMlpOffW1 + kMlpH * kMlpIn, kMlpOffW2 = kMlpOffB1 + kMlpH,
              kMlpOffB2 = kMlpOffW2 + kMlpH * kMlpH, kMlpOffW3 = kMlpOffB2 + kMlpH,
              kMlpOffB3 = kMlpOffW3 + kMlpH * kMlpH, kMlpOffW4 = kMlpOffB3 + kMlpH,
              kMlpOffB4 = kMlpOffW4 + kMlpOut * kMlpH, kMlpSize = kMlpOffB4 + kMlpOut;

__device__ __forceinline__ float bf16_round(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

// pair features in particle i's body frame, lengths over s = ri + rj
// (ri = cbrt(abc)): centre of j (3), rotation vector of q_i^-1 q_j (3),
// half-axes of i and j (6), (n - 2) / 6 of i and j (2)
__device__ __forceinline__ double pair_features(const double *ci, const double *qi, const double *si, double ni,
                                                const double *cj, const double *qj, const double *sj, double nj,
                                                const double *Ri, float *feat)
{
    const double ri = cbrt(si[0] * si[1] * si[2]), rj = cbrt(sj[0] * sj[1] * sj[2]);
    const double s = ri + rj, sinv = 1.0 / s;
    const double d[3] = {cj[0] - ci[0], cj[1] - ci[1], cj[2] - ci[2]};
    double dl[3];
    tmatvec(Ri, d, dl);
    // q_rel = conj(q_i) * q_j
    const double a0 = qi[0], a1 = -qi[1], a2 = -qi[2], a3 = -qi[3];
    double r0 = a0 * qj[0] - a1 * qj[1] - a2 * qj[2] - a3 * qj[3];
    double r1 = a0 * qj[1] + qj[0] * a1 + a2 * qj[3] - a3 * qj[2];
    double r2 = a0 * qj[2] + qj[0] * a2 + a3 * qj[1] - a1 * qj[3];
    double r3 = a0 * qj[3] + qj[0] * a3 + a1 * qj[2] - a2 * qj[1];
    if (r0 < 0) {
        r0 = -r0;
        r1 = -r1;
        r2 = -r2;
        r3 = -r3;
    }
    const double vn = sqrt(r1 * r1 + r2 * r2 + r3 * r3);
    const double ang = 2.0 * atan2(vn, r0);
    const double k = vn > 0 ? ang / vn : 2.0;
    feat[0] = (float)(dl[0] * sinv);
    feat[1] = (float)(dl[1] * sinv);
    feat[2] = (float)(dl[2] * sinv);
    feat[3] = (float)(k * r1);
    feat[4] = (float)(k * r2);
    feat[5] = (float)(k * r3);
    for (int c = 0; c < 3; c++) {
        feat[6 + c] = (float)(si[c] * sinv);
        feat[9 + c] = (float)(sj[c] * sinv);
    }
    feat[12] = (float)((ni - 2.0) / 6.0);
    feat[13] = (float)((nj - 2.0) / 6.0);
    return s;
}

// Inference on the tensor cores.  The parameters are staged once per block
// (weights rounded to BF16 and zero-padded exactly as the training kernel
// does), and each warp runs the forward pass of its 32 lanes' pairs as two
// 16-row tiles through the training kernel's own layers (mma.sync m16n8k16,
// FP32 accumulation, bias + ReLU, BF16 activations), so a guess is computed
// with the arithmetic the network was trained with.
struct MlpInfer {
    __nv_bfloat16 W1[kMlpH][16], W2[kMlpH][kMlpH], W3[kMlpH][kMlpH], W4[8][kMlpH];
    float b1[kMlpH], b2[kMlpH], b3[kMlpH], b4[8];
    float stat[2 * kMlpIn + 2 * kMlpOut];   // in_mean, in_std, out_mean, out_std
    __nv_bfloat16 X[4][32][16];             // per warp: normalised features
    __nv_bfloat16 H[4][2][16][kMlpH];       // per warp: activations of one tile
    float Y[4][32][kMlpOut];                // per warp: outputs
};

// all threads of the block; the caller synchronises the block afterwards
__device__ __forceinline__ void mlp_stage(MlpInfer &S, const float *__restrict__ P)
{
    const int tid = threadIdx.x, nt = blockDim.x;
    for (int e = tid; e < kMlpH * 16; e += nt) {
        const int o = e / 16, c = e % 16;
        S.W1[o][c] = __float2bfloat16_rn(c < kMlpIn ? P[kMlpOffW1 + o * kMlpIn + c] : 0.f);
    }
    for (int e = tid; e < kMlpH * kMlpH; e += nt) {
        S.W2[e / kMlpH][e % kMlpH] = __float2bfloat16_rn(P[kMlpOffW2 + e]);
        S.W3[e / kMlpH][e % kMlpH] = __float2bfloat16_rn(P[kMlpOffW3 + e]);
    }
    for (int e = tid; e < 8 * kMlpH; e += nt) {
        const int o = e / kMlpH;
        S.W4[o][e % kMlpH] = __float2bfloat16_rn(o < kMlpOut ? P[kMlpOffW4 + e] : 0.f);
    }
    for (int e = tid; e < kMlpH; e += nt) {
        S.b1[e] = P[kMlpOffB1 + e];
        S.b2[e] = P[kMlpOffB2 + e];
        S.b3[e] = P[kMlpOffB3 + e];
    }
    if (tid < 8) S.b4[tid] = tid < kMlpOut ? P[kMlpOffB4 + tid] : 0.f;
    for (int e = tid; e < 2 * kMlpIn + 2 * kMlpOut; e += nt) S.stat[e] = P[e];
}

// The forward pass of the warp's 32 lanes (called by the whole warp of a
// 128-thread block; lanes with active false contribute zero rows): out =
// de-normalised (point in i's frame / s, mu) of the lane's pair.
__device__ __forceinline__ void mlp_infer_warp(MlpInfer &S, bool active, const float *feat, float *out)
{
    const int lane = threadIdx.x & 31, w = (threadIdx.x >> 5) & 3;
    for (int c = 0; c < 16; c++) {
        const float v = (active && c < kMlpIn) ? (feat[c] - S.stat[c]) / S.stat[kMlpIn + c] : 0.f;
        S.X[w][lane][c] = __float2bfloat16_rn(v);
    }
    __syncwarp();
    const int g = lane >> 2, t = lane & 3;
    for (int tile = 0; tile < 2; tile++) {
        layer_fwd<16, kMlpH>(&S.X[w][16 * tile][0], &S.W1[0][0], S.b1, &S.H[w][0][0][0], true);
        __syncwarp();
        layer_fwd<kMlpH, kMlpH>(&S.H[w][0][0][0], &S.W2[0][0], S.b2, &S.H[w][1][0][0], true);
        __syncwarp();
        layer_fwd<kMlpH, kMlpH>(&S.H[w][1][0][0], &S.W3[0][0], S.b3, &S.H[w][0][0][0], true);
        __syncwarp();
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
        for (int k0 = 0; k0 < kMlpH; k0 += 16) {
            unsigned a[4], bb[2];
            load_a<false>(&S.H[w][0][0][0], kMlpH, 0, k0, a);
            load_b<true>(&S.W4[0][0], kMlpH, k0, 0, bb);
            mma16816(acc, a, bb);
        }
        for (int q = 0; q < 4; q++) {
            const int r = g + (q >> 1) * 8, c = 2 * t + (q & 1);
            if (c < kMlpOut) S.Y[w][16 * tile + r][c] = acc[q] + S.b4[c];
        }
        __syncwarp();
    }
    for (int c = 0; c < kMlpOut; c++)
        out[c] = S.Y[w][lane][c] * S.stat[2 * kMlpIn + kMlpOut + c] + S.stat[2 * kMlpIn + c];
    __syncwarp();
}

// Newton iterations granted to the solve from the learned guess.  A start
// the network places well converges in ~10; one that needs more is handed to
// the homotopy, whose result is the plain method's anyway, so the pairs that
// defeat both methods no longer pay the full iteration bound twice.
constexpr int kLearnedNewton = 48;

// Contact point of a pair without a previous point from the network's
// output `out` (point in i's frame / s, mu): one Newton solve of at most
// kLearnedNewton iterations.  The caller accepts it when it converged to
// merit < 1e-10 and otherwise runs the homotopy.
__device__ __forceinline__ void used_learned_guess(const float *out, const double *ci, const double *qi,
                                                   const double *si, double ni, const double *cj, const double *qj,
                                                   const double *sj, double nj, Newton &o, int &iters, int &solves)
{
    double Ri[9];
    quat_to_mat(qi, Ri);
    const double s = cbrt(si[0] * si[1] * si[2]) + cbrt(sj[0] * sj[1] * sj[2]);
    const double pl[3] = {out[0] * s, out[1] * s, out[2] * s};
    double g[3];
    matvec(Ri, pl, g);
    for (int k = 0; k < 3; k++) g[k] += ci[k];
    contact_point<kLearnedNewton>(ci, qi, si, ni, cj, qj, sj, nj, 1, g, true, (double)fabsf(out[3]), o, iters,
                                  solves);
}

// The network's features of a pair (i's body frame)
__device__ __forceinline__ void pair_features_of(const double *ci, const double *qi, const double *si, double ni,
                                                 const double *cj, const double *qj, const double *sj, double nj,
                                                 float *feat)
{
    double Ri[9];
    quat_to_mat(qi, Ri);
    pair_features(ci, qi, si, ni, cj, qj, sj, nj, Ri, feat);
}

// Contact point of a pair without a previous point in one call: the learned
// guess when the network's output is given, the homotopy when it is
// rejected or absent.  used: 1 learned guess accepted, -1 rejected, 0 off.
__device__ __forceinline__ void first_contact(const float *out, const double *ci, const double *qi, const double *si,
                                              double ni, const double *cj, const double *qj, const double *sj,
                                              double nj, Newton &o, int &iters, int &solves, int &used)
{
    used = 0;
    if (out) {
        int it1, sv1;
        used_learned_guess(out, ci, qi, si, ni, cj, qj, sj, nj, o, it1, sv1);
        if (!o.fail && o.merit < 1e-10) {
            iters = it1;
            solves = sv1;
            used = 1;
            return;
        }
        int it2, sv2;
        contact_point(ci, qi, si, ni, cj, qj, sj, nj, 0, nullptr, false, 0.0, o, it2, sv2);
        iters = it1 + it2;
        solves = sv1 + sv2;
        used = -1;
        return;
    }
    contact_point(ci, qi, si, ni, cj, qj, sj, nj, 0, nullptr, false, 0.0, o, iters, solves);
}

// ------------------------------------------------------------------
// pair pass (PairGran::compute with the superquadric surface model,
// src/pair_gran_base.h:255-430, src/surface_model_superquadric.h:108-205,
// non-spherical Hertz/history) in two kernels: k_sq_screen tests every
// half-list slot (bounding spheres, oriented boxes) and marks the slots
// that need a contact-point solve for one of two lists, first contacts and
// warm starts (a previous point exists), which stable selections gather in
// slot order; k_sq_solve runs the solves, each warp
// taking the next 32 items, first contacts first.  A step holds few solves
// (a few per cent of the slots), and its time is set by the longest solve
// chains -- first contacts through the homotopy or the learned guess -- so
// these start at once, on dense warps, and the short warm starts fill the
// GPU around them.  Every slot's result is the one-pass result (the solves
// are deterministic and independent).

// lists of one pair pass: 0 first contacts, 1 warm starts
struct SqWork {
    int *list[2];
    int *n;      // item counts, [2]
    int *next;   // items taken (over both lists)
};

// the work list a screened slot joins: 0 first contact, 1 warm start, -1 none
struct SlotKindIs {
    const signed char *kind;
    signed char want;
    __host__ __device__ bool operator()(int sl) const { return kind[sl] == want; }
};

// the slot's contact point, state and forces from a finished solve
__device__ __forceinline__ void sq_finish(const SqDev &D, int sl, int i, int j, int shearupdate, const Newton &o)
{
    D.cp[sl] = dbl4{o.point[0], o.point[1], o.point[2], 0.0};
    if (!(fmax(o.fi, o.fj) < 0.0)) {
        D.state[sl] = CLOSE;
        return;
    }
    const dbl4 xi4 = D.x[i], xj4 = D.x[j], qi4 = D.q[i], qj4 = D.q[j], si4 = D.shape[i], sj4 = D.shape[j];
    const double ci[3] = {xi4.x, xi4.y, xi4.z}, cj[3] = {xj4.x, xj4.y, xj4.z};
    const double qi[4] = {qi4.x, qi4.y, qi4.z, qi4.w}, qj[4] = {qj4.x, qj4.y, qj4.z, qj4.w};
    const double si[3] = {si4.x, si4.y, si4.z}, sj[3] = {sj4.x, sj4.y, sj4.z};
    double en[3] = {o.gB[0] - o.gA[0], o.gB[1] - o.gA[1], o.gB[2] - o.gA[2]};
    const double nrm = sqrt(en[0] * en[0] + en[1] * en[1] + en[2] * en[2]);
    const double inv = nrm == 0. ? 0. : 1. / nrm;
    for (int k = 0; k < 3; k++) en[k] *= inv;
    Body A, B;
    body_set(A, ci, qi, si, si4.w);
    body_set(B, cj, qj, sj, sj4.w);
    double2 al = D.alpha[sl];
    const double ne[3] = {-en[0], -en[1], -en[2]};
    double cpa[3], cpb[3];
    al.x = line_intersection(A, o.point, ne, al.x, cpa);
    al.y = line_intersection(B, o.point, en, al.y, cpb);
    D.alpha[sl] = al;
    const double deltan = fabs(al.x) + fabs(al.y);
    // forces: non-spherical kinematics, Hertz, tangential history
    const dbl4 vi4 = D.v[i], vj4 = D.v[j], wi4 = D.w[i], wj4 = D.w[j], ii4 = D.inert[i], ij4 = D.inert[j];
    const double wi[3] = {wi4.x, wi4.y, wi4.z}, wj[3] = {wj4.x, wj4.y, wj4.z};
    double xci[3], xcj[3], vri[3], vrj[3], vrel[3];
    for (int k = 0; k < 3; k++) {
        xci[k] = o.point[k] - ci[k];
        xcj[k] = o.point[k] - cj[k];
    }
    cross3(wi, xci, vri);
    cross3(wj, xcj, vrj);
    const double vi[3] = {vi4.x, vi4.y, vi4.z}, vj[3] = {vj4.x, vj4.y, vj4.z};
    for (int k = 0; k < 3; k++) vrel[k] = vi[k] - vj[k] + (vri[k] - vrj[k]);
    const double vn = dot3(vrel, en);
    const double vtr[3] = {vrel[0] - vn * en[0], vrel[1] - vn * en[1], vrel[2] - vn * en[2]};
    const double radi = ii4.w, radj = ij4.w, mi = vi4.w, mj = vj4.w, meff = mi * mj / (mi + mj);
    const double reff = radi * radj / (radi + radj);
    const double sqrtval = sqrt(reff * deltan);
    const double Sn = 2. * D.Yeff * sqrtval, St = 8. * D.Geff * sqrtval;
    const double kn = 4. / 3. * D.Yeff * sqrtval, kt = St;
    const double c56 = 0.91287092917527685576161630466800355658790782499663875;
    const double gamman = -2. * c56 * D.betaeff * sqrt(Sn * meff);
    const double gammat = -2. * c56 * D.betaeff * sqrt(St * meff);
    const double Fn = -gamman * vn + kn * deltan;
    const double Fi[3] = {Fn * en[0], Fn * en[1], Fn * en[2]}, Fnj[3] = {-Fi[0], -Fi[1], -Fi[2]};
    double Ti[3], Tj[3];
    cross3(xci, Fi, Ti);
    cross3(xcj, Fnj, Tj);
    dbl4 sh4 = D.shear[sl];
    double sh[3] = {sh4.x, sh4.y, sh4.z};
    if (shearupdate) {
        for (int k = 0; k < 3; k++) sh[k] += vtr[k] * D.dt;
        const double rsht = dot3(sh, en);
        for (int k = 0; k < 3; k++) sh[k] -= rsht * en[k];
    }
    const double shrmag = sqrt(dot3(sh, sh));
    double Ft[3] = {-(kt * sh[0]), -(kt * sh[1]), -(kt * sh[2])};
    const double Ft_shear = kt * shrmag, Ft_friction = D.mu * fabs(Fn);
    if (Ft_shear > Ft_friction) {
        if (shrmag != 0.0) {
            const double ratio = Ft_friction / Ft_shear;
            for (int k = 0; k < 3; k++) Ft[k] *= ratio;
            if (shearupdate)
                for (int k = 0; k < 3; k++) sh[k] = -Ft[k] / kt;
        } else {
            Ft[0] = Ft[1] = Ft[2] = 0.0;
        }
    } else {
        for (int k = 0; k < 3; k++) Ft[k] -= gammat * vtr[k];
    }
    D.shear[sl] = dbl4{sh[0], sh[1], sh[2], 0.0};
    double tti[3], ttj[3];
    const double Ftj[3] = {-Ft[0], -Ft[1], -Ft[2]};
    cross3(xci, Ft, tti);
    cross3(xcj, Ftj, ttj);
    D.pfi[sl] = dbl4{Fi[0] + Ft[0], Fi[1] + Ft[1], Fi[2] + Ft[2], 1.0};
    D.pti[sl] = dbl4{Ti[0] + tti[0], Ti[1] + tti[1], Ti[2] + tti[2], 0.0};
    D.ptj[sl] = dbl4{Tj[0] + ttj[0], Tj[1] + ttj[1], Tj[2] + ttj[2], 0.0};
    D.flag[sl] |= 5;
    D.state[sl] = INTERSECT;
}

// every slot: no force unless a solve below finds a contact; the bounding
// spheres and (for a pair not yet intersecting) the oriented boxes decide
// whether the slot needs a solve and which kind (kind[sl]; the host gathers
// the work lists from it in slot order, so they are the same in every run)
__global__ void k_sq_screen(SqDev D, const int *__restrict__ own, int nslots, signed char *kind_out)
{
    const int sl = blockIdx.x * blockDim.x + threadIdx.x;
    int kind = -1;
    if (sl < nslots) {
        const int i = own[sl], j = D.nbr[sl];
        const dbl4 xi4 = D.x[i], xj4 = D.x[j];
        D.pfi[sl] = dbl4{0, 0, 0, 0};
        D.pti[sl] = dbl4{0, 0, 0, 0};
        D.ptj[sl] = dbl4{0, 0, 0, 0};
        const double dx = xi4.x - xj4.x, dy = xi4.y - xj4.y, dz = xi4.z - xj4.z;
        const double rsq = dx * dx + dy * dy + dz * dz, radsum = xi4.w + xj4.w;
        if (rsq < radsum * radsum) {
            const int state = D.state[sl];
            bool obb = true;
            if (state != INTERSECT) {
                const dbl4 qi4 = D.q[i], qj4 = D.q[j], si4 = D.shape[i], sj4 = D.shape[j];
                const double ci[3] = {xi4.x, xi4.y, xi4.z}, cj[3] = {xj4.x, xj4.y, xj4.z};
                const double qi[4] = {qi4.x, qi4.y, qi4.z, qi4.w}, qj[4] = {qj4.x, qj4.y, qj4.z, qj4.w};
                const double si[3] = {si4.x, si4.y, si4.z}, sj[3] = {sj4.x, sj4.y, sj4.z};
                double Ri[9], Rj[9];
                quat_to_mat(qi, Ri);
                quat_to_mat(qj, Rj);
                obb = obb_intersect(ci, Ri, si, cj, Rj, sj);
            }
            if (!obb) D.state[sl] = FAR;
            else kind = state == FAR ? 0 : 1;
        }
    }
    if (sl < nslots) kind_out[sl] = (signed char)kind;
}

// the solve of one listed slot: a first contact (learned guess with the
// homotopy as fallback, or the homotopy) or a warm start (the previous point
// advanced with the mass-weighted contact-point velocity)
__device__ __forceinline__ void sq_solve_item(const SqDev &D, int sl, bool first, const int *own, int shearupdate,
                                              const float *guess)
{
    const int i = own[sl], j = D.nbr[sl];
    const dbl4 xi4 = D.x[i], xj4 = D.x[j], qi4 = D.q[i], qj4 = D.q[j], si4 = D.shape[i], sj4 = D.shape[j];
    const double ci[3] = {xi4.x, xi4.y, xi4.z}, cj[3] = {xj4.x, xj4.y, xj4.z};
    const double qi[4] = {qi4.x, qi4.y, qi4.z, qi4.w}, qj[4] = {qj4.x, qj4.y, qj4.z, qj4.w};
    const double si[3] = {si4.x, si4.y, si4.z}, sj[3] = {sj4.x, sj4.y, sj4.z};
    Newton o;
    int it = 0, sv = 0, used = 0;
    if (first) {
        first_contact(guess, ci, qi, si, si4.w, cj, qj, sj, sj4.w, o, it, sv, used);
    } else {
        const dbl4 cp4 = D.cp[sl], wi4 = D.w[i], wj4 = D.w[j], vi4 = D.v[i], vj4 = D.v[j];
        const double cp[3] = {cp4.x, cp4.y, cp4.z}, wi[3] = {wi4.x, wi4.y, wi4.z}, wj[3] = {wj4.x, wj4.y, wj4.z};
        double xci[3], xcj[3], vri[3], vrj[3], est[3];
        for (int k = 0; k < 3; k++) {
            xci[k] = cp[k] - ci[k];
            xcj[k] = cp[k] - cj[k];
        }
        cross3(wi, xci, vri);
        cross3(wj, xcj, vrj);
        const double mi = vi4.w, mj = vj4.w;
        const double vi[3] = {vi4.x, vi4.y, vi4.z}, vj[3] = {vj4.x, vj4.y, vj4.z};
        for (int k = 0; k < 3; k++) {
            const double a = vi[k] + vri[k], b = vj[k] + vrj[k];
            est[k] = cp[k] + (a * mi + b * mj) / (mi + mj) * D.dt;
        }
        contact_point(ci, qi, si, si4.w, cj, qj, sj, sj4.w, 1, est, false, 0.0, o, it, sv);
    }
    atomicAdd(&D.cnt[0], (unsigned long long)it);
    atomicAdd(&D.cnt[1], (unsigned long long)sv);
    atomicAdd(&D.cnt[2], 1ull);
    if (used == 1) atomicAdd(&D.cnt[3], 1ull);
    if (used == -1) atomicAdd(&D.cnt[4], 1ull);
    sq_finish(D, sl, i, j, shearupdate, o);
}

// the listed solves; each warp takes the next 32 items (the lists are
// complete when the kernel starts).  With a network, a warp holding first
// contacts computes their learned guesses together on the tensor cores.
__global__ void __launch_bounds__(128) k_sq_solve(SqDev D, SqWork W, const int *__restrict__ own, int shearupdate)
{
    __shared__ __align__(16) MlpInfer S;
    if (D.mlp) {
        mlp_stage(S, D.mlp);
        __syncthreads();
    }
    const int lane = threadIdx.x & 31;
    const int nfirst = W.n[0], total = nfirst + W.n[1];
    for (;;) {
        int base = 0;
        if (lane == 0) base = atomicAdd(W.next, 32);
        base = __shfl_sync(0xffffffffu, base, 0);
        if (base >= total) break;
        const int q = base + lane;
        const bool has = q < total, first = has && q < nfirst;
        const int sl = has ? (first ? W.list[0][q] : W.list[1][q - nfirst]) : 0;
        float out[kMlpOut] = {0.f, 0.f, 0.f, 0.f};
        const bool learned = D.mlp != nullptr && __any_sync(0xffffffffu, first);
        if (learned) {
            float feat[kMlpIn];
            if (first) {
                const int i = own[sl], j = D.nbr[sl];
                const dbl4 xi4 = D.x[i], xj4 = D.x[j], qi4 = D.q[i], qj4 = D.q[j], si4 = D.shape[i],
                           sj4 = D.shape[j];
                const double ci[3] = {xi4.x, xi4.y, xi4.z}, cj[3] = {xj4.x, xj4.y, xj4.z};
                const double qi[4] = {qi4.x, qi4.y, qi4.z, qi4.w}, qj[4] = {qj4.x, qj4.y, qj4.z, qj4.w};
                const double si[3] = {si4.x, si4.y, si4.z}, sj[3] = {sj4.x, sj4.y, sj4.z};
                pair_features_of(ci, qi, si, si4.w, cj, qj, sj, sj4.w, feat);
            }
            mlp_infer_warp(S, first, feat, out);
        }
        if (has) sq_solve_item(D, sl, first, own, shearupdate, learned ? out : nullptr);
    }
}

// per-atom sums in the reference's order: slots where the atom is the j
// side (ascending i), then its own slots
__global__ void k_sq_sum(SqDev D)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= D.n) return;
    double F[3] = {0, 0, 0}, T[3] = {0, 0, 0};
    for (int r = D.rstart[k]; r < D.rstart[k + 1]; r++) {
        const int sl = D.rslot[r];
        const dbl4 f = D.pfi[sl];
        if (f.w == 0.0) continue;
        const dbl4 t = D.ptj[sl];
        F[0] += -f.x;
        F[1] += -f.y;
        F[2] += -f.z;
        T[0] += t.x;
        T[1] += t.y;
        T[2] += t.z;
    }
    for (int sl = D.start[k]; sl < D.start[k + 1]; sl++) {
        const dbl4 f = D.pfi[sl];
        if (f.w == 0.0) continue;
        const dbl4 t = D.pti[sl];
        F[0] += f.x;
        F[1] += f.y;
        F[2] += f.z;
        T[0] += t.x;
        T[1] += t.y;
        T[2] += t.z;
    }
    D.f[k] = dbl4{F[0], F[1], F[2], 0.0};
    D.t[k] = dbl4{T[0], T[1], T[2], 0.0};
}

}  // namespace sq
}  // namespace gb2
