// gb2_mlp.cuh -- the learned initial guess of the superquadric contact solve:
// training data from the plain solver, BF16 tensor-core training kernels
// (mma.sync m16n8k16, FP32 accumulation), Adam, and the evaluation that
// compares the learned guess with the plain method.  Included by gb2_sq.cu.
//
// Network: 14 -> 64 -> 64 -> 64 -> 4, ReLU, parameters as laid out in
// gb2_sq_kernels.cuh (normalisation statistics first).  Training keeps an
// FP32 master copy of the weights; every forward pass uses them rounded to
// BF16, activations are rounded to BF16 between layers, products accumulate
// in FP32 -- the contact pass infers with these same layers (mlp_infer_warp).
// Loss: mean squared error of the normalised outputs (point in particle i's
// frame / (ri + rj), mu).
#pragma once

#include <cuda_bf16.h>

#include "gb2_mma.cuh"
#include "gb2_sq_kernels.cuh"

namespace gb2 {
namespace sq {

constexpr int kMlpSample = 22;   // per sample: feat[14], target[4], s, mu, iters, solves (as floats)

// ------------------------------------------------------------------ random pairs near contact

__device__ __forceinline__ unsigned long long mix64(unsigned long long z)
{
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ double urand(unsigned long long &s)
{
    s = mix64(s);
    return (double)(s >> 11) * (1.0 / 9007199254740992.0);
}
__device__ __forceinline__ void rand_quat(unsigned long long &s, double *q)
{
    const double u1 = urand(s), u2 = urand(s), u3 = urand(s);
    const double a = sqrt(1 - u1), b = sqrt(u1), t2 = 2 * M_PI * u2, t3 = 2 * M_PI * u3;
    q[0] = b * cos(t3);
    q[1] = a * sin(t2);
    q[2] = a * cos(t2);
    q[3] = b * sin(t3);
}

// One pair of superquadrics with half-axes U(1, 2) mm and blockiness U(2, 8),
// random orientations, j's centre at a random direction and a distance
// U(0.3, 1) x (rb_i + rb_j) from i's; kept when the oriented boxes intersect
// (the pairs the simulation hands to the first-contact solve).
struct PairSample {
    double ci[3], qi[4], si[3], ni, cj[3], qj[4], sj[3], nj;
};
__device__ __forceinline__ bool sample_pair(unsigned long long seed, long idx, PairSample &P)
{
    unsigned long long s = mix64(seed ^ mix64((unsigned long long)idx + 1));
    for (int d = 0; d < 3; d++) {
        P.si[d] = 1e-3 + 1e-3 * urand(s);
        P.sj[d] = 1e-3 + 1e-3 * urand(s);
        P.ci[d] = 0.0;
    }
    P.ni = 2.0 + 6.0 * urand(s);
    P.nj = 2.0 + 6.0 * urand(s);
    rand_quat(s, P.qi);
    rand_quat(s, P.qj);
    double dir[3];
    for (;;) {
        for (int d = 0; d < 3; d++) dir[d] = 2.0 * urand(s) - 1.0;
        const double m = dot3(dir, dir);
        if (m > 1e-6 && m <= 1.0) {
            const double inv = 1.0 / sqrt(m);
            for (int d = 0; d < 3; d++) dir[d] *= inv;
            break;
        }
    }
    // bounding radii from the box diagonal (an upper bound of every blockiness)
    const double rbi = sqrt(dot3(P.si, P.si)), rbj = sqrt(dot3(P.sj, P.sj));
    const double dist = (0.3 + 0.7 * urand(s)) * (rbi + rbj);
    for (int d = 0; d < 3; d++) P.cj[d] = dist * dir[d];
    double Ri[9], Rj[9];
    quat_to_mat(P.qi, Ri);
    quat_to_mat(P.qj, Rj);
    return obb_intersect(P.ci, Ri, P.si, P.cj, Rj, P.sj);
}

// Label one sample with the plain solver (homotopy from spheres): features,
// normalised-frame target (point in i's frame / s, mu), and its cost.
// out[21] = 1 when the sample is valid (OBB intersect, converged).
__global__ void k_mlp_make(unsigned long long seed, long n, float *out)
{
    const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    float *o = out + k * kMlpSample;
    PairSample P;
    o[21] = 0.f;
    if (!sample_pair(seed, k, P)) return;
    Newton sol;
    int it = 0, sv = 0;
    contact_point(P.ci, P.qi, P.si, P.ni, P.cj, P.qj, P.sj, P.nj, 0, nullptr, false, 0.0, sol, it, sv);
    if (sol.fail || !(sol.merit < 1e-10)) return;
    double Ri[9];
    quat_to_mat(P.qi, Ri);
    float feat[kMlpIn];
    const double s = pair_features(P.ci, P.qi, P.si, P.ni, P.cj, P.qj, P.sj, P.nj, Ri, feat);
    double pl[3];
    const double d[3] = {sol.point[0] - P.ci[0], sol.point[1] - P.ci[1], sol.point[2] - P.ci[2]};
    tmatvec(Ri, d, pl);
    for (int c = 0; c < kMlpIn; c++) o[c] = feat[c];
    o[14] = (float)(pl[0] / s);
    o[15] = (float)(pl[1] / s);
    o[16] = (float)(pl[2] / s);
    o[17] = (float)sol.mu;
    o[18] = (float)it;
    o[19] = (float)sv;
    o[20] = (float)s;
    o[21] = 1.f;
}

// Learned guess against the plain method on fresh samples: per sample the
// plain cost, the learned cost (guess solve + fallback), whether the learned
// guess was accepted, and the distance between the two converged points.
__global__ void __launch_bounds__(128) k_mlp_eval(unsigned long long seed, long n, const float *__restrict__ P,
                                                  long long *stats, double *maxdiff_bits)
{
    __shared__ __align__(16) MlpInfer M;
    mlp_stage(M, P);
    __syncthreads();
    const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    PairSample S;
    const bool valid = k < n && sample_pair(seed, k, S);
    float feat[kMlpIn], out[kMlpOut];
    if (valid) pair_features_of(S.ci, S.qi, S.si, S.ni, S.cj, S.qj, S.sj, S.nj, feat);
    mlp_infer_warp(M, valid, feat, out);
    if (!valid) return;
    Newton plain, learned;
    int it0, sv0, it1, sv1, used;
    contact_point(S.ci, S.qi, S.si, S.ni, S.cj, S.qj, S.sj, S.nj, 0, nullptr, false, 0.0, plain, it0, sv0);
    first_contact(out, S.ci, S.qi, S.si, S.ni, S.cj, S.qj, S.sj, S.nj, learned, it1, sv1, used);
    atomicAdd((unsigned long long *)&stats[0], 1ull);
    atomicAdd((unsigned long long *)&stats[1], (unsigned long long)it0);
    atomicAdd((unsigned long long *)&stats[2], (unsigned long long)sv0);
    atomicAdd((unsigned long long *)&stats[3], (unsigned long long)it1);
    atomicAdd((unsigned long long *)&stats[4], (unsigned long long)sv1);
    if (used == 1) atomicAdd((unsigned long long *)&stats[5], 1ull);
    if (plain.fail || !(plain.merit < 1e-10)) atomicAdd((unsigned long long *)&stats[6], 1ull);
    if (learned.fail || !(learned.merit < 1e-10)) atomicAdd((unsigned long long *)&stats[7], 1ull);
    if (!plain.fail && plain.merit < 1e-10 && !learned.fail && learned.merit < 1e-10) {
        double dm = 0;
        for (int c = 0; c < 3; c++) dm = fmax(dm, fabs(plain.point[c] - learned.point[c]));
        // same-point test: merit < 1e-10 bounds the angle between the two
        // gradients by 1e-5, so converged points may slide by ~1e-5 of the
        // size along the surfaces; count pairs apart by more than 1e-4
        const double size = fmin(fmin(S.si[0], S.si[1]), S.si[2]);
        if (dm > 1e-4 * size) atomicAdd((unsigned long long *)&stats[8], 1ull);
        atomicMax((unsigned long long *)maxdiff_bits, (unsigned long long)__double_as_longlong(dm / size));
    }
}

// Timed comparison of the two first-contact solves on the same stored pairs:
// k_mlp_store_pairs keeps the valid samples; the plain method is one launch
// of the homotopy from spheres (one thread per pair); the learned method is a
// launch of the learned attempts (guesses on the tensor cores, one warp per
// 32 pairs) that gathers the rejected pairs in a list, then the homotopy over
// that list (k_mlp_solve_rejected), so the few pairs the guess does not
// settle no longer hold warps of settled ones.  Points and iteration counts
// are those of one call of first_contact() per pair.
__global__ void k_mlp_store_pairs(unsigned long long seed, long n, PairSample *out, int *nvalid)
{
    const long k = (long)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    PairSample S;
    if (!sample_pair(seed, k, S)) return;
    out[atomicAdd(nvalid, 1)] = S;
}

template <bool LEARNED>
__global__ void __launch_bounds__(128) k_mlp_solve(const PairSample *pairs, const int *nvalid,
                                                   const float *__restrict__ P, double *point, long long *iters,
                                                   int *rejected, int *nrejected)
{
    __shared__ __align__(16) MlpInfer M;
    if constexpr (LEARNED) {
        mlp_stage(M, P);
        __syncthreads();
    }
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = k < *nvalid;
    bool reject = false;
    PairSample S;
    if (valid) S = pairs[k];
    float out[kMlpOut];
    if constexpr (LEARNED) {
        float feat[kMlpIn];
        if (valid) pair_features_of(S.ci, S.qi, S.si, S.ni, S.cj, S.qj, S.sj, S.nj, feat);
        mlp_infer_warp(M, valid, feat, out);
    }
    if (valid) {
        Newton o;
        int it, sv;
        if constexpr (LEARNED) {
            used_learned_guess(out, S.ci, S.qi, S.si, S.ni, S.cj, S.qj, S.sj, S.nj, o, it, sv);
            reject = o.fail || !(o.merit < 1e-10);
        } else {
            contact_point(S.ci, S.qi, S.si, S.ni, S.cj, S.qj, S.sj, S.nj, 0, nullptr, false, 0.0, o, it, sv);
        }
        if (!reject)
            for (int c = 0; c < 3; c++) point[3 * k + c] = o.point[c];
        atomicAdd((unsigned long long *)iters, (unsigned long long)it);
    }
    if constexpr (LEARNED) {   // warp-aggregated append of the rejected pairs
        const unsigned m = __ballot_sync(0xffffffffu, reject);
        if (m) {
            const int lane = threadIdx.x & 31, leader = __ffs(m) - 1;
            int base = 0;
            if (lane == leader) base = atomicAdd(nrejected, __popc(m));
            base = __shfl_sync(0xffffffffu, base, leader);
            if (reject) rejected[base + __popc(m & ((1u << lane) - 1u))] = k;
        }
    }
}

// the homotopy for the pairs whose learned guess was rejected
__global__ void k_mlp_solve_rejected(const PairSample *pairs, const int *rejected, const int *nrejected, double *point,
                                     long long *iters)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= *nrejected) return;
    const int k = rejected[q];
    const PairSample S = pairs[k];
    Newton o;
    int it, sv;
    contact_point(S.ci, S.qi, S.si, S.ni, S.cj, S.qj, S.sj, S.nj, 0, nullptr, false, 0.0, o, it, sv);
    for (int c = 0; c < 3; c++) point[3 * k + c] = o.point[c];
    atomicAdd((unsigned long long *)iters, (unsigned long long)it);
}

// ------------------------------------------------------------------ training (BF16 tensor cores)

// padded layer shapes: in 14 -> 16, out 4 -> 8 (zero rows/columns)
constexpr int kK1 = 16, kOutP = 8;
constexpr int kWarps = 4, kTile = 16;   // 4 warps x 16 samples per CTA

struct MlpSmem {
    __nv_bfloat16 W1[kMlpH][kK1];
    __nv_bfloat16 W2[kMlpH][kMlpH];
    __nv_bfloat16 W3[kMlpH][kMlpH];
    __nv_bfloat16 W4[16][kMlpH];   // rows 4..15 zero
    float b1[kMlpH], b2[kMlpH], b3[kMlpH], b4[kOutP];
    // per warp activations (bf16) and backward deltas (bf16)
    __nv_bfloat16 X[kWarps][kTile][kK1];
    __nv_bfloat16 H1[kWarps][kTile][kMlpH], H2[kWarps][kTile][kMlpH], H3[kWarps][kTile][kMlpH];
    __nv_bfloat16 D[kWarps][kTile][kMlpH];   // delta of the current layer (pre-activation)
    __nv_bfloat16 E[kWarps][kTile][kMlpH];   // delta of the layer below
    __nv_bfloat16 DY[kWarps][kTile][16];     // output delta, columns 4..15 zero
};

// E(16 x K) = D(16 x N) W (W [N][K]); masked by the ReLU of Hin (> 0)
template <int N, int K>
__device__ __forceinline__ void layer_bwd_x(const __nv_bfloat16 *Dm, const __nv_bfloat16 *W, const __nv_bfloat16 *Hin,
                                            __nv_bfloat16 *E)
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    for (int n0 = 0; n0 < K; n0 += 8) {
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
        for (int k0 = 0; k0 < N; k0 += 16) {
            unsigned a[4], bb[2];
            load_a<false>(Dm, N, 0, k0, a);
            load_b<false>(W, K, k0, n0, bb);
            mma16816(acc, a, bb);
        }
        const int c = n0 + 2 * t;
        const float m0 = __bfloat162float(Hin[g * K + c]) > 0.f ? 1.f : 0.f;
        const float m1 = __bfloat162float(Hin[g * K + c + 1]) > 0.f ? 1.f : 0.f;
        const float m2 = __bfloat162float(Hin[(g + 8) * K + c]) > 0.f ? 1.f : 0.f;
        const float m3 = __bfloat162float(Hin[(g + 8) * K + c + 1]) > 0.f ? 1.f : 0.f;
        E[g * K + c] = __float2bfloat16_rn(acc[0] * m0);
        E[g * K + c + 1] = __float2bfloat16_rn(acc[1] * m1);
        E[(g + 8) * K + c] = __float2bfloat16_rn(acc[2] * m2);
        E[(g + 8) * K + c + 1] = __float2bfloat16_rn(acc[3] * m3);
    }
}

// dW(Nout x K) += D^T(Nout x 16 samples) Xin(16 x K), db += column sums of D,
// accumulated into the FP32 gradient in global memory
template <int NOUT, int K>
__device__ __forceinline__ void layer_bwd_w(const __nv_bfloat16 *Dm, int ldd, const __nv_bfloat16 *Xin, float *gW,
                                            float *gb, int nvalid_out, int kvalid)
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    for (int m0 = 0; m0 < NOUT; m0 += 16)
        for (int n0 = 0; n0 < K; n0 += 8) {
            float acc[4] = {0.f, 0.f, 0.f, 0.f};
            unsigned a[4], bb[2];
            load_a<true>(Dm, ldd, m0, 0, a);    // A(m = out, k = sample) = D[sample][out]
            load_b<false>(Xin, K, 0, n0, bb);   // B(k = sample, n = in) = X[sample][in]
            mma16816(acc, a, bb);
            const int r0 = m0 + g, r1 = m0 + g + 8, c = n0 + 2 * t;
            if (r0 < nvalid_out) {
                if (c < kvalid) atomicAdd(&gW[r0 * kvalid + c], acc[0]);
                if (c + 1 < kvalid) atomicAdd(&gW[r0 * kvalid + c + 1], acc[1]);
            }
            if (r1 < nvalid_out) {
                if (c < kvalid) atomicAdd(&gW[r1 * kvalid + c], acc[2]);
                if (c + 1 < kvalid) atomicAdd(&gW[r1 * kvalid + c + 1], acc[3]);
            }
        }
    // bias: lanes stride over outputs, each sums the 16 samples
    for (int o = lane; o < nvalid_out; o += 32) {
        float s = 0.f;
        for (int r = 0; r < kTile; r++) s += __bfloat162float(Dm[r * ldd + o]);
        atomicAdd(&gb[o], s);
    }
}

// One forward + backward pass over a batch: samples [row0, row0 + nrows) of
// data (kMlpSample floats each, features normalised on the fly with the
// statistics in P), gradient accumulated into G (layout of P), loss into
// loss[0].  Master weights P are FP32; they are rounded to BF16 here.
__global__ void __launch_bounds__(128) k_mlp_fwd_bwd(const float *__restrict__ P, const float *__restrict__ data,
                                                      const int *__restrict__ idx, long nrows, float *G, float *loss)
{
    extern __shared__ __align__(16) unsigned char smraw[];
    MlpSmem &S = *reinterpret_cast<MlpSmem *>(smraw);
    const int tid = threadIdx.x, wid = tid >> 5, lane = tid & 31;
    // weights to shared memory, rounded to bf16, padded with zeros
    for (int e = tid; e < kMlpH * kK1; e += blockDim.x) {
        const int o = e / kK1, c = e % kK1;
        S.W1[o][c] = __float2bfloat16_rn(c < kMlpIn ? P[kMlpOffW1 + o * kMlpIn + c] : 0.f);
    }
    for (int e = tid; e < kMlpH * kMlpH; e += blockDim.x) {
        S.W2[e / kMlpH][e % kMlpH] = __float2bfloat16_rn(P[kMlpOffW2 + e]);
        S.W3[e / kMlpH][e % kMlpH] = __float2bfloat16_rn(P[kMlpOffW3 + e]);
    }
    for (int e = tid; e < 16 * kMlpH; e += blockDim.x) {
        const int o = e / kMlpH;
        S.W4[o][e % kMlpH] = __float2bfloat16_rn(o < kMlpOut ? P[kMlpOffW4 + e] : 0.f);
    }
    for (int e = tid; e < kMlpH; e += blockDim.x) {
        S.b1[e] = P[kMlpOffB1 + e];
        S.b2[e] = P[kMlpOffB2 + e];
        S.b3[e] = P[kMlpOffB3 + e];
    }
    if (tid < kOutP) S.b4[tid] = tid < kMlpOut ? P[kMlpOffB4 + tid] : 0.f;
    // this warp's 16 samples
    const long r0 = ((long)blockIdx.x * kWarps + wid) * kTile;
    for (int e = lane; e < kTile * kK1; e += 32) {
        const int r = e / kK1, c = e % kK1;
        const long row = r0 + r;
        float v = 0.f;
        if (row < nrows && c < kMlpIn) v = (data[(long)idx[row] * kMlpSample + c] - P[c]) / P[kMlpIn + c];
        S.X[wid][r][c] = __float2bfloat16_rn(v);
    }
    __syncthreads();
    layer_fwd<kK1, kMlpH>(&S.X[wid][0][0], &S.W1[0][0], S.b1, &S.H1[wid][0][0], true);
    __syncwarp();
    layer_fwd<kMlpH, kMlpH>(&S.H1[wid][0][0], &S.W2[0][0], S.b2, &S.H2[wid][0][0], true);
    __syncwarp();
    layer_fwd<kMlpH, kMlpH>(&S.H2[wid][0][0], &S.W3[0][0], S.b3, &S.H3[wid][0][0], true);
    __syncwarp();
    // output layer in FP32 (4 outputs), loss and its gradient
    {
        const int g = lane >> 2, t = lane & 3;
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
        for (int k0 = 0; k0 < kMlpH; k0 += 16) {
            unsigned a[4], bb[2];
            load_a<false>(&S.H3[wid][0][0], kMlpH, 0, k0, a);
            load_b<true>(&S.W4[0][0], kMlpH, k0, 0, bb);
            mma16816(acc, a, bb);
        }
        float lsum = 0.f;
        const float scale = 2.0f / (float)(nrows * kMlpOut);
        for (int q = 0; q < 4; q++) {
            const int r = g + (q >> 1) * 8, c = 2 * t + (q & 1);
            const long row = r0 + r;
            float dy = 0.f;
            if (row < nrows && c < kMlpOut) {
                const float y = acc[q] + S.b4[c];
                const float tgt = (data[(long)idx[row] * kMlpSample + 14 + c] - P[2 * kMlpIn + c]) /
                                  P[2 * kMlpIn + kMlpOut + c];
                const float e = y - tgt;
                lsum += e * e;
                dy = scale * e;
            }
            S.DY[wid][r][c] = __float2bfloat16_rn(dy);
        }
        for (int e = lane; e < kTile * 8; e += 32) S.DY[wid][e / 8][8 + e % 8] = __float2bfloat16_rn(0.f);
        for (int o = 16; o >= 1; o >>= 1) lsum += __shfl_xor_sync(0xffffffffu, lsum, o);
        if (lane == 0) atomicAdd(loss, lsum / (float)(nrows * kMlpOut));
    }
    __syncwarp();
    // backward: layer 4
    layer_bwd_w<16, kMlpH>(&S.DY[wid][0][0], 16, &S.H3[wid][0][0], G + kMlpOffW4, G + kMlpOffB4, kMlpOut, kMlpH);
    layer_bwd_x<16, kMlpH>(&S.DY[wid][0][0], &S.W4[0][0], &S.H3[wid][0][0], &S.D[wid][0][0]);
    __syncwarp();
    // layer 3
    layer_bwd_w<kMlpH, kMlpH>(&S.D[wid][0][0], kMlpH, &S.H2[wid][0][0], G + kMlpOffW3, G + kMlpOffB3, kMlpH, kMlpH);
    layer_bwd_x<kMlpH, kMlpH>(&S.D[wid][0][0], &S.W3[0][0], &S.H2[wid][0][0], &S.E[wid][0][0]);
    __syncwarp();
    // layer 2
    layer_bwd_w<kMlpH, kMlpH>(&S.E[wid][0][0], kMlpH, &S.H1[wid][0][0], G + kMlpOffW2, G + kMlpOffB2, kMlpH, kMlpH);
    layer_bwd_x<kMlpH, kMlpH>(&S.E[wid][0][0], &S.W2[0][0], &S.H1[wid][0][0], &S.D[wid][0][0]);
    __syncwarp();
    // layer 1
    layer_bwd_w<kMlpH, kK1>(&S.D[wid][0][0], kMlpH, &S.X[wid][0][0], G + kMlpOffW1, G + kMlpOffB1, kMlpH, kMlpIn);
}

// Adam on the trainable parameters (everything after the 36 statistics)
__global__ void k_mlp_adam(float *P, const float *G, float *m, float *v, int n, float lr, float b1, float b2,
                           float eps, float c1, float c2)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x + kMlpOffW1;
    if (k >= n) return;
    const float g = G[k];
    const float mk = b1 * m[k] + (1.f - b1) * g;
    const float vk = b2 * v[k] + (1.f - b2) * g * g;
    m[k] = mk;
    v[k] = vk;
    P[k] -= lr * (mk / c1) / (sqrtf(vk / c2) + eps);
}

}  // namespace sq
}  // namespace gb2
