// gb2_mma.cuh -- warp-level BF16 tensor-core building blocks (mma.sync
// m16n8k16, FP32 accumulation) shared by the learned-guess training kernels
// and the warp-cooperative inference of the superquadric contact pass.
#pragma once

#include <cuda_bf16.h>

namespace gb2 {
namespace sq {

__device__ __forceinline__ unsigned pack_bf16(__nv_bfloat16 lo, __nv_bfloat16 hi)
{
    return (unsigned)__bfloat16_as_ushort(lo) | ((unsigned)__bfloat16_as_ushort(hi) << 16);
}

// D(16x8, f32) += A(16x16, bf16, row) * B(16x8, bf16, col)
__device__ __forceinline__ void mma16816(float *d, const unsigned *a, const unsigned *b)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// A fragment of a 16x16 tile at (row0, col0) of a row-major bf16 matrix with
// leading dimension ld, optionally transposed (element (r, c) read at [c][r])
template <bool TRANS>
__device__ __forceinline__ void load_a(const __nv_bfloat16 *M, int ld, int row0, int col0, unsigned *a)
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    auto at = [&](int r, int c) { return TRANS ? M[(col0 + c) * ld + row0 + r] : M[(row0 + r) * ld + col0 + c]; };
    a[0] = pack_bf16(at(g, 2 * t), at(g, 2 * t + 1));
    a[1] = pack_bf16(at(g + 8, 2 * t), at(g + 8, 2 * t + 1));
    a[2] = pack_bf16(at(g, 2 * t + 8), at(g, 2 * t + 9));
    a[3] = pack_bf16(at(g + 8, 2 * t + 8), at(g + 8, 2 * t + 9));
}
// B fragment of a 16x8 tile (k0, n0) where element (k, n) is read at
// M[n][k] (NK: weights [out][in] used as B = W^T) or M[k][n] (KN)
template <bool NK>
__device__ __forceinline__ void load_b(const __nv_bfloat16 *M, int ld, int k0, int n0, unsigned *b)
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    auto at = [&](int k, int n) { return NK ? M[(n0 + n) * ld + k0 + k] : M[(k0 + k) * ld + n0 + n]; };
    b[0] = pack_bf16(at(2 * t, g), at(2 * t + 1, g));
    b[1] = pack_bf16(at(2 * t + 8, g), at(2 * t + 9, g));
}

// Y(16 x N) = X(16 x K) W^T with W [N][K] in shared memory; epilogue
// bias + ReLU, result rounded to bf16 into H (row-major 16 x N)
template <int K, int N>
__device__ __forceinline__ void layer_fwd(const __nv_bfloat16 *X, const __nv_bfloat16 *W, const float *b,
                                          __nv_bfloat16 *H, bool relu)
{
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    for (int n0 = 0; n0 < N; n0 += 8) {
        float acc[4] = {0.f, 0.f, 0.f, 0.f};
        for (int k0 = 0; k0 < K; k0 += 16) {
            unsigned a[4], bb[2];
            load_a<false>(X, K, 0, k0, a);
            load_b<true>(W, K, k0, n0, bb);
            mma16816(acc, a, bb);
        }
        const int c = n0 + 2 * t;
        float v0 = acc[0] + b[c], v1 = acc[1] + b[c + 1], v2 = acc[2] + b[c], v3 = acc[3] + b[c + 1];
        if (relu) {
            v0 = fmaxf(v0, 0.f);
            v1 = fmaxf(v1, 0.f);
            v2 = fmaxf(v2, 0.f);
            v3 = fmaxf(v3, 0.f);
        }
        H[g * N + c] = __float2bfloat16_rn(v0);
        H[g * N + c + 1] = __float2bfloat16_rn(v1);
        H[(g + 8) * N + c] = __float2bfloat16_rn(v2);
        H[(g + 8) * N + c + 1] = __float2bfloat16_rn(v3);
    }
}

}  // namespace sq
}  // namespace gb2
