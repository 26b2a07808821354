// gb2_split.cu -- split-precision instantiation of the fused pair step.
//
// Same kernel source as the FP64 path (gb2_step.cuh) with SPLIT = true:
// neighbour screening, positions, the overlap of each touching pair, walls,
// gravity and the Velocity-Verlet integration stay FP64; the sphere-sphere
// contact chain runs in FP32 on FP64-differenced relative positions and the
// per-atom pair sums are FP32 with Kahan compensation.  This unit is built
// with FMA contraction and the fast FP32 intrinsics allowed; the FP64 unit
// is not.
#include "gb2_step.cuh"

namespace gb2 {

template <bool R, int MINB>
static void launch(const Dev &D, int nblocks, cudaStream_t st, int shearupdate, int integrate, int fuse_next,
                   int store_f, size_t smem)
{
    k_pair_step<R, MINB, true><<<nblocks, 128, smem, st>>>(D, shearupdate, integrate, fuse_next, store_f);
}

void launch_pair_split(const Dev &D, int nblocks, cudaStream_t st, int minb, int shearupdate, int integrate,
                       int fuse_next, int store_f, size_t smem)
{
    const int mb = minb ? minb : 5;   // 5 (96 registers, no spill) measured fastest on the packed 1M hopper
    if (D.rolling) {
        if (mb == 4) launch<true, 4>(D, nblocks, st, shearupdate, integrate, fuse_next, store_f, smem);
        else if (mb == 5) launch<true, 5>(D, nblocks, st, shearupdate, integrate, fuse_next, store_f, smem);
        else if (mb == 6) launch<true, 6>(D, nblocks, st, shearupdate, integrate, fuse_next, store_f, smem);
        else if (mb == 7) launch<true, 7>(D, nblocks, st, shearupdate, integrate, fuse_next, store_f, smem);
        else launch<true, 8>(D, nblocks, st, shearupdate, integrate, fuse_next, store_f, smem);
    } else {
        if (mb == 4) launch<false, 4>(D, nblocks, st, shearupdate, integrate, fuse_next, store_f, smem);
        else if (mb == 5) launch<false, 5>(D, nblocks, st, shearupdate, integrate, fuse_next, store_f, smem);
        else if (mb == 6) launch<false, 6>(D, nblocks, st, shearupdate, integrate, fuse_next, store_f, smem);
        else if (mb == 7) launch<false, 7>(D, nblocks, st, shearupdate, integrate, fuse_next, store_f, smem);
        else launch<false, 8>(D, nblocks, st, shearupdate, integrate, fuse_next, store_f, smem);
    }
}

void launch_tail_split(const Dev &D, int nblocks, cudaStream_t st, int shearupdate, int integrate, int fuse_next,
                       int store_f)
{
    if (D.rolling) launch_pair_tail<true, true>(D, nblocks, st, shearupdate, integrate, fuse_next, store_f);
    else launch_pair_tail<false, true>(D, nblocks, st, shearupdate, integrate, fuse_next, store_f);
}

}  // namespace gb2
