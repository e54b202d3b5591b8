/*
 * Frame-pair decoder kernels, part 1 of the instantiations (the parts
 * compile in parallel; ldpc_pair.cu concatenates them in part order).
 */
#include "ldpc_pair.cuh"

namespace drxg {

static const PairKernel kPart[] = {
    DRXG_PAIR_KERNEL(14, 15, 0, 2, 0),
    DRXG_PAIR_KERNEL(16, 16, 0, 4, 0),
    DRXG_PAIR_KERNEL(17, 18, 0, 2, 0),
    DRXG_PAIR_KERNEL(20, 20, 0, 3, 0),
    DRXG_PAIR_KERNEL(25, 25, 0, 6, 0),
    DRXG_PAIR_KERNEL(27, 28, 0, 2, 0),
    DRXG_PAIR_KERNEL(28, 28, 0, 4, 0),
    DRXG_PAIR_KERNEL(1, 1, 7, 3, 0),
    DRXG_PAIR_KERNEL(1, 1, 11, 3, 0),
    DRXG_PAIR_KERNEL(1, 1, 14, 3, 0),
    DRXG_PAIR_KERNEL(1, 1, 22, 5, 0),
    DRXG_PAIR_KERNEL(1, 1, 32, 6, 0),
};

const PairKernel* pair_kernel_part1(int* n)
{
    *n = (int)(sizeof(kPart) / sizeof(kPart[0]));
    return kPart;
}

}  // namespace drxg
