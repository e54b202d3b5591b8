/*
 * Frame-pair decoder kernels, part 2 of the instantiations (the parts
 * compile in parallel; ldpc_pair.cu concatenates them in part order).
 */
#include "ldpc_pair.cuh"

namespace drxg {

static const PairKernel kPart[] = {
    DRXG_PAIR_KERNEL(1, 2, 0, 2, 1),
    DRXG_PAIR_KERNEL(1, 2, 0, 2, 2),
    DRXG_PAIR_KERNEL(2, 2, 0, 2, 1),
    DRXG_PAIR_KERNEL(2, 2, 0, 2, 2),
    DRXG_PAIR_KERNEL(2, 3, 0, 2, 1),
    DRXG_PAIR_KERNEL(2, 3, 0, 2, 2),
    DRXG_PAIR_KERNEL(3, 3, 0, 2, 1),
    DRXG_PAIR_KERNEL(3, 3, 0, 2, 2),
    DRXG_PAIR_KERNEL(4, 4, 0, 2, 1),
    DRXG_PAIR_KERNEL(4, 4, 0, 2, 2),
    DRXG_PAIR_KERNEL(5, 5, 0, 2, 1),
};

const PairKernel* pair_kernel_part2(int* n)
{
    *n = (int)(sizeof(kPart) / sizeof(kPart[0]));
    return kPart;
}

}  // namespace drxg
