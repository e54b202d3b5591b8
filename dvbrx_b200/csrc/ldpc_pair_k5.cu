/*
 * Frame-pair decoder kernels, part 5 of the instantiations (the parts
 * compile in parallel; ldpc_pair.cu concatenates them in part order).
 */
#include "ldpc_pair.cuh"

namespace drxg {

static const PairKernel kPart[] = {
    DRXG_PAIR_KERNEL(12, 12, 0, 2, 2),
    DRXG_PAIR_KERNEL(9, 9, 0, 3, 1),
    DRXG_PAIR_KERNEL(9, 9, 0, 3, 2),
    DRXG_PAIR_KERNEL(1, 1, 7, 3, 1),
    DRXG_PAIR_KERNEL(1, 1, 7, 3, 2),
    DRXG_PAIR_KERNEL(1, 1, 11, 3, 1),
    DRXG_PAIR_KERNEL(1, 1, 11, 3, 2),
    DRXG_PAIR_KERNEL(1, 1, 14, 3, 1),
    DRXG_PAIR_KERNEL(1, 1, 14, 3, 2),
    DRXG_PAIR_KERNEL(16, 16, 0, 4, 2),
    DRXG_PAIR_KERNEL(1, 1, 22, 5, 1),
    DRXG_PAIR_KERNEL(25, 25, 0, 6, 1),
};

const PairKernel* pair_kernel_part5(int* n)
{
    *n = (int)(sizeof(kPart) / sizeof(kPart[0]));
    return kPart;
}

}  // namespace drxg
