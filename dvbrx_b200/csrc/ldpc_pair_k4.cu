/*
 * Frame-pair decoder kernels, part 4 of the instantiations (the parts
 * compile in parallel; ldpc_pair.cu concatenates them in part order).
 */
#include "ldpc_pair.cuh"

namespace drxg {

static const PairKernel kPart[] = {
    DRXG_PAIR_KERNEL(8, 9, 0, 2, 1),
    DRXG_PAIR_KERNEL(8, 9, 0, 2, 2),
    DRXG_PAIR_KERNEL(9, 9, 0, 2, 1),
    DRXG_PAIR_KERNEL(9, 9, 0, 2, 2),
    DRXG_PAIR_KERNEL(9, 10, 0, 2, 1),
    DRXG_PAIR_KERNEL(9, 10, 0, 2, 2),
    DRXG_PAIR_KERNEL(11, 11, 0, 2, 1),
    DRXG_PAIR_KERNEL(11, 11, 0, 2, 2),
    DRXG_PAIR_KERNEL(11, 12, 0, 2, 1),
    DRXG_PAIR_KERNEL(11, 12, 0, 2, 2),
    DRXG_PAIR_KERNEL(12, 12, 0, 2, 1),
};

const PairKernel* pair_kernel_part4(int* n)
{
    *n = (int)(sizeof(kPart) / sizeof(kPart[0]));
    return kPart;
}

}  // namespace drxg
