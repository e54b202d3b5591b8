/*
 * Frame-pair decoder kernels, part 3 of the instantiations (the parts
 * compile in parallel; ldpc_pair.cu concatenates them in part order).
 */
#include "ldpc_pair.cuh"

namespace drxg {

static const PairKernel kPart[] = {
    DRXG_PAIR_KERNEL(5, 5, 0, 2, 2),
    DRXG_PAIR_KERNEL(5, 6, 0, 2, 1),
    DRXG_PAIR_KERNEL(5, 6, 0, 2, 2),
    DRXG_PAIR_KERNEL(6, 7, 0, 2, 1),
    DRXG_PAIR_KERNEL(6, 7, 0, 2, 2),
    DRXG_PAIR_KERNEL(7, 7, 0, 2, 1),
    DRXG_PAIR_KERNEL(7, 7, 0, 2, 2),
    DRXG_PAIR_KERNEL(7, 8, 0, 2, 1),
    DRXG_PAIR_KERNEL(7, 8, 0, 2, 2),
    DRXG_PAIR_KERNEL(8, 8, 0, 2, 1),
    DRXG_PAIR_KERNEL(8, 8, 0, 2, 2),
};

const PairKernel* pair_kernel_part3(int* n)
{
    *n = (int)(sizeof(kPart) / sizeof(kPart[0]));
    return kPart;
}

}  // namespace drxg
