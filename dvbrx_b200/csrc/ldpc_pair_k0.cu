/*
 * Frame-pair decoder kernels, part 0 of the instantiations (the parts
 * compile in parallel; ldpc_pair.cu concatenates them in part order).
 */
#include "ldpc_pair.cuh"

namespace drxg {

static const PairKernel kPart[] = {
    DRXG_PAIR_KERNEL(1, 2, 0, 2, 0),
    DRXG_PAIR_KERNEL(2, 2, 0, 2, 0),
    DRXG_PAIR_KERNEL(2, 3, 0, 2, 0),
    DRXG_PAIR_KERNEL(3, 3, 0, 2, 0),
    DRXG_PAIR_KERNEL(4, 4, 0, 2, 0),
    DRXG_PAIR_KERNEL(5, 5, 0, 2, 0),
    DRXG_PAIR_KERNEL(5, 6, 0, 2, 0),
    DRXG_PAIR_KERNEL(6, 7, 0, 2, 0),
    DRXG_PAIR_KERNEL(7, 7, 0, 2, 0),
    DRXG_PAIR_KERNEL(7, 8, 0, 2, 0),
    DRXG_PAIR_KERNEL(8, 8, 0, 2, 0),
    DRXG_PAIR_KERNEL(8, 9, 0, 2, 0),
    DRXG_PAIR_KERNEL(9, 9, 0, 2, 0),
    DRXG_PAIR_KERNEL(9, 10, 0, 2, 0),
    DRXG_PAIR_KERNEL(11, 11, 0, 2, 0),
    DRXG_PAIR_KERNEL(11, 12, 0, 2, 0),
    DRXG_PAIR_KERNEL(12, 12, 0, 2, 0),
    DRXG_PAIR_KERNEL(9, 9, 0, 3, 0),
    DRXG_PAIR_KERNEL(12, 13, 0, 2, 0),
    DRXG_PAIR_KERNEL(13, 14, 0, 2, 0),
};

const PairKernel* pair_kernel_part0(int* n)
{
    *n = (int)(sizeof(kPart) / sizeof(kPart[0]));
    return kPart;
}

}  // namespace drxg
