/*
 * One-launch, two-frames-per-CTA decoding of a mixed batch
 * (ldpc_mixpair.cu): parameters and launcher.
 */
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "ldpc_device.h"

namespace drxg {

/* A mixed batch as the one-launch frame-pair kernel reads it: the rows of
 * code c are base.order[code_start[c] .. + code_count[c]], taken through the
 * counter code_work[c]; code_shape[c] is the code's kernel shape
 * (mix_pair_shape); code_weight[c] its Tanner-graph edges; cta_code[k] the
 * first code of CTA k. */
struct MixPairParams {
    MixParams base;
    const int* code_start;
    const int* code_count;
    const int* code_shape;
    const int* code_weight;
    unsigned* code_work;
    const int* cta_code;
    int ncodes;
};

/* shape index of a one-CTA frame-pair kernel, -1 if the mixed kernel lacks it */
int mix_pair_shape(int a, int b, int gdm, int ls);
int decode_mix_pair_ctas_per_sm(size_t smem);
cudaError_t launch_decode_mix_pair(const MixPairParams& p, size_t smem, int grid, cudaStream_t stream);

/* (a, b, gdm, ls, pm) of frame-pair kernel kid (ldpc_pair.cu); false if none */
bool pair_kernel_shape(int kid, int* a, int* b, int* gdm, int* ls, int* pm);

}  // namespace drxg
