/*
 * Synthetic-frame generator (encoder, mapper, AWGN, max-log demapper) on the GPU.
 */
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "ldpc_device.h"

namespace drxg {

struct ChannelParams {
    const DevCode* code;
    unsigned long long seed;
    float n0;
    int bits;      /* bits per symbol */
    int qpsk;      /* closed-form QPSK, bits 2j and 2j+1 (no interleaver) */
    int order[8];  /* bit-interleaver column of label bit b */
    float re[256], im[256], e[256]; /* unit-energy points by label, |p|^2 */
    int8_t* llr;   /* nframes rows, or null */
    size_t llr_stride;
    __half* llr_f16; /* nframes rows of unquantised LLRs, or null */
    size_t llr_f16_stride;
    uint8_t* info; /* nframes rows of packed information bits, or null */
    size_t info_stride;
};

cudaError_t launch_channel(const ChannelParams& p, int nframes, int N, cudaStream_t s);

}  // namespace drxg
