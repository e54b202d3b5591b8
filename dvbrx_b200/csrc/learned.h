/*
 * Learned (neural offset / scaled) min-sum: training kernels and parameters.
 */
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "ldpc_device.h"

namespace drxg {

constexpr int kLearnedMaxDeg = 32;  /* links of a check node */
constexpr int kLearnedMaxClass = 8; /* check-degree classes */

/* One training or evaluation launch over nframes frames of one code. */
struct LearnedParams {
    const DevCode* code; /* device */
    int nframes;
    int iters;
    int DS;              /* message slots per check: the code's largest degree */
    const __half* llr;   /* nframes rows of llr_stride halves: unquantised 2 x LLR */
    size_t llr_stride;
    const uint8_t* bits; /* nframes rows: kldpc information bits, MSB first */
    size_t bits_stride;
    const __half* beta;  /* iters x nclass FP16 scales */
    const __half* alpha; /* iters x nclass FP16 offsets */
    int nclass;
    const int8_t* cls;   /* class of each check degree 0..32 (device) */
    float* P;            /* workspace: nframes x N posteriors */
    float* M;            /* nframes x DS*R messages */
    float* X;            /* backward: nframes x DS*R extrinsic inputs */
    float* gP;           /* backward: nframes x N */
    float* gM;           /* backward: nframes x DS*R */
    float* Pck;          /* training: iters x nframes x N checkpoints (null: none) */
    float* Mck;          /* iters x nframes x DS*R */
    float* loss;         /* iters: sums of the BCE of every iteration's output */
    float* dbeta;        /* backward: iters x nclass */
    float* dalpha;
    float loss_scale;    /* backward: d loss / d (each per-iteration BCE sum) */
    const float* loss_w; /* backward, optional: per-iteration weights of the BCE sums (device) */
    float* post;         /* forward, optional: nframes x kldpc final posteriors */
};

size_t learned_workspace_bytes(const DevCode& host_code_shape, int R, int N, int DS, int nframes, int iters,
                               bool train);
cudaError_t launch_learned(const LearnedParams& p, bool backward, cudaStream_t s);

}  // namespace drxg
