/*
 * Device-side code descriptor and the launchers of the plain decoder.
 */
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace drxg {

constexpr int kThreads = 384; /* 360 checks of a layer, 12 warps */

/* One code as the kernels read it (device memory). */
struct DevCode {
    int N, K, R, q, kldpc, nbytes;
    int nent, nsteps, dclass;
    int pad;
    const int2* ent;       /* nent pairs (360 g - a, a), layer-major */
    const uint16_t* eoff;  /* q + 1 */
    const uint32_t* steps; /* nsteps: layer | start << 8 | count << 17 | perm << 26 */
    const uint16_t* perm;  /* q * 360 */
    const uint8_t* nlev;   /* q: wavefront levels of each layer */
    const unsigned long long* lmeta; /* q * 360: level | in slots << 8 | out slots << 32 */
};

/* Work of one launch of the plain decoder. */
struct DecodeParams {
    const DevCode* code;   /* device pointer */
    const int8_t* llr;     /* nframes rows of llr_stride bytes (N used) */
    size_t llr_stride;
    uint8_t* out;          /* nframes rows of out_stride bytes (nbytes used) */
    size_t out_stride;
    int32_t* iters;        /* nframes, may be null */
    uint8_t* ok;           /* nframes, may be null */
    int nframes;
    int max_iter;
    int group;             /* 0: each frame stops on its own; G > 0: groups of G
                              consecutive frames stop together (reference
                              batch semantics), launched cooperatively */
    int nteams;            /* group mode: grid / group */
    unsigned* work;        /* per-frame mode: frame counter, zeroed by the launcher */
    unsigned* team_sync;   /* group mode: 2 * nteams * groups_per_team * (max_iter + 1) */
    void* msg;             /* message scratch: grid * msg_stride bytes */
    size_t msg_stride;
    int* err;              /* device error word (0 = fine) */
    const int32_t* rows;   /* per-frame mode, optional: work item k is row rows[k] of
                              llr / out / iters / ok (null: row k) */
};

/* A batch of frames of several codes (one launch over all of them). */
struct MixParams {
    const DevCode* const* codes; /* device array: code of each code index */
    const int32_t* frame_code;   /* code index of every row */
    const int32_t* order;        /* rows in processing order (nframes) */
    const int8_t* llr;
    size_t llr_stride;
    uint8_t* out;
    size_t out_stride;
    int32_t* iters;
    uint8_t* ok;
    int nframes;
    int max_iter;
    unsigned* work;
    void* msg;
    size_t msg_stride;
};

/* One persistent launch over a mixed batch: one frame per CTA, the CTA
 * restages the code tables in shared memory when the next frame's code
 * differs.  `dclass` is the largest degree class of the mix. */
cudaError_t launch_decode_mix(const MixParams& p, int dclass, size_t smem, int grid, cudaStream_t stream);
int decode_mix_ctas_per_sm(int dclass, size_t smem);

/* Largest dynamic shared memory of the plain kernel for a code. */
size_t decode_smem_bytes(int N, int nent, int nsteps, int q);
/* Message scratch per CTA. */
size_t decode_msg_bytes(int R, int dclass);
/* Resident CTAs per SM of the plain kernel for a class and smem size. */
int decode_ctas_per_sm(int dclass, size_t smem);

/* Launch the plain decoder on `grid` CTAs.  Group mode uses a cooperative
 * launch (co-resident CTAs are required by the group barrier). */
cudaError_t launch_decode(const DecodeParams& p, int dclass, size_t smem, int grid,
                          cudaStream_t stream);

}  // namespace drxg

namespace drxg {

/* Frame-pair variant (ldpc_pair.cu): two frames per CTA in 16x2 SIMD, codes
 * up to check degree 14; per-frame stopping only.  pair_kernel_id picks the
 * instantiation for a code (-1: not run by the frame-pair kernel). */
struct Code;
int pair_kernel_id(const Code& c);
size_t decode_pair_smem_bytes(int N, int nent, int nsteps, int q);
size_t decode_pair_msg_bytes(int R);
int decode_pair_ctas_per_sm(int kid, size_t smem);
cudaError_t launch_decode_pair(const DecodeParams& p, int kid, size_t smem, int grid, cudaStream_t stream);

}  // namespace drxg
