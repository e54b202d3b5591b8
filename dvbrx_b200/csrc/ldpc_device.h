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
    const int* nframes_dev; /* per-frame mode, optional: the number of work items, read on
                               the device at kernel start (replaces nframes) */
    const uint32_t* learn; /* learned check nodes (null: the plain offset 1): learn_iters
                              rows of kLearnClasses words, see learned_mag */
    const int8_t* learn_class; /* degree class of every check degree 0..32 */
    int learn_iters;
    int wait_limit;        /* group mode: polls of a group barrier before the launch gives
                              up and sets the error word to 2 (0: kDefaultWaitLimit) */
    int skip_vote;         /* group mode, testing only: CTA skip_vote - 1 never arrives at
                              its team's barriers (the others time out); 0: none */
};

/* Polls of a group barrier (about 200 ns apart) before it gives up. */
constexpr int kDefaultWaitLimit = 1 << 22;

/* Learned check nodes (the neural offset / scaled min-sum at int8): the
 * outgoing magnitude of a node in iteration t is
 *     max((scale * m - offset + 128) >> 8, 0),   m = min(minimum, 127),
 * with scale and offset in Q8 from row min(t, learn_iters - 1) and the
 * check's degree class: word = scale (16 bits) | offset (signed 16) << 16.
 * Scale 256 and offset 256 give max(m - 1, 0), the plain decoder. */
constexpr int kLearnClasses = 8;
constexpr int kLearnMaxIters = 32;
#ifdef __CUDACC__
__device__ __forceinline__ int learned_mag(int m, uint32_t w)
{
    return max(((int)(w & 0xFFFFu) * m - ((int)w >> 16) + 128) >> 8, 0);
}

/* The learned table of a launch, staged in shared memory by stage_learn
 * (one copy per translation unit; kernels that never stage it do not
 * allocate it). */
static __shared__ uint32_t s_learn_tab[kLearnMaxIters * kLearnClasses];
static __shared__ int8_t s_learn_cls[33];

/* Stage a learned table (T rows of kLearnClasses words, classes of the
 * degrees 0..32); returns the staged row count, 0 for the plain decoder.
 * The caller synchronises the block before the table is read. */
__device__ __forceinline__ int stage_learn(const uint32_t* tab, const int8_t* cls, int T)
{
    if (!tab || !cls || T <= 0)
        return 0;
    T = min(T, kLearnMaxIters);
    for (int k = threadIdx.x; k < T * kLearnClasses; k += blockDim.x)
        s_learn_tab[k] = tab[k];
    for (int k = threadIdx.x; k < 33; k += blockDim.x)
        s_learn_cls[k] = cls[k];
    return T;
}

/* First word of the learned row of iteration `it` (T > 0). */
__device__ __forceinline__ int learn_row(int it, int T) { return kLearnClasses * min(it, T - 1); }
#endif

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
    /* learned check nodes per code index (null entries, or a null array:
     * the plain offset 1); layout as DecodeParams::learn */
    const uint32_t* const* learn;
    const int8_t* const* learn_class;
    const int* learn_iters;
    const int* nframes_dev; /* optional: the number of rows of `order`, read on the device */
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
 * up to check degree 32; per-frame stopping, or group stopping on teams of
 * co-resident CTAs.  pair_kernel_id picks the one-CTA-per-SM instantiation
 * for a code (-1: not run by the frame-pair kernel); pair_kernel_twin gives
 * its two-CTA forms. */
struct Code;
int pair_kernel_id(const Code& c);
/* The twin of kernel kid compiled for two CTAs per SM: pm 1 keeps every
 * posterior in shared memory, pm 2 keeps the parity posteriors in the CTA's
 * global slab and in registers (about half the shared memory); -1 if none */
int pair_kernel_twin(int kid, int pm);
size_t decode_pair_smem_bytes(int N, int K, int nent, int nsteps, int q, int kid);
size_t decode_pair_msg_bytes(int R, int kid);
int decode_pair_ctas_per_sm(int kid, size_t smem);
cudaError_t launch_decode_pair(const DecodeParams& p, int kid, size_t smem, int grid, cudaStream_t stream);

}  // namespace drxg
