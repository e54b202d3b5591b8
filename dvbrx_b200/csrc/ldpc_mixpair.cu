/*
 * Mixed batches in one persistent launch with two frames per CTA.
 *
 * The frame-pair decoder (ldpc_pair.cuh) is compiled per code shape; a
 * mixed batch holds frames of many codes.  This kernel holds the shapes of
 * the DVB-S2 codes (normal and short frames) behind one switch: a CTA takes
 * a code, stages its tables in shared memory and runs that code's frames
 * with the shape's streaming loop (two lanes, each taking the code's next
 * frame when its own is done), pulling from the code's own counter.  When
 * the code has no frames left, the CTA takes the code with the most work
 * left and restages.  CTAs start spread over the codes in proportion to
 * their work (edges x frames), so that each CTA changes code a few times
 * only and every change costs at most one lane idling while the other
 * finishes its last frame of the old code.
 *
 * One CTA per SM (the largest shapes, check degree up to 30, need up to 168
 * registers, and normal frames at rate 8/9 and 9/10 fill shared memory), so
 * every code runs its one-CTA shape.  Plain decoding (offset 1), per-frame
 * stopping; results identical to every other kernel of the library.
 */
#include <cuda_runtime.h>

#include "ldpc_pair.cuh"
#include "mixpair.h"

namespace drxg {

/* the shapes behind the switch: (A, B, GDM, LS) of the one-CTA frame-pair
 * kernels that pair_kernel_id picks for the DVB-S2 codes */
#define DRXG_MIX_SHAPES(X)                                                                               \
    X(0, 1, 2, 0, 2) X(1, 2, 2, 0, 2) X(2, 3, 3, 0, 2) X(3, 4, 4, 0, 2) X(4, 5, 5, 0, 2) X(5, 8, 8, 0, 2) \
    X(6, 9, 9, 0, 2) X(7, 12, 12, 0, 2) X(8, 9, 9, 0, 3) X(9, 16, 16, 0, 4) X(10, 20, 20, 0, 3)          \
    X(11, 25, 25, 0, 6) X(12, 28, 28, 0, 4) X(13, 1, 1, 7, 3) X(14, 1, 1, 14, 3) X(15, 1, 1, 22, 5)

/* One code's frames with its shape: its tables staged in the shape's form,
 * then the streaming loop of the frame-pair kernel. */
template <int A, int B, int GDM, int LS>
__device__ __noinline__ void mix_code_frames(const DecodeParams& p, const DevCode& c, char* smem, void* msg,
                                             PairLanes& st)
{
    const PairFrame fr = stage_pair<false, pair_key_form(A, B, GDM, LS)>(c, smem, nullptr);
    __syncthreads();
    stream_frames<A, B, GDM, LS, false>(p, c, fr, msg, 0, p.nframes, st);
}

/* The code with the most work left (frames not yet taken x edges), -1 if none. */
__device__ int mix_next_code(const MixPairParams& mp)
{
    int best = -1;
    long long most = 0;
    for (int c = 0; c < mp.ncodes; c++) {
        const unsigned taken = *(volatile unsigned*)(mp.code_work + c);
        const int left = mp.code_count[c] - (int)min(taken, (unsigned)mp.code_count[c]);
        const long long w = (long long)left * mp.code_weight[c];
        if (left > 0 && w > most) {
            most = w;
            best = c;
        }
    }
    return best;
}

__global__ void __launch_bounds__(384, 1) k_decode_mix_pair(MixPairParams mp)
{
    extern __shared__ __align__(16) char smem[];
    __shared__ PairLanes st;
    __shared__ int s_code;
    const int t = threadIdx.x;
    void* msg = (char*)mp.base.msg + (size_t)blockIdx.x * mp.base.msg_stride;
    if (t == 0)
        s_code = mp.cta_code[blockIdx.x];
    __syncthreads();
    for (int code = s_code; code >= 0;) {
        const DevCode c = *mp.base.codes[code];
        if (t == 0) {
            st.frame[0] = st.frame[1] = -1;
            st.flag = 0;
            st.reload = 3;
            st.row[0] = st.row[1] = 0;
        }
        __syncthreads();
        DecodeParams p{};
        p.code = mp.base.codes[code];
        p.llr = mp.base.llr;
        p.llr_stride = mp.base.llr_stride;
        p.out = mp.base.out;
        p.out_stride = mp.base.out_stride;
        p.iters = mp.base.iters;
        p.ok = mp.base.ok;
        p.nframes = mp.code_count[code];
        p.max_iter = mp.base.max_iter;
        p.rows = mp.base.order + mp.code_start[code];
        p.work = mp.code_work + code;
        switch (mp.code_shape[code]) {
#define DRXG_MIX_CASE(k, a, b, g, ls)                    \
    case k:                                              \
        mix_code_frames<a, b, g, ls>(p, c, smem, msg, st); \
        break;
            DRXG_MIX_SHAPES(DRXG_MIX_CASE)
#undef DRXG_MIX_CASE
        default:
            break;
        }
        __syncthreads(); /* every thread done with this code's tables */
        if (t == 0)
            s_code = mix_next_code(mp);
        __syncthreads();
        code = s_code;
    }
}

/* The shape index of a one-CTA frame-pair kernel (a, b, gdm, ls), -1 if the
 * switch does not hold it. */
int mix_pair_shape(int a, int b, int gdm, int ls)
{
    int k = -1;
#define DRXG_MIX_FIND(i, aa, bb, gg, ll)                          \
    if (gg == gdm && ll == ls && (gg > 0 || (aa == a && bb == b))) \
        k = k < 0 ? i : k;
    DRXG_MIX_SHAPES(DRXG_MIX_FIND)
#undef DRXG_MIX_FIND
    return k;
}

int decode_mix_pair_ctas_per_sm(size_t smem)
{
    if (cudaFuncSetAttribute((const void*)k_decode_mix_pair, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return 0;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, (const void*)k_decode_mix_pair, 384, smem) != cudaSuccess)
        return 0;
    return n;
}

cudaError_t launch_decode_mix_pair(const MixPairParams& p, size_t smem, int grid, cudaStream_t stream)
{
    cudaError_t e = cudaFuncSetAttribute((const void*)k_decode_mix_pair, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess)
        return e;
    MixPairParams pc = p;
    void* args[] = { &pc };
    return cudaLaunchKernel((const void*)k_decode_mix_pair, dim3(grid), dim3(384), args, smem, stream);
}

}  // namespace drxg
