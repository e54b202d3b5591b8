/*
 * Plain LDPC decoder for sm_100a: layered offset min-sum (offset 1) on
 * saturating int8 values, bit-exact to the reference C decoder
 * libdvbrx/src/ldpc.c (drx_ldpc_decode, ldpc.c:614-638).
 *
 * Mapping
 *   - one frame per CTA, persistent CTAs pulling frames from a counter;
 *   - the frame's posteriors live in shared memory for the whole decode:
 *     K information bits, then the R parity bits in layer order
 *     (parity of check q*j + i at K + 360*i + j, as ldpc.c:624-626);
 *   - 384 threads; in a layer step thread t runs one check node serially over
 *     its links, in registers (the reference's check_node, ldpc.c:321-362);
 *   - layers run in order; a layer whose checks share information bits runs
 *     as several steps (wavefront levels, see codes.h), one barrier each;
 *   - check-to-variable messages are kept compressed, as the reference's
 *     check_node_c keeps them (ldpc.c:376-462): both clamped minimums, the
 *     index of the link holding the smallest input and one sign bit per link,
 *     one 32-bit word per check (64-bit above degree 16), in a per-CTA
 *     scratch slab that stays in L2.  Each word is written and read back by
 *     the same thread only.
 *
 * Semantics kept from the reference
 *   - extrinsic input x = sat8(posterior - message); |x| taken as 0..128;
 *   - offset and the cap at 127 applied once per node to both minimums;
 *   - posterior = sat8(x + o) with the unclamped output o; the stored message
 *     is o clamped to [-32, 31];
 *   - syndrome before every iteration, a posterior of exactly 0 fails it
 *     (ldpc.c:286-305); iteration count and flag as drx_ldpc_decode returns;
 *   - hard decision bit = posterior < 0 over the first kldpc bits, packed
 *     MSB first (ldpc.c:581-612).
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "codes.h"
#include "ldpc_device.h"

namespace drxg {

constexpr int kQC = 360;

/* One 32-bit word per check up to degree 16 (6 + 6 + 4 bits, 16 signs),
 * two above (6 + 6 + 5 bits, 32 signs). */
template <int DMAX>
struct MsgWord {
    typedef typename std::conditional<(DMAX > 16), uint2, uint32_t>::type T;
};

/* meta = min0 (6 bits) | min1 << 6 | index << 12; signs: bit c = link c */
__device__ __forceinline__ void unpack(uint32_t w, uint32_t& meta, uint32_t& sg)
{
    meta = w & 0xFFFFu;
    sg = w >> 16;
}
__device__ __forceinline__ void unpack(uint2 w, uint32_t& meta, uint32_t& sg)
{
    meta = w.x;
    sg = w.y;
}
__device__ __forceinline__ void pack(uint32_t& w, uint32_t meta, uint32_t sg) { w = meta | sg << 16; }
__device__ __forceinline__ void pack(uint2& w, uint32_t meta, uint32_t sg) { w = make_uint2(meta, sg); }

__device__ __forceinline__ uint32_t ld_msg(const uint32_t* p) { return __ldcg(p); }
__device__ __forceinline__ uint2 ld_msg(const uint2* p) { return __ldcg(p); }
__device__ __forceinline__ void st_msg(uint32_t* p, uint32_t v) { __stcg(p, v); }
__device__ __forceinline__ void st_msg(uint2* p, uint2 v) { __stcg(p, v); }

__device__ __forceinline__ int sat8(int v) { return max(-128, min(127, v)); }

/*
 * One check node (i, j).  Links: slot 0 = its parity bit, slot 1 = the
 * previous parity bit (absent for check (0, 0)), slots 2.. = information
 * bits.  The result of a min-sum node does not depend on the link order, so
 * the parity links go first to sit at fixed register slots.
 */
template <int CNT, int IDXMASK>
__device__ __forceinline__ void check_node_n(int8_t* __restrict__ post, const int2* __restrict__ ent,
                                             int K, int q, int i, int j, bool first, uint32_t meta,
                                             uint32_t sgn, bool learned, uint32_t lw, uint32_t& meta_out,
                                             uint32_t& sgn_out)
{
    constexpr int D = CNT + 2;
    int addr[D];
    int x[D];
    const bool has_pp = (i | j) != 0;
    addr[0] = K + kQC * i + j;
    addr[1] = i ? addr[0] - kQC : K + kQC * (q - 1) + j - 1;
#pragma unroll
    for (int c = 2; c < D; c++) {
        const int2 e = ent[c - 2];
        addr[c] = e.x + j + (j < e.y ? kQC : 0);
    }

    const int idx = (meta >> 12) & IDXMASK;
    const int m0 = meta & 63, m1 = (meta >> 6) & 63;
    /* minus the stored message: +m if the message is negative, else -min(m, 31) */
    const int p0 = -min(m0, 31), n0 = m0, p1 = -min(m1, 31), n1 = m1;

    int min0 = 255, min1 = 255, sg = 0;
#pragma unroll
    for (int c = 0; c < D; c++) {
        int v;
        if (c == 1 && !has_pp) {
            v = 255; /* no link: larger than every |x|, positive */
        } else {
            v = post[addr[c]];
            if (!first) {
                const bool s = (sgn >> c) & 1u;
                const int nm = c == idx ? (s ? n1 : p1) : (s ? n0 : p0);
                v = sat8(v + nm);
            }
        }
        x[c] = v;
        const int a = abs(v);
        min1 = min(min1, max(min0, a));
        min0 = min(min0, a);
        sg ^= v;
    }
    const int mn0 = learned ? learned_mag(min(min0, 127), lw) : max(min(min0, 127) - 1, 0);
    const int mn1 = learned ? learned_mag(min(min1, 127), lw) : max(min(min1, 127) - 1, 0);
    int nidx = 0;
    uint32_t nsg = 0;
#pragma unroll
    for (int c = 0; c < D; c++) {
        const int v = x[c];
        const bool eq = abs(v) == min0;
        const int mag = eq ? mn1 : mn0;
        const int sm = (sg ^ v) >> 31; /* -1: negative output */
        const int o = (mag ^ sm) - sm;
        if (c != 1 || has_pp)
            post[addr[c]] = (int8_t)sat8(v + o);
        nidx = eq ? c : nidx;
        nsg |= (uint32_t)sm & (1u << c);
    }
    meta_out = (uint32_t)min(mn0, 32) | (uint32_t)min(mn1, 32) << 6 | (uint32_t)nidx << 12;
    sgn_out = nsg;
}

/* Dispatch on the layer's information-link count (uniform over the CTA):
 * every case is fully unrolled, with no predicated-off link slots. */
template <int DMAX>
__device__ __forceinline__ void check_node(int8_t* __restrict__ post, const int2* __restrict__ ent,
                                           int cnt, int K, int q, int i, int j, bool first,
                                           uint32_t meta, uint32_t sgn, bool learned, uint32_t lw,
                                           uint32_t& meta_out, uint32_t& sgn_out)
{
    constexpr int M = DMAX > 16 ? 31 : 15;
#define DRXG_CASE(n)                                                                           \
    case n:                                                                                    \
        if (n + 2 <= DMAX)                                                                     \
            check_node_n<(n + 2 <= DMAX ? n : 1), M>(post, ent, K, q, i, j, first, meta, sgn, \
                                                     learned, lw, meta_out, sgn_out);          \
        break;
    switch (cnt) {
        DRXG_CASE(1) DRXG_CASE(2) DRXG_CASE(3) DRXG_CASE(4) DRXG_CASE(5) DRXG_CASE(6)
        DRXG_CASE(7) DRXG_CASE(8) DRXG_CASE(9) DRXG_CASE(10) DRXG_CASE(11) DRXG_CASE(12)
        DRXG_CASE(13) DRXG_CASE(14) DRXG_CASE(15) DRXG_CASE(16) DRXG_CASE(17) DRXG_CASE(18)
        DRXG_CASE(19) DRXG_CASE(20) DRXG_CASE(21) DRXG_CASE(22) DRXG_CASE(23) DRXG_CASE(24)
        DRXG_CASE(25) DRXG_CASE(26) DRXG_CASE(27) DRXG_CASE(28) DRXG_CASE(29) DRXG_CASE(30)
    default:
        break;
    }
#undef DRXG_CASE
}

/* Shared-memory image of one code plus the frame's posteriors. */
struct Frame {
    int8_t* post;
    const int2* ent;
    const uint16_t* eoff;
    const uint32_t* steps;
};

__device__ __forceinline__ size_t align16(size_t v) { return (v + 15) & ~(size_t)15; }

/* Lay the code tables out after the posteriors and copy them in. */
__device__ Frame stage_code(const DevCode& c, char* smem)
{
    Frame f;
    f.post = (int8_t*)smem;
    size_t off = align16(c.N);
    int2* ent = (int2*)(smem + off);
    off += align16(sizeof(int2) * c.nent);
    uint16_t* eoff = (uint16_t*)(smem + off);
    off += align16(sizeof(uint16_t) * (c.q + 1));
    uint32_t* steps = (uint32_t*)(smem + off);
    for (int k = threadIdx.x; k < c.nent; k += blockDim.x)
        ent[k] = c.ent[k];
    for (int k = threadIdx.x; k <= c.q; k += blockDim.x)
        eoff[k] = c.eoff[k];
    for (int k = threadIdx.x; k < c.nsteps; k += blockDim.x)
        steps[k] = c.steps[k];
    f.ent = ent;
    f.eoff = eoff;
    f.steps = steps;
    return f;
}

/* LLRs of one frame into shared memory: information bits as they are, the
 * parity bits transposed to layer order (ldpc.c:624-626). */
__device__ void load_frame(const DevCode& c, const Frame& fr, const int8_t* __restrict__ src)
{
    const int t = threadIdx.x;
    if (((uintptr_t)src & 7) == 0) {
        const uint2* s8 = (const uint2*)src;
        for (int b = t; b < c.K / 8; b += blockDim.x)
            ((uint2*)fr.post)[b] = __ldcs(s8 + b);
        const uint32_t qm = 0xFFFFFFFFu / (uint32_t)c.q + 1u; /* k / q = umulhi(k, qm), k < 2^16 */
        for (int u = t; u < c.R / 8; u += blockDim.x) {
            const uint2 v = __ldcs(s8 + c.K / 8 + u);
#pragma unroll
            for (int r = 0; r < 8; r++) {
                const uint32_t k = 8u * u + r;
                const uint32_t jj = __umulhi(k, qm), ii = k - jj * c.q;
                const uint32_t word = r < 4 ? v.x : v.y;
                fr.post[c.K + kQC * ii + jj] = (int8_t)(word >> (8 * (r & 3)));
            }
        }
    } else {
        for (int b = t; b < c.K; b += blockDim.x)
            fr.post[b] = src[b];
        for (int k = t; k < c.R; k += blockDim.x)
            fr.post[c.K + kQC * (k % c.q) + k / c.q] = src[c.K + k];
    }
}

/* Syndrome before an iteration (ldpc.c:286-305): true if some check fails.
 * Thread t checks column t of every layer; the first failure stops all. */
__device__ bool syndrome_fails(const DevCode& c, const Frame& fr, volatile int* sflag)
{
    const int t = threadIdx.x;
    bool fail = false;
    if (t < kQC) {
        const int8_t* post = fr.post;
        for (int i = 0; i < c.q; i++) {
            if (*sflag)
                break;
            const int pc = post[c.K + kQC * i + t];
            const int pp = i ? post[c.K + kQC * (i - 1) + t]
                             : (t ? post[c.K + kQC * (c.q - 1) + t - 1] : 1);
            int s = pc ^ pp;
            bool z = pc == 0 || pp == 0;
            const int e1 = fr.eoff[i + 1];
            for (int e = fr.eoff[i]; e < e1; e++) {
                const int2 en = fr.ent[e];
                const int v = post[en.x + t + (t < en.y ? kQC : 0)];
                s ^= v;
                z |= v == 0;
            }
            if (z || s < 0) {
                fail = true;
                *sflag = 1;
                break;
            }
        }
    }
    return __syncthreads_or(fail);
}

/* One decoding iteration: every step (layer level) in order. */
template <int DMAX, bool LEARNED>
__device__ void iterate(const DevCode& c, const Frame& fr, typename MsgWord<DMAX>::T* __restrict__ msg,
                        bool first, int lrow)
{
    typedef typename MsgWord<DMAX>::T W;
    const int t = threadIdx.x;
    W wn = W();
    int jn = 0;
    auto fetch = [&](int s, W& w, int& jj) {
        const uint32_t st = fr.steps[s];
        const int i = st & 0xFF, start = (st >> 8) & 0x1FF, n = (st >> 17) & 0x1FF;
        if (t < n) {
            const int pos = start + t;
            jj = (st >> 26) ? (int)__ldg(c.perm + kQC * i + pos) : pos;
            if (!first)
                w = ld_msg(msg + kQC * i + pos);
        }
    };
    fetch(0, wn, jn);
    for (int s = 0; s < c.nsteps; s++) {
        const W w = wn;
        const int j = jn;
        const uint32_t st = fr.steps[s];
        const int i = st & 0xFF, start = (st >> 8) & 0x1FF, n = (st >> 17) & 0x1FF;
        if (s + 1 < c.nsteps)
            fetch(s + 1, wn, jn);
        if (t < n) {
            uint32_t meta = 0, sgn = 0, mo, so;
            if (!first)
                unpack(w, meta, sgn);
            const int e0 = fr.eoff[i];
            const int cnt = fr.eoff[i + 1] - e0;
            uint32_t lw = 0;
            if (LEARNED)
                lw = s_learn_tab[lrow + s_learn_cls[cnt + 2 - ((i | j) == 0)]];
            check_node<DMAX>(fr.post, fr.ent + e0, cnt, c.K, c.q, i, j, first, meta, sgn, LEARNED, lw, mo, so);
            W wo;
            pack(wo, mo, so);
            st_msg(msg + kQC * i + start + t, wo);
        }
        __syncthreads();
    }
}

/* Hard decisions of the first kldpc bits, MSB first. */
__device__ void store_bits(const DevCode& c, const Frame& fr, uint8_t* __restrict__ dst)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int nchunks = (c.kldpc + 31) / 32;
    for (int ch = warp; ch < nchunks; ch += nw) {
        const int b = ch * 32 + lane;
        const int v = b < c.kldpc ? fr.post[b] : 0;
        const unsigned m = __ballot_sync(0xFFFFFFFFu, v < 0);
        const unsigned r = __byte_perm(__brev(m), 0, 0x0123); /* byte k = output byte 4ch+k */
        if (lane < 4 && 4 * ch + lane < c.nbytes)
            dst[4 * ch + lane] = (uint8_t)(r >> (8 * lane));
    }
}

/* Group barrier of a team of G co-resident CTAs: returns 1 if every member
 * passed its syndrome, 0 if not, -1 if the barrier timed out after `limit`
 * polls (the device error word is set to 2).  skip: this CTA does not
 * arrive (a test of the time-out) and returns -1. */
__device__ int team_vote(unsigned* slot, int G, bool fail, int* err, int limit, bool skip)
{
    __shared__ int s_res;
    if (threadIdx.x == 0) {
        unsigned* arrive = slot;
        unsigned* fails = slot + 1;
        int res = 0;
        if (skip) {
            res = -1;
        } else {
            if (fail)
                atomicAdd(fails, 1u);
            __threadfence();
            atomicAdd(arrive, 1u);
            int spins = 0;
            while (*(volatile unsigned*)arrive < (unsigned)G) {
                if (++spins > limit) {
                    atomicExch(err, 2);
                    res = -1;
                    break;
                }
                __nanosleep(200);
            }
            __threadfence();
            if (res == 0)
                res = *(volatile unsigned*)fails == 0 ? 1 : 0;
        }
        s_res = res;
    }
    __syncthreads();
    const int r = s_res;
    __syncthreads();
    return r;
}

template <int DMAX>
__device__ __forceinline__ void decode_frame(const DevCode& c, const Frame& fr, const DecodeParams& p, int nframes, int f,
                             typename MsgWord<DMAX>::T* msg, volatile int* sflag, unsigned* sync, int lT)
{
    const bool real = f < nframes;
    const int row = real && p.rows ? p.rows[f] : f;
    if (real)
        load_frame(c, fr, p.llr + (size_t)row * p.llr_stride);
    __syncthreads();
    int it = 0;
    bool ok = true;
    for (;;) {
        bool fail = false;
        if (real)
            fail = syndrome_fails(c, fr, sflag);
        if (threadIdx.x == 0)
            *sflag = 0; /* read again only after later barriers */
        if (sync) {
            const int v = team_vote(sync + 2 * it, p.group, fail, p.err,
                                    p.wait_limit > 0 ? p.wait_limit : kDefaultWaitLimit,
                                    (int)blockIdx.x + 1 == p.skip_vote);
            ok = v == 1;
            if (v < 0)
                break;
        } else {
            ok = !fail;
        }
        if (ok || it >= p.max_iter)
            break;
        if (real) {
            if (lT)
                iterate<DMAX, true>(c, fr, msg, it == 0, learn_row(it, lT));
            else
                iterate<DMAX, false>(c, fr, msg, it == 0, 0);
        }
        it++;
    }
    if (real) {
        store_bits(c, fr, p.out + (size_t)row * p.out_stride);
        if (threadIdx.x == 0) {
            if (p.iters)
                p.iters[row] = it;
            if (p.ok)
                p.ok[row] = ok ? 1 : 0;
        }
    }
    __syncthreads();
}

template <int DMAX, int MINB>
__global__ void __launch_bounds__(kThreads, MINB) k_decode(DecodeParams p)
{
    extern __shared__ __align__(16) char smem[];
    __shared__ int s_frame;
    __shared__ int s_flag;
    const DevCode c = *p.code;
    const Frame fr = stage_code(c, smem);
    const int lT = stage_learn(p.learn, p.learn_class, p.learn_iters);
    const int nframes = p.nframes_dev ? *p.nframes_dev : p.nframes;
    typedef typename MsgWord<DMAX>::T W;
    W* msg = (W*)((char*)p.msg + (size_t)blockIdx.x * p.msg_stride);
    if (threadIdx.x == 0)
        s_flag = 0;
    __syncthreads();
    if (p.group == 0) {
        for (;;) {
            if (threadIdx.x == 0)
                s_frame = (int)atomicAdd(p.work, 1u);
            __syncthreads();
            const int f = s_frame;
            __syncthreads();
            if (f >= nframes)
                break;
            decode_frame<DMAX>(c, fr, p, nframes, f, msg, &s_flag, nullptr, lT);
        }
    } else {
        const int G = p.group;
        const int team = blockIdx.x / G, member = blockIdx.x % G;
        const int ngroups = (p.nframes + G - 1) / G;
        const int per = p.max_iter + 1;
        for (int g = team, k = 0; g < ngroups; g += p.nteams, k++) {
            unsigned* sync = p.team_sync + 2 * (size_t)per * ((size_t)team * ((ngroups + p.nteams - 1) / p.nteams) + k);
            decode_frame<DMAX>(c, fr, p, nframes, g * G + member, msg, &s_flag, sync, lT);
        }
    }
}

/* Mixed batch, one launch: frames of several codes in `order` (longest
 * work first), one frame per CTA; the code tables are restaged when the
 * next frame's code differs from the one in shared memory. */
template <int DMAX, int MINB>
__global__ void __launch_bounds__(kThreads, MINB) k_decode_mix(MixParams mp)
{
    extern __shared__ __align__(16) char smem[];
    __shared__ int s_k;
    __shared__ int s_flag;
    typedef typename MsgWord<DMAX>::T W;
    W* msg = (W*)((char*)mp.msg + (size_t)blockIdx.x * mp.msg_stride);
    DecodeParams p{};
    p.llr = mp.llr;
    p.llr_stride = mp.llr_stride;
    p.out = mp.out;
    p.out_stride = mp.out_stride;
    p.iters = mp.iters;
    p.ok = mp.ok;
    p.nframes = mp.nframes;
    p.max_iter = mp.max_iter;
    p.rows = mp.order;
    if (threadIdx.x == 0)
        s_flag = 0;
    int staged = -1;
    DevCode c{};
    Frame fr{};
    int lT = 0;
    const int nframes = mp.nframes_dev ? *mp.nframes_dev : mp.nframes;
    for (;;) {
        if (threadIdx.x == 0)
            s_k = (int)atomicAdd(mp.work, 1u);
        __syncthreads();
        const int k = s_k;
        __syncthreads();
        if (k >= nframes)
            break;
        const int ci = mp.frame_code[mp.order[k]];
        if (ci != staged) {
            c = *mp.codes[ci];
            fr = stage_code(c, smem);
            lT = mp.learn ? stage_learn(mp.learn[ci], mp.learn_class[ci], mp.learn_iters[ci]) : 0;
            staged = ci;
            __syncthreads();
        }
        decode_frame<DMAX>(c, fr, p, nframes, k, msg, &s_flag, nullptr, lT);
    }
}

static const void* mix_kernel_for(int dclass)
{
    switch (dclass) {
    case 0:
        return (const void*)k_decode_mix<7, 4>;
    case 1:
        return (const void*)k_decode_mix<11, 3>;
    case 2:
        return (const void*)k_decode_mix<14, 3>;
    case 3:
        return (const void*)k_decode_mix<18, 2>;
    case 4:
        return (const void*)k_decode_mix<22, 2>;
    default:
        return (const void*)k_decode_mix<32, 1>;
    }
}

int decode_mix_ctas_per_sm(int dclass, size_t smem)
{
    const void* k = mix_kernel_for(dclass);
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return 0;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, kThreads, smem) != cudaSuccess)
        return 0;
    return n;
}

cudaError_t launch_decode_mix(const MixParams& p, int dclass, size_t smem, int grid, cudaStream_t stream)
{
    const void* k = mix_kernel_for(dclass);
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
        return e;
    MixParams pc = p;
    void* args[] = { &pc };
    return cudaLaunchKernel(k, dim3(grid), dim3(kThreads), args, smem, stream);
}

size_t decode_smem_bytes(int N, int nent, int nsteps, int q)
{
    auto a16 = [](size_t v) { return (v + 15) & ~(size_t)15; };
    return a16(N) + a16(sizeof(int2) * nent) + a16(sizeof(uint16_t) * (q + 1)) +
           a16(sizeof(uint32_t) * nsteps);
}

size_t decode_msg_bytes(int R, int dclass)
{
    return (size_t)R * (kClassDeg[dclass < 0 ? kNumClasses - 1 : dclass] > 16 ? 8 : 4);
}

template <int DMAX, int MINB>
static const void* kernel_ptr()
{
    return (const void*)k_decode<DMAX, MINB>;
}

static const void* kernel_for(int dclass)
{
    static_assert(kNumClasses == 6, "one kernel per degree class");
    switch (dclass) {
    case 0:
        return kernel_ptr<7, 4>();
    case 1:
        return kernel_ptr<11, 3>();
    case 2:
        return kernel_ptr<14, 3>();
    case 3:
        return kernel_ptr<18, 2>();
    case 4:
        return kernel_ptr<22, 2>();
    default:
        return kernel_ptr<32, 1>();
    }
}

int decode_ctas_per_sm(int dclass, size_t smem)
{
    const void* k = kernel_for(dclass);
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return 0;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, kThreads, smem) != cudaSuccess)
        return 0;
    return n;
}

cudaError_t launch_decode(const DecodeParams& p, int dclass, size_t smem, int grid, cudaStream_t stream)
{
    const void* k = kernel_for(dclass);
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
        return e;
    DecodeParams pc = p;
    void* args[] = { &pc };
    if (p.group > 0)
        return cudaLaunchCooperativeKernel(k, dim3(grid), dim3(kThreads), args, smem, stream);
    return cudaLaunchKernel(k, dim3(grid), dim3(kThreads), args, smem, stream);
}

}  // namespace drxg
