/*
 * Synthetic DVB-S2 frames on the GPU: the input source of the benchmark and
 * of the learned decoder's training.  One CTA per frame:
 *
 *   1. information bits from a counter-based generator (Philox4x32-10,
 *      Salmon et al., "Parallel random numbers: as easy as 1, 2, 3", SC 2011)
 *      keyed by (seed, frame);
 *   2. the systematic encoder of EN 302 307-1 5.3.2 in the layer form of the
 *      decoder's code: parity p_k of check k = q*j + i is the XOR of the
 *      check's information links, then p_k ^= p_{k-1} (a block-wide prefix XOR);
 *   3. the bit interleaver and mapping of the MODCOD (bit b of symbol j is
 *      codeword bit order[b] * nsym + j; QPSK: bits 2j, 2j+1), unit average
 *      energy points;
 *   4. complex AWGN of power n0 = 10^(-Es/N0 / 10) per symbol (Box-Muller);
 *   5. the max-log demapper with the reference receiver's scale and
 *      quantiser (libdvbrx/src/demap.c:32-34,225-229,491-533): LLR =
 *      quantise(2/n0 * (min_{bit=1} d - min_{bit=0} d)), d = |p|^2 - 2 Re(y p*)
 *      formed as x*(-2 re) + (y*(-2 im) + |p|^2) with fused multiply-adds,
 *      QPSK in closed form 2/n0 * 4/sqrt(2) * component; quantise = clamp to
 *      +-127 then round half to even.  Optionally the unquantised values as
 *      FP16 (for training).
 */
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "channel.h"

namespace drxg {

constexpr int kChThreads = 512;
constexpr int kQCc = 360;

/* Philox4x32-10 */
struct P4 {
    uint32_t x, y, z, w;
};
__device__ __forceinline__ P4 philox(P4 c, uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; r++) {
        const uint32_t hi0 = __umulhi(0xD2511F53u, c.x), lo0 = 0xD2511F53u * c.x;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z), lo1 = 0xCD9E8D57u * c.z;
        c = P4{ hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0 };
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

__device__ __forceinline__ float u01(uint32_t v) { return ((float)(v >> 8) + 0.5f) * (1.0f / 16777216.0f); }

__device__ __forceinline__ int quantise(float v)
{
    v = fminf(fmaxf(v, -127.0f), 127.0f);
    return __float2int_rn(v);
}

__global__ void __launch_bounds__(kChThreads) k_channel(ChannelParams p)
{
    extern __shared__ __align__(16) uint8_t cw[]; /* N codeword bits, one per byte */
    __shared__ uint32_t scan[kChThreads];
    const DevCode c = *p.code;
    const int f = blockIdx.x;
    const int t = threadIdx.x;
    const uint32_t k0 = (uint32_t)p.seed, k1 = (uint32_t)(p.seed >> 32);

    /* 1. information bits: counter (frame, block of 128 bits, stream 0) */
    for (int b = t; b < (c.K + 127) / 128; b += blockDim.x) {
        const P4 r = philox(P4{ (uint32_t)b, (uint32_t)f, 0u, 0x494E464Fu }, k0, k1);
        const uint32_t w[4] = { r.x, r.y, r.z, r.w };
        for (int k = 0; k < 128; k++) {
            const int idx = b * 128 + k;
            if (idx < c.K)
                cw[idx] = (w[k >> 5] >> (k & 31)) & 1u;
        }
    }
    __syncthreads();

    /* 2. parity: check k = q*j + i sums information bits 360 g - a + j (+360) */
    for (int k = t; k < c.R; k += blockDim.x) {
        const int j = k / c.q, i = k - j * c.q;
        uint32_t s = 0;
        for (int e = c.eoff[i]; e < c.eoff[i + 1]; e++) {
            const int2 en = c.ent[e];
            s ^= cw[en.x + j + (j < en.y ? kQCc : 0)];
        }
        cw[c.K + k] = (uint8_t)s;
    }
    __syncthreads();
    /* accumulator: prefix XOR over the R parity bits, chunk per thread */
    const int chunk = (c.R + blockDim.x - 1) / blockDim.x;
    const int lo = t * chunk, hi = min(c.R, lo + chunk);
    uint32_t acc = 0;
    for (int k = lo; k < hi; k++)
        acc ^= cw[c.K + k];
    scan[t] = acc;
    __syncthreads();
    /* exclusive prefix XOR of the chunk sums (Hillis-Steele on 512 words) */
    for (int off = 1; off < (int)blockDim.x; off <<= 1) {
        const uint32_t v = t >= off ? scan[t - off] : 0u;
        __syncthreads();
        scan[t] ^= v;
        __syncthreads();
    }
    uint32_t run = t ? scan[t - 1] : 0u;
    for (int k = lo; k < hi; k++) {
        run ^= cw[c.K + k];
        cw[c.K + k] = (uint8_t)run;
    }
    __syncthreads();

    /* information bits out, packed MSB first */
    if (p.info) {
        uint8_t* dst = p.info + (size_t)f * p.info_stride;
        for (int B = t; B < c.nbytes; B += blockDim.x) {
            uint32_t v = 0;
            for (int k = 0; k < 8; k++) {
                const int idx = 8 * B + k;
                v = (v << 1) | (idx < c.kldpc ? cw[idx] : 0u);
            }
            dst[B] = (uint8_t)v;
        }
    }

    /* 3-5. symbols, noise, demapper */
    const float n0 = p.n0, sig = sqrtf(0.5f * n0), kk = 2.0f / n0;
    int8_t* llr = p.llr ? p.llr + (size_t)f * p.llr_stride : nullptr;
    __half* llrh = p.llr_f16 ? p.llr_f16 + (size_t)f * p.llr_f16_stride : nullptr;
    const int bits = p.bits, np = 1 << bits;
    const int nsym = (c.N + bits - 1) / bits;
    for (int j = t; j < nsym; j += blockDim.x) {
        const P4 r = philox(P4{ (uint32_t)j, (uint32_t)f, 1u, 0x5eedu }, k0, k1);
        const float rad = sqrtf(-2.0f * logf(u01(r.x)));
        float sn, cs;
        sincospif(2.0f * u01(r.y), &sn, &cs);
        const float nx = sig * rad * cs, ny = sig * rad * sn;
        if (p.qpsk) {
            const int b0 = cw[2 * j], b1 = cw[2 * j + 1];
            const float x = (b0 ? -p.re[0] : p.re[0]) + nx;
            const float y = (b1 ? -p.im[0] : p.im[0]) + ny;
            const float kq = kk * 4.0f * 0.70710678118654752f;
            const float vx = __fmul_rn(kq, x), vy = __fmul_rn(kq, y);
            if (llr) {
                llr[2 * j] = (int8_t)quantise(vx);
                llr[2 * j + 1] = (int8_t)quantise(vy);
            }
            if (llrh) {
                llrh[2 * j] = __float2half_rn(vx);
                llrh[2 * j + 1] = __float2half_rn(vy);
            }
            continue;
        }
        int label = 0;
        for (int b = 0; b < bits; b++) {
            const int pos = p.order[b] * nsym + j;
            label = (label << 1) | (pos < c.N ? cw[pos] : 0);
        }
        const float x = p.re[label] + nx, y = p.im[label] + ny;
        float m0[8], m1[8];
        for (int b = 0; b < bits; b++) {
            m0[b] = 3.0e38f;
            m1[b] = 3.0e38f;
        }
        for (int q = 0; q < np; q++) {
            const float d = fmaf(x, -2.0f * p.re[q], fmaf(y, -2.0f * p.im[q], p.e[q]));
            for (int b = 0; b < bits; b++) {
                if ((q >> (bits - 1 - b)) & 1)
                    m1[b] = fminf(m1[b], d);
                else
                    m0[b] = fminf(m0[b], d);
            }
        }
        for (int b = 0; b < bits; b++) {
            const int pos = p.order[b] * nsym + j;
            if (pos >= c.N)
                continue;
            const float v = __fmul_rn(kk, __fsub_rn(m1[b], m0[b]));
            if (llr)
                llr[pos] = (int8_t)quantise(v);
            if (llrh)
                llrh[pos] = __float2half_rn(v);
        }
    }
}

cudaError_t launch_channel(const ChannelParams& p, int nframes, int N, cudaStream_t s)
{
    const size_t smem = ((size_t)N + 15) & ~(size_t)15;
    cudaError_t e = cudaFuncSetAttribute(k_channel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
        return e;
    k_channel<<<nframes, kChThreads, smem, s>>>(p);
    return cudaGetLastError();
}

}  // namespace drxg
