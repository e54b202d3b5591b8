/*
 * The soft demapper of the reference receiver on the GPU
 * (libdvbrx/src/demap.c:491-533, drx_demap_frame): received symbols of a
 * PLFRAME (complex, interleaved float I/Q, unit average energy) to the
 * decoder's int8 LLRs in codeword order, ahead of the LDPC decoder on the
 * same stream.
 *
 * Max-log LLRs on the reference's scale: for bit b of symbol j,
 *     LLR = quantise(2/n0 * (min_{label bit b = 1} d - min_{bit b = 0} d)),
 *     d = x (-2 re p) + (y (-2 im p) + |p|^2)   (two fused multiply-adds,
 *         as the reference's vector paths form it, demap.c:318-330),
 * quantise = clamp to +-127 then round half to even; bit b of symbol j goes
 * to codeword position order[b] * nsym + j (the bit interleaver).  QPSK has
 * no interleaver and the closed form LLR = 2/n0 * 4/sqrt(2) * component.
 * Points are the standard's, normalised to unit average energy
 * (demap.c:183-190).  The results equal the reference's builds with fused
 * multiply-adds (AVX2, AVX-512); its SSE2 build rounds the two products
 * separately and can differ by one unit on rare ties.
 *
 * Constellations of 64 to 256 points take the minima by groups of 16 points
 * (the four low label bits inside a group, the high ones from the groups'
 * minima; a minimum does not depend on its order, so the LLRs are the full
 * search's).  The 256APSK tables made of 8 rings of the same 32 phases take
 * the reference's ring metric instead (demap.c:447-496), whose minima equal
 * the full search's only up to rounding: c_j (-2 R_r) + R_r^2 with c_j the
 * projection of the symbol on phase j.
 *
 * Grid rows walk the frames, threads take four consecutive symbols (16-byte
 * loads, 4-byte stores per bit column); the points and their constants are
 * kernel parameters (constant bank).
 */
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <string>

#include "../../include/dvbrx_b200.h"
#include "codes_gen.h"
#include "handle.h"

namespace drxg {

struct DemapParams {
    int bits, nsym, nldpc, qpsk;
    int order[8];
    float ar[256], ai[256], e[256]; /* -2 re, -2 im, |p|^2 */
    /* 256-point constellations made of 8 rings of the same 32 phases (ring in
     * the high label bits): unit phase vectors (rc, rs), -2 R and R^2 */
    int ring;
    float rc[32], rs[32], rm2[8], rr2[8];
    const float* sym;
    size_t sym_stride; /* floats per frame */
    const float* n0;   /* per frame */
    int8_t* llr;
    size_t llr_stride;
    int nframes;
};

__device__ __forceinline__ int8_t quantise8(float v)
{
    v = fminf(fmaxf(v, -127.0f), 127.0f);
    return (int8_t)__float2int_rn(v);
}

/* LLRs of one symbol, label bit b in out[b] */
template <int BITS>
__device__ __forceinline__ void demap_symbol(const DemapParams& p, float x, float y, float k, int8_t* out)
{
    if (BITS == 2) {
        const float kq = k * 4.0f * 0.70710678118654752f; /* demap.c:496-500 */
        out[0] = quantise8(__fmul_rn(kq, x));
        out[1] = quantise8(__fmul_rn(kq, y));
        return;
    }
    float m0[BITS], m1[BITS];
#pragma unroll
    for (int b = 0; b < BITS; b++)
        m0[b] = m1[b] = INFINITY;
    bool done = false;
    if constexpr (BITS == 8) {
        if (p.ring) {
            done = true;
        /* ring constellations (demap.c:447-496): the metric of ring r, phase j
         * is c_j (-2 R_r) + R_r^2 with c_j = x rc_j + y rs_j; the phase bits
         * take the minimum over rings of each phase, the ring bits the metric
         * at the largest projection */
        float cmax = -INFINITY;
#pragma unroll
        for (int j = 0; j < 32; j++) {
            const float c = fmaf(x, p.rc[j], __fmul_rn(y, p.rs[j]));
            cmax = fmaxf(cmax, c);
            float a = fmaf(c, p.rm2[0], p.rr2[0]);
#pragma unroll
            for (int r = 1; r < 8; r++)
                a = fminf(a, fmaf(c, p.rm2[r], p.rr2[r]));
#pragma unroll
            for (int L = 0; L < 5; L++) {
                float& m = (j >> L) & 1 ? m1[BITS - 1 - L] : m0[BITS - 1 - L];
                m = fminf(m, a);
            }
        }
#pragma unroll
        for (int r = 0; r < 8; r++) {
            const float v = fmaf(cmax, p.rm2[r], p.rr2[r]);
#pragma unroll
            for (int L = 5; L < 8; L++) {
                float& m = (r >> (L - 5)) & 1 ? m1[BITS - 1 - L] : m0[BITS - 1 - L];
                m = fminf(m, v);
            }
        }
        }
    }
    if constexpr (BITS >= 6) {
        if (!done) {
        /* 64 to 256 points by groups of 16 (the minimum is order-free, so the
         * result is the full search's): the four low label bits from a tree
         * inside the group, the high bits from the groups' minima */
        float gmin[1 << (BITS - 4)];
#pragma unroll 1
        for (int g = 0; g < (1 << (BITS - 4)); g++) {
            float v[16];
#pragma unroll
            for (int q = 0; q < 16; q++) {
                const int pt = 16 * g + q;
                v[q] = fmaf(x, p.ar[pt], fmaf(y, p.ai[pt], p.e[pt]));
            }
            float t[16];
#pragma unroll
            for (int q = 0; q < 16; q++)
                t[q] = v[q];
#pragma unroll
            for (int L = 0, n = 16; L < 4; L++, n /= 2) {
                float lo = t[0], hi = t[1];
#pragma unroll
                for (int q = 2; q < n; q += 2) {
                    lo = fminf(lo, t[q]);
                    hi = fminf(hi, t[q + 1]);
                }
                m0[BITS - 1 - L] = fminf(m0[BITS - 1 - L], lo);
                m1[BITS - 1 - L] = fminf(m1[BITS - 1 - L], hi);
#pragma unroll
                for (int q = 0; q < n / 2; q++)
                    t[q] = fminf(t[2 * q], t[2 * q + 1]);
            }
            gmin[g] = t[0];
        }
#pragma unroll
        for (int L = 4; L < BITS; L++) {
            float lo = INFINITY, hi = INFINITY;
#pragma unroll
            for (int g = 0; g < (1 << (BITS - 4)); g++) {
                if ((g >> (L - 4)) & 1)
                    hi = fminf(hi, gmin[g]);
                else
                    lo = fminf(lo, gmin[g]);
            }
            m0[BITS - 1 - L] = lo;
            m1[BITS - 1 - L] = hi;
        }
        }
    } else {
#pragma unroll 8
        for (int q = 0; q < (1 << BITS); q++) {
            const float d = fmaf(x, p.ar[q], fmaf(y, p.ai[q], p.e[q]));
#pragma unroll
            for (int b = 0; b < BITS; b++) {
                if ((q >> (BITS - 1 - b)) & 1)
                    m1[b] = fminf(m1[b], d);
                else
                    m0[b] = fminf(m0[b], d);
            }
        }
    }
#pragma unroll
    for (int b = 0; b < BITS; b++)
        out[b] = quantise8(__fmul_rn(k, __fsub_rn(m1[b], m0[b])));
}

/* Codeword position of label bit b of symbol j: QPSK bits 2j, 2j + 1;
 * otherwise the bit interleaver's column order[b] */
template <int BITS>
__device__ __forceinline__ int llr_pos(const DemapParams& p, int b, int j)
{
    return BITS == 2 ? 2 * j + b : p.order[b] * p.nsym + j;
}

/* Grid rows walk the frames, threads take four consecutive symbols: two
 * 16-byte loads, and per label bit one 4-byte store (eight bytes for QPSK)
 * where the row layout allows it.  Every thread forms 2/n0 itself (one
 * broadcast load), so the warps of a block never wait for one another and
 * one warp's loads overlap another's arithmetic. */
template <int BITS>
__device__ __forceinline__ void demap_group(const DemapParams& p, const float4& a, const float4& c, int j0, float k,
                                            int8_t* __restrict__ llr)
{
    int8_t v[4][BITS];
    demap_symbol<BITS>(p, a.x, a.y, k, v[0]);
    demap_symbol<BITS>(p, a.z, a.w, k, v[1]);
    demap_symbol<BITS>(p, c.x, c.y, k, v[2]);
    demap_symbol<BITS>(p, c.z, c.w, k, v[3]);
    if (BITS == 2) {
        uint2 w;
        w.x = (uint32_t)(uint8_t)v[0][0] | (uint32_t)(uint8_t)v[0][1] << 8 | (uint32_t)(uint8_t)v[1][0] << 16 |
              (uint32_t)(uint8_t)v[1][1] << 24;
        w.y = (uint32_t)(uint8_t)v[2][0] | (uint32_t)(uint8_t)v[2][1] << 8 | (uint32_t)(uint8_t)v[3][0] << 16 |
              (uint32_t)(uint8_t)v[3][1] << 24;
        *(uint2*)(llr + 2 * (size_t)j0) = w;
    } else {
#pragma unroll
        for (int b = 0; b < BITS; b++) {
            const int pos = llr_pos<BITS>(p, b, j0);
            if (pos + 3 < p.nldpc)
                *(uint32_t*)(llr + pos) = (uint32_t)(uint8_t)v[0][b] | (uint32_t)(uint8_t)v[1][b] << 8 |
                                          (uint32_t)(uint8_t)v[2][b] << 16 | (uint32_t)(uint8_t)v[3][b] << 24;
            else
                for (int s = 0; s < 4; s++)
                    if (pos + s < p.nldpc)
                        llr[pos + s] = v[s][b];
        }
    }
}

/* Grid rows walk the frames, thread g of a row takes symbols 4g .. 4g + 3
 * of each of its frames (the launch covers every group of a frame): two
 * 16-byte loads, and per label bit one 4-byte store (eight bytes for QPSK)
 * where the row layout allows it.  The next frame's symbols are loaded
 * before this frame's arithmetic, and every thread forms 2/n0 itself (one
 * broadcast load), so loads stay in flight while the warps compute. */
template <int BITS>
__global__ void __launch_bounds__(256) k_demap(const __grid_constant__ DemapParams p)
{
    const int ngroups = (p.nsym + 3) / 4;
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= ngroups)
        return;
    const int j0 = 4 * g;
    auto vec_of = [&](int f) {
        const float* sym = p.sym + (size_t)f * p.sym_stride;
        const int8_t* llr = p.llr + (size_t)f * p.llr_stride;
        return ((uintptr_t)sym & 15) == 0 && ((uintptr_t)llr & 7) == 0 && (p.nsym & 3) == 0;
    };
    int f = blockIdx.y;
    if (f >= p.nframes)
        return;
    bool vec = vec_of(f);
    float4 a = make_float4(0.f, 0.f, 0.f, 0.f), c = a;
    if (vec) {
        const float* sym = p.sym + (size_t)f * p.sym_stride + 2 * (size_t)j0;
        a = __ldcs((const float4*)sym);
        c = __ldcs((const float4*)sym + 1);
    }
    for (; f < p.nframes; f += gridDim.y) {
        const int fn = f + gridDim.y;
        bool vecn = false;
        float4 an = make_float4(0.f, 0.f, 0.f, 0.f), cn = an;
        if (fn < p.nframes) {
            vecn = vec_of(fn);
            if (vecn) {
                const float* sym = p.sym + (size_t)fn * p.sym_stride + 2 * (size_t)j0;
                an = __ldcs((const float4*)sym);
                cn = __ldcs((const float4*)sym + 1);
            }
        }
        const float k = 2.0f / __ldg(p.n0 + f);
        int8_t* llr = p.llr + (size_t)f * p.llr_stride;
        if (vec) {
            demap_group<BITS>(p, a, c, j0, k, llr);
        } else {
            const float* sym = p.sym + (size_t)f * p.sym_stride;
            int8_t v[BITS];
            for (int s = 0; s < 4; s++) {
                const int j = j0 + s;
                if (j >= p.nsym)
                    break;
                demap_symbol<BITS>(p, sym[2 * (size_t)j], sym[2 * (size_t)j + 1], k, v);
#pragma unroll
                for (int b = 0; b < BITS; b++) {
                    const int pos = llr_pos<BITS>(p, b, j);
                    if (pos < p.nldpc)
                        llr[pos] = v[b];
                }
            }
        }
        a = an;
        c = cn;
        vec = vecn;
    }
}

}  // namespace drxg

using namespace drxg;

struct drx_demapper {
    int device = 0, sms = 0;
    DemapParams p{};
    cudaStream_t stream = nullptr;
    float* d_sym = nullptr;
    float* d_n0 = nullptr;
    int8_t* d_llr = nullptr;
};

namespace {

cudaError_t launch_demap(const DemapParams& p, int sms, cudaStream_t s)
{
    const int gx = (((p.nsym + 3) / 4) + 255) / 256;
    const int gy = std::max(1, std::min(p.nframes, std::max(1, 8 * sms / gx)));
    const dim3 grid(gx, std::min(gy, 65535));
    switch (p.qpsk ? 2 : p.bits) {
    case 2:
        k_demap<2><<<grid, 256, 0, s>>>(p);
        break;
    case 3:
        k_demap<3><<<grid, 256, 0, s>>>(p);
        break;
    case 4:
        k_demap<4><<<grid, 256, 0, s>>>(p);
        break;
    case 5:
        k_demap<5><<<grid, 256, 0, s>>>(p);
        break;
    case 6:
        k_demap<6><<<grid, 256, 0, s>>>(p);
        break;
    case 7:
        k_demap<7><<<grid, 256, 0, s>>>(p);
        break;
    case 8:
        k_demap<8><<<grid, 256, 0, s>>>(p);
        break;
    default:
        return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace

extern "C" {

drx_demapper* drx_demapper_new(const char* constellation, const char* rate, int short_frame)
{
    if (!constellation || !rate) {
        set_error("drx_demapper_new: NULL argument");
        return nullptr;
    }
    const cg_const* row = nullptr;
    for (size_t i = 0; i < sizeof(cg_consts) / sizeof(*cg_consts); i++)
        if (!strcmp(cg_consts[i].name, constellation) && !strcmp(cg_consts[i].rate, rate) &&
            cg_consts[i].short_frame == (short_frame ? 1 : 0))
            row = &cg_consts[i];
    if (!row || (row->order[0] >= 0 && (row->bits < 3 || row->bits > 8))) {
        set_error(std::string("drx_demapper_new: no DVB-S2/S2X constellation ") + constellation + " " + rate);
        return nullptr;
    }
    drx_demapper* m = new drx_demapper();
    DemapParams& p = m->p;
    p.bits = row->bits;
    p.qpsk = row->order[0] < 0;
    p.nldpc = short_frame ? 16200 : 64800;
    p.nsym = (p.nldpc + p.bits - 1) / p.bits;
    for (int b = 0; b < 8; b++)
        p.order[b] = row->order[b] < 0 ? 0 : row->order[b];
    const int np = 1 << row->bits;
    double e = 0;
    for (int i = 0; i < np; i++)
        e += (double)row->points[2 * i] * row->points[2 * i] + (double)row->points[2 * i + 1] * row->points[2 * i + 1];
    const float g = (float)(1.0 / sqrt(e / np));
    float pre[256], pim[256];
    for (int i = 0; i < np; i++) {
        const float re = row->points[2 * i] * g, im = row->points[2 * i + 1] * g;
        pre[i] = re;
        pim[i] = im;
        p.ar[i] = -2.0f * re;
        p.ai[i] = -2.0f * im;
        p.e[i] = fmaf(re, re, im * im);
    }
    /* 8 rings of the same 32 phases, the ring in the high label bits
     * (demap.c:136-162): ring radii, unit phase vectors, and the check that
     * every point is radius times phase */
    p.ring = 0;
    if (row->bits == 8) {
        for (int r = 0; r < 8; r++) {
            const float R = hypotf(pre[r << 5], pim[r << 5]);
            p.rm2[r] = -2.0f * R;
            p.rr2[r] = R * R;
        }
        const float R0 = hypotf(pre[0], pim[0]);
        for (int j = 0; j < 32; j++) {
            p.rc[j] = pre[j] / R0;
            p.rs[j] = pim[j] / R0;
        }
        bool ring = true;
        for (int i = 0; i < 256 && ring; i++) {
            const float R = -0.5f * p.rm2[i >> 5];
            ring = fabsf(R * p.rc[i & 31] - pre[i]) <= 1e-5f && fabsf(R * p.rs[i & 31] - pim[i]) <= 1e-5f;
        }
        p.ring = ring ? 1 : 0;
    }
    if (!cuda_check(cudaGetDevice(&m->device), "cudaGetDevice") ||
        !cuda_check(cudaDeviceGetAttribute(&m->sms, cudaDevAttrMultiProcessorCount, m->device), "attribute") ||
        !cuda_check(cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking), "cudaStreamCreate") ||
        !cuda_check(drxg::dev_malloc(&m->d_sym, sizeof(float) * 2 * (size_t)p.nsym), "cudaMalloc") ||
        !cuda_check(drxg::dev_malloc(&m->d_n0, sizeof(float)), "cudaMalloc") ||
        !cuda_check(drxg::dev_malloc(&m->d_llr, (size_t)p.nldpc), "cudaMalloc")) {
        drx_demapper_free(m);
        return nullptr;
    }
    return m;
}

void drx_demapper_free(drx_demapper* m)
{
    if (!m)
        return;
    if (m->stream)
        cudaStreamSynchronize(m->stream);
    cudaFree(m->d_sym);
    cudaFree(m->d_n0);
    cudaFree(m->d_llr);
    if (m->stream)
        cudaStreamDestroy(m->stream);
    delete m;
}

int drx_demapper_symbols(const drx_demapper* m) { return m ? m->p.nsym : -1; }

int drx_demapper_run(drx_demapper* m, const float* sym, size_t sym_stride, const float* n0, int8_t* llr,
                     size_t llr_stride, int nframes, void* stream)
{
    if (!m || (nframes > 0 && (!sym || !n0 || !llr))) {
        set_error("drx_demapper_run: NULL argument");
        return -1;
    }
    if (sym_stride < 2 * (size_t)m->p.nsym || llr_stride < (size_t)m->p.nldpc || (sym_stride & 1) ||
        ((uintptr_t)sym & 7)) {
        set_error("drx_demapper_run: strides below the frame size or unaligned symbols");
        return -1;
    }
    if (nframes <= 0)
        return 0;
    DemapParams p = m->p;
    p.sym = sym;
    p.sym_stride = sym_stride;
    p.n0 = n0;
    p.llr = llr;
    p.llr_stride = llr_stride;
    p.nframes = nframes;
    return cuda_check(launch_demap(p, m->sms, stream ? (cudaStream_t)stream : m->stream), "demapper launch") ? 0
                                                                                                                : -1;
}

int drx_demapper_frame(drx_demapper* m, const float* sym, float n0, int8_t* llr)
{
    if (!m || !sym || !llr) {
        set_error("drx_demapper_frame: NULL argument");
        return -1;
    }
    const size_t ns = 2 * (size_t)m->p.nsym;
    if (!cuda_check(cudaMemcpyAsync(m->d_sym, sym, sizeof(float) * ns, cudaMemcpyHostToDevice, m->stream),
                    "cudaMemcpyAsync") ||
        !cuda_check(cudaMemcpyAsync(m->d_n0, &n0, sizeof(float), cudaMemcpyHostToDevice, m->stream),
                    "cudaMemcpyAsync") ||
        drx_demapper_run(m, m->d_sym, ns, m->d_n0, m->d_llr, (size_t)m->p.nldpc, 1, m->stream) ||
        !cuda_check(cudaMemcpyAsync(llr, m->d_llr, (size_t)m->p.nldpc, cudaMemcpyDeviceToHost, m->stream),
                    "cudaMemcpyAsync") ||
        !cuda_check(cudaStreamSynchronize(m->stream), "demapper"))
        return -1;
    return 0;
}

}  // extern "C"
