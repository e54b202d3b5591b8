/*
 * BCH decoding of DVB-S2 BBFRAMEs on the GPU (EN 302 307-1 5.3.1), with the
 * reference's results (libdvbrx/src/bch.c:189-290, declared
 * libdvbrx/include/dvbrx/fec.h:27-37): the corrected codeword in place and
 * the number of corrected bits, or -1 with the word untouched.
 *
 * The code: g(x) = product of the minimal polynomials of alpha^(2i+1),
 * i < t, over GF(2^16) (normal frames, primitive x^16+x^5+x^3+x^2+1) or
 * GF(2^14) (short frames, x^14+x^5+x^3+x+1); W = deg g = 16 t or 14 t parity
 * bits; codewords of nbch = kldpc bits, MSB first, the highest degree first.
 *
 * k_bch_remainder: one thread per frame divides c(x) x^W by g(x), four
 * message bytes per step through four 256-entry tables (slicing by four,
 * tables in shared memory; the remainder register is 192 bits, x^(W-1) at
 * the top).  A zero remainder ends the frame (no error).  Otherwise the
 * thread forms the syndromes S_j = R(alpha^j) alpha^(-jW) (odd j; even ones
 * by squaring), runs Berlekamp-Massey, and queues the frame for the Chien
 * search if the locator degree is at most t.
 * k_bch_chien: one CTA per queued frame evaluates the locator at every
 * position of the shortened code; when the roots number the degree, their
 * bits are flipped.  For a correctable word the locator is unique, so the
 * result does not depend on how it was found.
 */
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <string>
#include <vector>

#include "../../include/dvbrx_b200.h"
#include "handle.h"

namespace drxg {

constexpr int kBchMaxT = 12;
constexpr int kBchWords = 3; /* 192-bit remainder register */
constexpr int kBchThreads = 64;
constexpr int kChienThreads = 512;

struct BchDev {
    int m, q, t, W, nbch;
    const unsigned long long* tab; /* [4][256][3] */
    const uint16_t* exp;           /* 2q */
    const uint16_t* log;           /* q + 1 */
};

struct BchBatch {
    BchDev c;
    uint8_t* cw;
    size_t stride;
    int32_t* result;
    int nframes;
    uint16_t* loc;   /* per frame: 16 locator coefficients */
    int32_t* queue;  /* frames for the Chien search */
    int* count;      /* queue length */
};

__device__ __forceinline__ uint16_t gmul(const BchDev& c, uint16_t a, uint16_t b)
{
    if (!a || !b)
        return 0;
    return __ldg(c.exp + __ldg(c.log + a) + __ldg(c.log + b));
}

__device__ __forceinline__ uint16_t gpow(const BchDev& c, long long e)
{
    e %= c.q;
    if (e < 0)
        e += c.q;
    return __ldg(c.exp + e);
}

__global__ void __launch_bounds__(kBchThreads) k_bch_remainder(BchBatch b)
{
    __shared__ unsigned long long tab[4 * 256 * kBchWords];
    for (int k = threadIdx.x; k < 4 * 256 * kBchWords; k += blockDim.x)
        tab[k] = b.c.tab[k];
    __syncthreads();
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= b.nframes)
        return;
    const BchDev& c = b.c;
    const uint8_t* w = b.cw + (size_t)f * b.stride;
    unsigned long long r0 = 0, r1 = 0, r2 = 0;
    const int nbytes = c.nbch / 8;
    int i = 0;
    for (; i + 4 <= nbytes; i += 4) {
        const uint32_t top = (uint32_t)(r0 >> 32) ^ ((uint32_t)w[i] << 24 | (uint32_t)w[i + 1] << 16 |
                                                     (uint32_t)w[i + 2] << 8 | (uint32_t)w[i + 3]);
        const unsigned long long* t3 = tab + (3 * 256 + (top >> 24)) * kBchWords;
        const unsigned long long* t2 = tab + (2 * 256 + ((top >> 16) & 255)) * kBchWords;
        const unsigned long long* t1 = tab + (1 * 256 + ((top >> 8) & 255)) * kBchWords;
        const unsigned long long* t0 = tab + (top & 255) * kBchWords;
        r0 = (r0 << 32 | r1 >> 32) ^ t3[0] ^ t2[0] ^ t1[0] ^ t0[0];
        r1 = (r1 << 32 | r2 >> 32) ^ t3[1] ^ t2[1] ^ t1[1] ^ t0[1];
        r2 = (r2 << 32) ^ t3[2] ^ t2[2] ^ t1[2] ^ t0[2];
    }
    for (; i < nbytes; i++) {
        const unsigned long long* t0 = tab + ((uint32_t)(r0 >> 56) ^ w[i]) * kBchWords;
        r0 = (r0 << 8 | r1 >> 56) ^ t0[0];
        r1 = (r1 << 8 | r2 >> 56) ^ t0[1];
        r2 = (r2 << 8) ^ t0[2];
    }
    if (!(r0 | r1 | r2)) {
        b.result[f] = 0;
        return;
    }
    /* syndromes: coefficient of x^k of the remainder at register bit 192 - W + k */
    const int t2n = 2 * c.t;
    uint16_t S[2 * kBchMaxT + 1];
    for (int j = 1; j <= t2n; j += 2) {
        uint16_t s = 0;
        for (int k = 0; k < c.W; k++) {
            const int bit = 192 - c.W + k; /* 0 = least significant of r2 */
            const unsigned long long word = bit < 64 ? r2 : bit < 128 ? r1 : r0;
            if ((word >> (bit & 63)) & 1ull)
                s ^= gpow(c, (long long)j * k);
        }
        S[j] = gmul(c, s, gpow(c, -(long long)j * c.W));
    }
    for (int j = 2; j <= t2n; j += 2)
        S[j] = gmul(c, S[j / 2], S[j / 2]);
    /* Berlekamp-Massey: the shortest LFSR L(x) generating S_1 .. S_2t */
    /* the running length can pass t + 1 on uncorrectable words: the arrays
     * hold 2t + 2 coefficients (updates stop at degree t + 1, as in bch.c) */
    uint16_t L[2 * kBchMaxT + 2] = { 1 }, B[2 * kBchMaxT + 2] = { 1 }, T[2 * kBchMaxT + 2];
    int len = 0, shift = 1;
    uint16_t bdisc = 1;
    for (int n = 0; n < t2n; n++) {
        uint16_t d = S[n + 1];
        for (int k = 1; k <= len; k++)
            d ^= gmul(c, L[k], S[n + 1 - k]);
        if (!d) {
            shift++;
            continue;
        }
        const uint16_t coef = gmul(c, d, __ldg(c.exp + c.q - __ldg(c.log + bdisc)));
        for (int k = 0; k < 2 * kBchMaxT + 2; k++)
            T[k] = L[k];
        for (int k = 0; k + shift <= c.t + 1; k++)
            L[k + shift] ^= gmul(c, coef, B[k]);
        if (2 * len <= n) {
            len = n + 1 - len;
            for (int k = 0; k < 2 * kBchMaxT + 2; k++)
                B[k] = T[k];
            bdisc = d;
            shift = 1;
        } else {
            shift++;
        }
    }
    if (len > c.t) {
        b.result[f] = -1;
        return;
    }
    uint16_t* loc = b.loc + (size_t)f * 16;
    for (int k = 0; k < 16; k++)
        loc[k] = k <= len ? L[k] : 0;
    b.result[f] = 1000 + len; /* pending: the Chien search sets the result */
    b.queue[atomicAdd(b.count, 1)] = f;
}

/* Systematic encoding in place: the kbch message bits of each row are
 * followed by the W parity bits of m(x) x^W mod g(x), highest degree first
 * (the remainder of the same table division over the message bytes). */
__global__ void __launch_bounds__(kBchThreads) k_bch_encode(BchBatch b, int kbytes)
{
    __shared__ unsigned long long tab[4 * 256 * kBchWords];
    for (int k = threadIdx.x; k < 4 * 256 * kBchWords; k += blockDim.x)
        tab[k] = b.c.tab[k];
    __syncthreads();
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= b.nframes)
        return;
    uint8_t* w = b.cw + (size_t)f * b.stride;
    unsigned long long r0 = 0, r1 = 0, r2 = 0;
    for (int i = 0; i < kbytes; i++) {
        const unsigned long long* t0 = tab + ((uint32_t)(r0 >> 56) ^ w[i]) * kBchWords;
        r0 = (r0 << 8 | r1 >> 56) ^ t0[0];
        r1 = (r1 << 8 | r2 >> 56) ^ t0[1];
        r2 = (r2 << 8) ^ t0[2];
    }
    const unsigned long long r[3] = { r0, r1, r2 };
    for (int k = 0; k < b.c.W / 8; k++)
        w[kbytes + k] = (uint8_t)(r[k / 8] >> (56 - 8 * (k % 8)));
}

__global__ void __launch_bounds__(kChienThreads) k_bch_chien(BchBatch b)
{
    __shared__ int s_roots, s_pos[kBchMaxT + 1];
    __shared__ int s_lg[kBchMaxT + 1], s_step[kBchMaxT + 1], s_nt;
    __shared__ uint16_t s_l0;
    const BchDev& c = b.c;
    const int n = *b.count;
    for (int qi = blockIdx.x; qi < n; qi += gridDim.x) {
        const int f = b.queue[qi];
        const uint16_t* loc = b.loc + (size_t)f * 16;
        const int len = b.result[f] - 1000;
        if (threadIdx.x == 0) {
            int nt = 0;
            for (int k = 1; k <= len; k++)
                if (loc[k]) {
                    s_lg[nt] = __ldg(c.log + loc[k]);
                    s_step[nt++] = c.q - k % c.q;
                }
            s_nt = nt;
            s_l0 = loc[0];
            s_roots = 0;
        }
        __syncthreads();
        const int nt = s_nt;
        for (int p = threadIdx.x; p < c.nbch; p += blockDim.x) {
            uint16_t sum = s_l0;
            for (int k = 0; k < nt; k++)
                sum ^= __ldg(c.exp + (unsigned)(((unsigned long long)s_lg[k] + (unsigned long long)s_step[k] * p) %
                                                (unsigned)c.q));
            if (!sum) {
                const int r = atomicAdd(&s_roots, 1);
                if (r <= kBchMaxT)
                    s_pos[r] = p;
            }
        }
        __syncthreads();
        const int roots = s_roots;
        if (threadIdx.x == 0) {
            if (roots == len) { /* distinct positions: one thread flips them */
                uint8_t* w = b.cw + (size_t)f * b.stride;
                for (int k = 0; k < roots; k++) {
                    const int bit = c.nbch - 1 - s_pos[k];
                    w[bit / 8] ^= (uint8_t)(0x80u >> (bit % 8));
                }
                b.result[f] = len;
            } else {
                b.result[f] = -1;
            }
        }
        __syncthreads();
    }
}

}  // namespace drxg

using namespace drxg;

struct drx_bch {
    int device = 0;
    int sms = 0;
    int short_frame = 0, m = 0, q = 0, t = 0, kbch = 0, nbch = 0, W = 0;
    void* blob = nullptr;
    BchDev dev{};
    cudaStream_t stream = nullptr;
    uint16_t* loc = nullptr;
    int32_t* queue = nullptr;
    int* count = nullptr;
    size_t cap = 0;
    uint8_t* d_cw = nullptr;
    int32_t* d_res = nullptr;
};

namespace {

bool bch_tables(drx_bch* b, std::vector<unsigned long long>& tab, std::vector<uint16_t>& ex, std::vector<uint16_t>& lg)
{
    const int m = b->m, q = b->q;
    const unsigned prim = b->short_frame ? 0x402Bu : 0x1002Du;
    ex.assign(2 * (size_t)q, 0);
    lg.assign((size_t)q + 1, 0);
    unsigned x = 1;
    for (int i = 0; i < q; i++) {
        ex[i] = ex[i + q] = (uint16_t)x;
        lg[x] = (uint16_t)i;
        x <<= 1;
        if (x >> m)
            x ^= prim;
    }
    auto mul = [&](uint16_t a, uint16_t c) -> uint16_t { return a && c ? ex[lg[a] + lg[c]] : 0; };
    /* g(x): product of the minimal polynomials of alpha^i, i = 1, 3, .., 2t-1 */
    std::vector<uint8_t> g(1, 1);
    for (int i = 1; i < 2 * b->t; i += 2) {
        std::vector<uint16_t> p(1, 1);
        int e = i % q;
        do {
            const uint16_t beta = ex[e];
            p.push_back(0);
            for (size_t k = p.size() - 1; k > 0; k--)
                p[k] = p[k - 1] ^ mul(p[k], beta);
            p[0] = mul(p[0], beta);
            e = (2 * e) % q;
        } while (e != i % q);
        std::vector<uint8_t> r(g.size() + p.size() - 1, 0);
        for (size_t a = 0; a < g.size(); a++)
            if (g[a])
                for (size_t c = 0; c < p.size(); c++)
                    r[a + c] ^= (uint8_t)(p[c] & 1);
        g = r;
    }
    b->W = (int)g.size() - 1;
    if (b->W > 64 * kBchWords || b->W != b->nbch - b->kbch)
        return false;
    /* T0[v]: (v(x) x^W) mod g(x) for a byte v (v's MSB = highest degree),
     * left-aligned: x^(W-1) at register bit 191; Ts[v] = T(s-1)[v] x^8 mod g */
    tab.assign(4 * 256 * kBchWords, 0);
    const int W = b->W;
    auto setbit = [&](unsigned long long* r, int bitpos) { /* bitpos 191 = MSB of r[0] */
        r[2 - bitpos / 64] ^= 1ull << (bitpos % 64);
    };
    for (int v = 0; v < 256; v++) {
        unsigned long long r[3] = { 0, 0, 0 };
        for (int bit = 7; bit >= 0; bit--) {
            const int top = (int)(r[0] >> 63) ^ ((v >> bit) & 1);
            r[0] = r[0] << 1 | r[1] >> 63;
            r[1] = r[1] << 1 | r[2] >> 63;
            r[2] <<= 1;
            if (top)
                for (int k = 0; k < W; k++)
                    if (g[k])
                        setbit(r, 192 - W + k);
        }
        for (int w = 0; w < 3; w++)
            tab[(size_t)v * 3 + w] = r[w];
    }
    for (int s = 1; s < 4; s++)
        for (int v = 0; v < 256; v++) {
            unsigned long long r[3];
            for (int w = 0; w < 3; w++)
                r[w] = tab[((size_t)(s - 1) * 256 + v) * 3 + w];
            const unsigned long long* t0 = &tab[(size_t)(r[0] >> 56) * 3];
            const unsigned long long n0 = (r[0] << 8 | r[1] >> 56) ^ t0[0];
            const unsigned long long n1 = (r[1] << 8 | r[2] >> 56) ^ t0[1];
            const unsigned long long n2 = (r[2] << 8) ^ t0[2];
            tab[((size_t)s * 256 + v) * 3 + 0] = n0;
            tab[((size_t)s * 256 + v) * 3 + 1] = n1;
            tab[((size_t)s * 256 + v) * 3 + 2] = n2;
        }
    return true;
}

bool bch_scratch(drx_bch* b, size_t n)
{
    if (b->cap >= n)
        return true;
    cudaStreamSynchronize(b->stream);
    cudaFree(b->loc);
    cudaFree(b->queue);
    b->loc = nullptr;
    b->queue = nullptr;
    b->cap = 0;
    if (!cuda_check(drxg::dev_malloc(&b->loc, n * 16 * sizeof(uint16_t)), "cudaMalloc(bch)") ||
        !cuda_check(drxg::dev_malloc(&b->queue, n * sizeof(int32_t)), "cudaMalloc(bch)"))
        return false;
    b->cap = n;
    return true;
}

int bch_enqueue(drx_bch* b, uint8_t* cw, size_t stride, int32_t* result, int nframes, cudaStream_t s)
{
    if (nframes <= 0)
        return 0;
    if (!cw || !result || stride < (size_t)(b->nbch / 8)) {
        set_error("drx_bch_decode_device: bad arguments");
        return -1;
    }
    if (!bch_scratch(b, (size_t)nframes))
        return -1;
    BchBatch p{};
    p.c = b->dev;
    p.cw = cw;
    p.stride = stride;
    p.result = result;
    p.nframes = nframes;
    p.loc = b->loc;
    p.queue = b->queue;
    p.count = b->count;
    if (!cuda_check(cudaMemsetAsync(b->count, 0, sizeof(int), s), "cudaMemsetAsync"))
        return -1;
    k_bch_remainder<<<(nframes + kBchThreads - 1) / kBchThreads, kBchThreads, 0, s>>>(p);
    if (!cuda_check(cudaGetLastError(), "BCH remainder"))
        return -1;
    k_bch_chien<<<std::min(nframes, 4 * b->sms), kChienThreads, 0, s>>>(p);
    return cuda_check(cudaGetLastError(), "BCH Chien search") ? 0 : -1;
}

}  // namespace

extern "C" {

drx_bch* drx_bch_new(const drx_fec_params* p)
{
    if (!p || p->t < 1 || p->t > kBchMaxT || p->kldpc <= p->kbch || p->kldpc % 8) {
        set_error("drx_bch_new: not a DVB-S2 BCH code");
        return nullptr;
    }
    drx_bch* b = new drx_bch();
    b->short_frame = p->short_frame ? 1 : 0;
    b->m = b->short_frame ? 14 : 16;
    b->q = (1 << b->m) - 1;
    b->t = p->t;
    b->kbch = p->kbch;
    b->nbch = p->kldpc;
    std::vector<unsigned long long> tab;
    std::vector<uint16_t> ex, lg;
    if (!bch_tables(b, tab, ex, lg)) {
        set_error("drx_bch_new: parity length does not match the code");
        delete b;
        return nullptr;
    }
    bool ok = cuda_check(cudaGetDevice(&b->device), "cudaGetDevice") &&
              cuda_check(cudaDeviceGetAttribute(&b->sms, cudaDevAttrMultiProcessorCount, b->device), "attribute") &&
              cuda_check(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    const size_t o_ex = tab.size() * 8, o_lg = o_ex + ex.size() * 2, total = o_lg + lg.size() * 2 + 64;
    ok = ok && cuda_check(drxg::dev_malloc(&b->blob, total), "cudaMalloc(bch tables)") &&
         cuda_check(drxg::dev_malloc(&b->count, sizeof(int)), "cudaMalloc") &&
         cuda_check(drxg::dev_malloc(&b->d_cw, (size_t)b->nbch / 8), "cudaMalloc") &&
         cuda_check(drxg::dev_malloc(&b->d_res, sizeof(int32_t)), "cudaMalloc");
    if (ok) {
        char* base = (char*)b->blob;
        ok = cuda_check(cudaMemcpy(base, tab.data(), o_ex, cudaMemcpyHostToDevice), "cudaMemcpy") &&
             cuda_check(cudaMemcpy(base + o_ex, ex.data(), ex.size() * 2, cudaMemcpyHostToDevice), "cudaMemcpy") &&
             cuda_check(cudaMemcpy(base + o_lg, lg.data(), lg.size() * 2, cudaMemcpyHostToDevice), "cudaMemcpy");
        b->dev.m = b->m;
        b->dev.q = b->q;
        b->dev.t = b->t;
        b->dev.W = b->W;
        b->dev.nbch = b->nbch;
        b->dev.tab = (const unsigned long long*)base;
        b->dev.exp = (const uint16_t*)(base + o_ex);
        b->dev.log = (const uint16_t*)(base + o_lg);
    }
    if (!ok) {
        drx_bch_free(b);
        return nullptr;
    }
    return b;
}

void drx_bch_free(drx_bch* b)
{
    if (!b)
        return;
    if (b->stream)
        cudaStreamSynchronize(b->stream);
    cudaFree(b->blob);
    cudaFree(b->loc);
    cudaFree(b->queue);
    cudaFree(b->count);
    cudaFree(b->d_cw);
    cudaFree(b->d_res);
    if (b->stream)
        cudaStreamDestroy(b->stream);
    delete b;
}

int drx_bch_decode_device(drx_bch* b, uint8_t* cw, size_t stride, int32_t* result, int nframes, void* stream)
{
    if (!b) {
        set_error("drx_bch_decode_device: NULL handle");
        return -1;
    }
    return bch_enqueue(b, cw, stride, result, nframes, stream ? (cudaStream_t)stream : b->stream);
}

int drx_bch_encode_device(drx_bch* b, uint8_t* cw, size_t stride, int nframes, void* stream)
{
    if (!b || (nframes > 0 && !cw) || stride < (size_t)(b->nbch / 8) || b->kbch % 8) {
        set_error("drx_bch_encode_device: bad arguments");
        return -1;
    }
    if (nframes <= 0)
        return 0;
    BchBatch p{};
    p.c = b->dev;
    p.cw = cw;
    p.stride = stride;
    p.nframes = nframes;
    k_bch_encode<<<(nframes + kBchThreads - 1) / kBchThreads, kBchThreads, 0,
                   stream ? (cudaStream_t)stream : b->stream>>>(p, b->kbch / 8);
    return cuda_check(cudaGetLastError(), "BCH encode") ? 0 : -1;
}

int drx_bch_decode(drx_bch* b, uint8_t* cw)
{
    if (!b || !cw) {
        set_error("drx_bch_decode: NULL argument");
        return -1;
    }
    const size_t nb = (size_t)b->nbch / 8;
    int32_t res = -1;
    if (!cuda_check(cudaMemcpyAsync(b->d_cw, cw, nb, cudaMemcpyHostToDevice, b->stream), "cudaMemcpyAsync") ||
        bch_enqueue(b, b->d_cw, nb, b->d_res, 1, b->stream) ||
        !cuda_check(cudaMemcpyAsync(&res, b->d_res, sizeof(int32_t), cudaMemcpyDeviceToHost, b->stream),
                    "cudaMemcpyAsync") ||
        !cuda_check(cudaStreamSynchronize(b->stream), "BCH decode"))
        return -1;
    if (res > 0 &&
        !cuda_check(cudaMemcpy(cw, b->d_cw, nb, cudaMemcpyDeviceToHost), "cudaMemcpy"))
        return -1;
    return res;
}

}  // extern "C"
