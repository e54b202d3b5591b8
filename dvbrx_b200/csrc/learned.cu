/*
 * Learned (neural offset / scaled) min-sum: training kernels.
 *
 * The decoder is the plain layered decoder's schedule (layers in order,
 * wavefront steps inside levelled layers) with the check node's offset 1
 * replaced by a learned scale and offset per iteration t and check-degree
 * class k:
 *
 *     x_c   = clamp(P_v - m_c, -128, 127)            extrinsic input
 *     mu_c  = min(min_{c' != c} |x_c'|, 127)
 *     mag_c = max(beta[t][k] * mu_c - alpha[t][k], 0)
 *     m'_c  = sign_{c' != c}(x) * mag_c               (sign of 0 is +)
 *     P'_v  = clamp(x_c + m'_c, -128, 127)            posterior
 *     m_c  <- clamp(m'_c, -32, 31)                    stored message
 *
 * on the int8 decoder's scale (2 x LLR), with the same saturations as the
 * int8 decoder, in fp32.  The plain decoder is beta = 1, alpha = 1 (with
 * rounding).  The loss is the binary cross-entropy of the information bits
 * after every iteration: sum_t sum_v softplus(-(1 - 2 b_v) P_v / 2).
 *
 * Forward (k_learned_fwd): one CTA per frame, state in global memory
 * (posteriors N floats, messages slots x DS floats, edge-major), and, when
 * training, a checkpoint of (P, m) at the start of every iteration.
 *
 * Backward (k_learned_bwd): for t = T-1 .. 0 it restores the iteration-t
 * checkpoint, re-runs iteration t saving every extrinsic input x (one float
 * per link), adds the iteration's loss gradient, then walks the steps in
 * reverse: the gradient of a check node's outputs goes to its inputs through
 * the straight path (P' = x + m'), the scale and offset, and the minimum
 * (the argmin link receives d mag / d mu; the sign is piecewise constant);
 * saturated clamps pass no gradient.  Memory is bounded by one checkpoint
 * per iteration instead of every intermediate.
 */
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "learned.h"

namespace drxg {

constexpr int kLT = 384;
constexpr int kQCl = 360;

__device__ __forceinline__ float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }
__device__ __forceinline__ float softplus(float u) { return fmaxf(u, 0.0f) + log1pf(expf(-fabsf(u))); }
__device__ __forceinline__ float sigmoid(float u) { return 1.0f / (1.0f + expf(-u)); }

struct LFrame {
    float* P;  /* N */
    float* M;  /* DS * R, edge-major: link c of slot s at c * R + s */
    float* X;  /* same layout, extrinsic inputs of the current iteration */
    float* gP; /* N */
    float* gM; /* DS * R */
};

__device__ __forceinline__ LFrame frame_state(const LearnedParams& p, int f)
{
    const DevCode& c = *p.code;
    const size_t E = (size_t)p.DS * c.R;
    LFrame s;
    s.P = p.P + (size_t)f * c.N;
    s.M = p.M + (size_t)f * E;
    s.X = p.X ? p.X + (size_t)f * E : nullptr;
    s.gP = p.gP ? p.gP + (size_t)f * c.N : nullptr;
    s.gM = p.gM ? p.gM + (size_t)f * E : nullptr;
    return s;
}

/* Links of check (i, j) at step position pos: slot 0 = parity, slot 1 =
 * previous parity (absent for (0, 0)), 2.. = information bits. */
__device__ __forceinline__ int link_var(const DevCode& c, int i, int j, int slot)
{
    if (slot == 0)
        return c.K + kQCl * i + j;
    if (slot == 1)
        return i ? c.K + kQCl * (i - 1) + j : c.K + kQCl * (c.q - 1) + j - 1;
    const int2 e = c.ent[c.eoff[i] + slot - 2];
    return e.x + j + (j < e.y ? kQCl : 0);
}

/* Forward of one check; X saved when non-null. */
__device__ void check_fwd(const DevCode& c, const LFrame& s, int i, int j, int slotpos, float beta, float alpha,
                          bool first)
{
    const int cnt = c.eoff[i + 1] - c.eoff[i];
    const int D = cnt + 2;
    const bool has_pp = (i | j) != 0;
    float x[kLearnedMaxDeg];
    int var[kLearnedMaxDeg];
    float min0 = 1e30f, min1 = 1e30f;
    int a0 = -1;
    int neg = 0;
    for (int k = 0; k < D; k++) {
        if (k == 1 && !has_pp)
            continue;
        var[k] = link_var(c, i, j, k);
        const size_t e = (size_t)k * c.R + slotpos;
        const float raw = s.P[var[k]] - (first ? 0.0f : s.M[e]);
        if (s.X)
            s.X[e] = raw;
        const float xv = clampf(raw, -128.0f, 127.0f);
        x[k] = xv;
        const float a = fabsf(xv);
        if (a < min0) {
            min1 = min0;
            min0 = a;
            a0 = k;
        } else if (a < min1) {
            min1 = a;
        }
        neg ^= xv < 0.0f;
    }
    for (int k = 0; k < D; k++) {
        if (k == 1 && !has_pp)
            continue;
        const float mu = fminf(k == a0 ? min1 : min0, 127.0f);
        const float mag = fmaxf(beta * mu - alpha, 0.0f);
        const bool sneg = neg ^ (x[k] < 0.0f);
        const float m = sneg ? -mag : mag;
        s.P[var[k]] = clampf(x[k] + m, -128.0f, 127.0f);
        s.M[(size_t)k * c.R + slotpos] = clampf(m, -32.0f, 31.0f);
    }
}

/* Backward of one check from its saved extrinsic inputs: reads the
 * gradients of its outputs (gP at its links, gM of its messages), writes
 * those of its inputs in their place, accumulates the parameter gradients. */
__device__ void check_bwd(const DevCode& c, const LFrame& s, int i, int j, int slotpos, float beta, float alpha,
                          bool first, float& dbeta, float& dalpha)
{
    const int cnt = c.eoff[i + 1] - c.eoff[i];
    const int D = cnt + 2;
    const bool has_pp = (i | j) != 0;
    float raw[kLearnedMaxDeg], x[kLearnedMaxDeg], gx[kLearnedMaxDeg];
    int var[kLearnedMaxDeg];
    float min0 = 1e30f, min1 = 1e30f;
    int a0 = -1, a1 = -1;
    int neg = 0;
    for (int k = 0; k < D; k++) {
        if (k == 1 && !has_pp)
            continue;
        var[k] = link_var(c, i, j, k);
        raw[k] = s.X[(size_t)k * c.R + slotpos];
        const float xv = clampf(raw[k], -128.0f, 127.0f);
        x[k] = xv;
        gx[k] = 0.0f;
        const float a = fabsf(xv);
        if (a < min0) {
            min1 = min0;
            a1 = a0;
            min0 = a;
            a0 = k;
        } else if (a < min1) {
            min1 = a;
            a1 = k;
        }
        neg ^= xv < 0.0f;
    }
    for (int k = 0; k < D; k++) {
        if (k == 1 && !has_pp)
            continue;
        const float muraw = k == a0 ? min1 : min0;
        const float mu = fminf(muraw, 127.0f);
        const float pre = beta * mu - alpha;
        const float mag = fmaxf(pre, 0.0f);
        const bool sneg = neg ^ (x[k] < 0.0f);
        const float sg = sneg ? -1.0f : 1.0f;
        const float m = sg * mag;
        const size_t e = (size_t)k * c.R + slotpos;
        const float gpo = s.gP[var[k]];       /* d L / d P' */
        const float gmo = s.gM ? s.gM[e] : 0; /* d L / d stored message */
        const float post = x[k] + m;
        const float gpost = (post >= -128.0f && post <= 127.0f) ? gpo : 0.0f;
        const float gmsg = (m >= -32.0f && m <= 31.0f) ? gmo : 0.0f;
        const float gm = gpost + gmsg;
        gx[k] += gpost;
        if (pre > 0.0f) {
            const float gmag = gm * sg;
            dbeta += gmag * mu;
            dalpha -= gmag;
            if (muraw < 127.0f) {
                const int src = k == a0 ? a1 : a0;
                gx[src] += gmag * beta * (x[src] < 0.0f ? -1.0f : 1.0f);
            }
        }
    }
    for (int k = 0; k < D; k++) {
        if (k == 1 && !has_pp)
            continue;
        const bool inside = raw[k] >= -128.0f && raw[k] <= 127.0f;
        const float g = inside ? gx[k] : 0.0f;
        s.gP[var[k]] = g;
        if (s.gM)
            s.gM[(size_t)k * c.R + slotpos] = first ? 0.0f : -g;
    }
}

/* One iteration (all steps), forward. */
__device__ void iteration_fwd(const DevCode& c, const LFrame& s, const LearnedParams& p, int t,
                              const float* sbeta, const float* salpha)
{
    const int tid = threadIdx.x;
    for (int st_i = 0; st_i < c.nsteps; st_i++) {
        const uint32_t st = c.steps[st_i];
        const int i = st & 0xFF, start = (st >> 8) & 0x1FF, n = (st >> 17) & 0x1FF;
        for (int g = tid; g < n; g += blockDim.x) {
            const int pos = start + g;
            const int j = (st >> 26) ? (int)c.perm[kQCl * i + pos] : pos;
            const int D = c.eoff[i + 1] - c.eoff[i] + 2 - ((i | j) ? 0 : 1);
            const int k = p.cls[D];
            check_fwd(c, s, i, j, kQCl * i + pos, sbeta[k], salpha[k], t == 0);
        }
        __syncthreads();
    }
}

/* Loss of the posteriors after iteration t; optionally its gradient into gP. */
__device__ float iteration_loss(const DevCode& c, const LFrame& s, const LearnedParams& p, int f, float gscale)
{
    const uint8_t* bits = p.bits + (size_t)f * p.bits_stride;
    float acc = 0.0f;
    for (int v = threadIdx.x; v < c.kldpc; v += blockDim.x) {
        const float sb = ((bits[v >> 3] >> (7 - (v & 7))) & 1) ? -1.0f : 1.0f; /* +1 for a 0 bit */
        const float u = -sb * s.P[v] * 0.5f;
        acc += softplus(u);
        if (gscale != 0.0f)
            s.gP[v] += gscale * (-sb * 0.5f) * sigmoid(u);
    }
    return acc;
}

__device__ float block_sum(float v, float* red)
{
    for (int o = 16; o > 0; o >>= 1)
        v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
    if ((threadIdx.x & 31) == 0)
        red[threadIdx.x >> 5] = v;
    __syncthreads();
    float r = 0.0f;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); w++)
            r += red[w];
    __syncthreads();
    return r;
}

__device__ void load_params(const LearnedParams& p, int t, float* sbeta, float* salpha)
{
    if ((int)threadIdx.x < p.nclass) {
        sbeta[threadIdx.x] = __half2float(p.beta[t * p.nclass + threadIdx.x]);
        salpha[threadIdx.x] = __half2float(p.alpha[t * p.nclass + threadIdx.x]);
    }
    __syncthreads();
}

__global__ void __launch_bounds__(kLT) k_learned_fwd(LearnedParams p)
{
    __shared__ float sbeta[kLearnedMaxClass], salpha[kLearnedMaxClass], red[kLT / 32];
    const DevCode& c = *p.code;
    const int f = blockIdx.x;
    const LFrame s = frame_state(p, f);
    const size_t E = (size_t)p.DS * c.R;
    const __half* src = p.llr + (size_t)f * p.llr_stride;
    for (int v = threadIdx.x; v < c.K; v += blockDim.x)
        s.P[v] = clampf(__half2float(src[v]), -128.0f, 127.0f);
    for (int k = threadIdx.x; k < c.R; k += blockDim.x)
        s.P[c.K + kQCl * (k % c.q) + k / c.q] = clampf(__half2float(src[c.K + k]), -128.0f, 127.0f);
    __syncthreads();
    for (int t = 0; t < p.iters; t++) {
        if (p.Pck) {
            float* pc = p.Pck + ((size_t)t * p.nframes + f) * c.N;
            float* mc = p.Mck + ((size_t)t * p.nframes + f) * E;
            for (int v = threadIdx.x; v < c.N; v += blockDim.x)
                pc[v] = s.P[v];
            if (t > 0)
                for (size_t e = threadIdx.x; e < E; e += blockDim.x)
                    mc[e] = s.M[e];
        }
        load_params(p, t, sbeta, salpha);
        LFrame sf = s;
        sf.X = nullptr;
        iteration_fwd(c, sf, p, t, sbeta, salpha);
        const float l = block_sum(iteration_loss(c, s, p, f, 0.0f), red);
        if (threadIdx.x == 0)
            atomicAdd(p.loss + t, l);
    }
    if (p.post)
        for (int v = threadIdx.x; v < c.kldpc; v += blockDim.x)
            p.post[(size_t)f * c.kldpc + v] = s.P[v];
}

__global__ void __launch_bounds__(kLT) k_learned_bwd(LearnedParams p)
{
    __shared__ float sbeta[kLearnedMaxClass], salpha[kLearnedMaxClass], red[kLT / 32];
    __shared__ float sdb[kLearnedMaxClass], sda[kLearnedMaxClass];
    const DevCode& c = *p.code;
    const int f = blockIdx.x;
    const LFrame s = frame_state(p, f);
    const size_t E = (size_t)p.DS * c.R;
    for (int v = threadIdx.x; v < c.N; v += blockDim.x)
        s.gP[v] = 0.0f;
    for (size_t e = threadIdx.x; e < E; e += blockDim.x)
        s.gM[e] = 0.0f;
    __syncthreads();
    for (int t = p.iters - 1; t >= 0; t--) {
        /* restore the state at the start of iteration t */
        const float* pc = p.Pck + ((size_t)t * p.nframes + f) * c.N;
        const float* mc = p.Mck + ((size_t)t * p.nframes + f) * E;
        for (int v = threadIdx.x; v < c.N; v += blockDim.x)
            s.P[v] = pc[v];
        if (t > 0)
            for (size_t e = threadIdx.x; e < E; e += blockDim.x)
                s.M[e] = mc[e];
        if ((int)threadIdx.x < kLearnedMaxClass) {
            sdb[threadIdx.x] = 0.0f;
            sda[threadIdx.x] = 0.0f;
        }
        load_params(p, t, sbeta, salpha);
        iteration_fwd(c, s, p, t, sbeta, salpha); /* saves X */
        iteration_loss(c, s, p, f, p.loss_scale * (p.loss_w ? p.loss_w[t] : 1.0f));
        __syncthreads();
        float db[kLearnedMaxClass], da[kLearnedMaxClass];
        for (int k = 0; k < p.nclass; k++)
            db[k] = da[k] = 0.0f;
        for (int st_i = c.nsteps - 1; st_i >= 0; st_i--) {
            const uint32_t st = c.steps[st_i];
            const int i = st & 0xFF, start = (st >> 8) & 0x1FF, n = (st >> 17) & 0x1FF;
            for (int g = threadIdx.x; g < n; g += blockDim.x) {
                const int pos = start + g;
                const int j = (st >> 26) ? (int)c.perm[kQCl * i + pos] : pos;
                const int D = c.eoff[i + 1] - c.eoff[i] + 2 - ((i | j) ? 0 : 1);
                const int k = p.cls[D];
                float b = 0.0f, a = 0.0f;
                check_bwd(c, s, i, j, kQCl * i + pos, sbeta[k], salpha[k], t == 0, b, a);
                for (int kk = 0; kk < p.nclass; kk++)
                    if (kk == k) {
                        db[kk] += b;
                        da[kk] += a;
                    }
            }
            __syncthreads();
        }
        for (int k = 0; k < p.nclass; k++) {
            const float b = block_sum(db[k], red), a = block_sum(da[k], red);
            if (threadIdx.x == 0) {
                atomicAdd(p.dbeta + t * p.nclass + k, b);
                atomicAdd(p.dalpha + t * p.nclass + k, a);
            }
        }
    }
}

size_t learned_workspace_bytes(const DevCode& host_code_shape, int R, int N, int DS, int nframes, int iters,
                               bool train)
{
    (void)host_code_shape;
    const size_t E = (size_t)DS * R;
    size_t b = (size_t)nframes * (N + E) * sizeof(float); /* P, M */
    if (train)
        b += (size_t)nframes * (N + 2 * E) * sizeof(float) +          /* gP, gM, X */
             (size_t)iters * nframes * (N + E) * sizeof(float);        /* checkpoints */
    return b;
}

cudaError_t launch_learned(const LearnedParams& p, bool backward, cudaStream_t s)
{
    if (backward)
        k_learned_bwd<<<p.nframes, kLT, 0, s>>>(p);
    else
        k_learned_fwd<<<p.nframes, kLT, 0, s>>>(p);
    return cudaGetLastError();
}

}  // namespace drxg
