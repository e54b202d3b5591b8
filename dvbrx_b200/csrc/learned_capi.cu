/*
 * C ABI of the learned decoder's training kernels (learned.cu) and of the
 * schedule introspection used by float references.
 *
 * The caller owns all memory: a workspace sized by
 * drx_learned_workspace_bytes, the per-iteration loss sums and the gradient
 * accumulators.  Workspace layout: 64 bytes of check-degree classes, then
 * (16-byte aligned) P, M, and for training X, gP, gM, the P checkpoints and
 * the message checkpoints, all fp32.
 */
#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "handle.h"
#include "learned.h"

using namespace drxg;

namespace {

size_t a16(size_t v) { return (v + 15) & ~(size_t)15; }

struct WsLayout {
    size_t cls, P, M, X, gP, gM, Pck, Mck, total;
};

WsLayout layout(const drx_ldpc* d, int nframes, int iters, bool train)
{
    const size_t N = d->code.N, E = (size_t)d->code.deg_max * d->code.R, F = nframes;
    WsLayout w{};
    size_t off = 0;
    w.cls = off;
    off += 64;
    w.P = off;
    off = a16(off + F * N * 4);
    w.M = off;
    off = a16(off + F * E * 4);
    if (train) {
        w.X = off;
        off = a16(off + F * E * 4);
        w.gP = off;
        off = a16(off + F * N * 4);
        w.gM = off;
        off = a16(off + F * E * 4);
        w.Pck = off;
        off = a16(off + (size_t)iters * F * N * 4);
        w.Mck = off;
        off = a16(off + (size_t)iters * F * E * 4);
    }
    w.total = off;
    return w;
}

int fill(drx_ldpc* d, LearnedParams& p, int nframes, const void* llr, size_t llr_stride, const uint8_t* bits,
         size_t bits_stride, int iters, const void* beta, const void* alpha, int nclass,
         const int8_t* class_of_degree, void* ws, size_t ws_bytes, bool train, cudaStream_t s)
{
    if (!d || nframes <= 0 || iters <= 0 || !llr || !bits || !beta || !alpha || !ws || !class_of_degree) {
        set_error("learned decoder: bad arguments");
        return -1;
    }
    if (nclass < 1 || nclass > kLearnedMaxClass || d->code.deg_max > kLearnedMaxDeg) {
        set_error("learned decoder: unsupported class count or degree");
        return -1;
    }
    for (int k = 0; k <= 32; k++)
        if (class_of_degree[k] < 0 || class_of_degree[k] >= nclass) {
            set_error("learned decoder: class of a degree out of range");
            return -1;
        }
    if (llr_stride < (size_t)d->code.N || bits_stride < (size_t)d->nbytes) {
        set_error("learned decoder: row stride below the frame size");
        return -1;
    }
    const WsLayout w = layout(d, nframes, iters, train);
    if (ws_bytes < w.total) {
        set_error("learned decoder: workspace too small");
        return -1;
    }
    char* b = (char*)ws;
    if (!cuda_check(cudaMemcpyAsync(b + w.cls, class_of_degree, 33, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync"))
        return -1;
    p = LearnedParams{};
    p.code = d->dcode;
    p.nframes = nframes;
    p.iters = iters;
    p.DS = d->code.deg_max;
    p.llr = (const __half*)llr;
    p.llr_stride = llr_stride;
    p.bits = bits;
    p.bits_stride = bits_stride;
    p.beta = (const __half*)beta;
    p.alpha = (const __half*)alpha;
    p.nclass = nclass;
    p.cls = (const int8_t*)(b + w.cls);
    p.P = (float*)(b + w.P);
    p.M = (float*)(b + w.M);
    if (train) {
        p.X = (float*)(b + w.X);
        p.gP = (float*)(b + w.gP);
        p.gM = (float*)(b + w.gM);
        p.Pck = (float*)(b + w.Pck);
        p.Mck = (float*)(b + w.Mck);
    }
    return 0;
}

}  // namespace

extern "C" {

size_t drx_learned_workspace_bytes(const drx_ldpc* d, int nframes, int iters, int train)
{
    if (!d || nframes <= 0 || iters <= 0)
        return 0;
    return layout(d, nframes, iters, train != 0).total;
}

int drx_learned_forward(drx_ldpc* d, int nframes, const void* llr_f16, size_t llr_stride, const uint8_t* bits,
                        size_t bits_stride, int iters, const void* beta_f16, const void* alpha_f16, int nclass,
                        const int8_t* class_of_degree, float* loss, float* post, void* workspace,
                        size_t workspace_bytes, int train, void* stream)
{
    cudaStream_t s = stream ? (cudaStream_t)stream : (d ? d->stream : nullptr);
    LearnedParams p;
    if (fill(d, p, nframes, llr_f16, llr_stride, bits, bits_stride, iters, beta_f16, alpha_f16, nclass,
             class_of_degree, workspace, workspace_bytes, train != 0, s))
        return -1;
    if (!loss) {
        set_error("learned decoder: loss buffer missing");
        return -1;
    }
    p.loss = loss;
    p.post = post;
    return cuda_check(launch_learned(p, false, s), "learned forward") ? 0 : -1;
}

int drx_learned_backward(drx_ldpc* d, int nframes, const void* llr_f16, size_t llr_stride, const uint8_t* bits,
                         size_t bits_stride, int iters, const void* beta_f16, const void* alpha_f16, int nclass,
                         const int8_t* class_of_degree, float loss_scale, const float* iter_weights,
                         float* dbeta, float* dalpha, float* loss_scratch, void* workspace,
                         size_t workspace_bytes, void* stream)
{
    cudaStream_t s = stream ? (cudaStream_t)stream : (d ? d->stream : nullptr);
    LearnedParams p;
    if (fill(d, p, nframes, llr_f16, llr_stride, bits, bits_stride, iters, beta_f16, alpha_f16, nclass,
             class_of_degree, workspace, workspace_bytes, true, s))
        return -1;
    if (!dbeta || !dalpha || !loss_scratch) {
        set_error("learned decoder: gradient buffers missing");
        return -1;
    }
    p.loss = loss_scratch;
    p.loss_scale = loss_scale;
    p.loss_w = iter_weights;
    p.dbeta = dbeta;
    p.dalpha = dalpha;
    return cuda_check(launch_learned(p, true, s), "learned backward") ? 0 : -1;
}

int drx_ldpc_schedule(int short_frame, const char* rate, int* nsteps, int* deg_max, int32_t* check_step,
                      int32_t* links)
{
    const int table = find_table(short_frame, rate);
    if (table < 0) {
        set_error("no LDPC table for this rate");
        return -1;
    }
    Code c;
    std::string err;
    if (!compile_code(table, &c, &err)) {
        set_error(err);
        return -1;
    }
    if (nsteps)
        *nsteps = (int)c.steps.size();
    if (deg_max)
        *deg_max = c.deg_max;
    if (!check_step && !links)
        return 0;
    for (size_t s = 0; s < c.steps.size(); s++) {
        const uint32_t st = c.steps[s];
        const int i = st & 0xFF, start = (st >> 8) & 0x1FF, n = (st >> 17) & 0x1FF;
        for (int g = 0; g < n; g++) {
            const int j = c.perm[(size_t)QC * i + start + g];
            const int chk = QC * i + j;
            if (check_step)
                check_step[chk] = (int32_t)s;
            if (links) {
                int32_t* l = links + (size_t)chk * c.deg_max;
                for (int k = 0; k < c.deg_max; k++)
                    l[k] = -1;
                const int k0 = c.q * j + i; /* the check's index in codeword order */
                l[0] = c.K + k0;
                l[1] = k0 ? c.K + k0 - 1 : -1;
                const int e0 = c.eoff[i], e1 = c.eoff[i + 1];
                for (int e = e0; e < e1; e++) {
                    const int bx = c.ent[2 * e], a = c.ent[2 * e + 1];
                    l[2 + e - e0] = bx + j + (j < a ? QC : 0);
                }
            }
        }
    }
    return 0;
}

}  // extern "C"
