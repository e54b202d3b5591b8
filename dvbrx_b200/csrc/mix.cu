/*
 * Mixed batches: frames of several codes (MODCODs, normal and short) in one
 * device batch, decoded with per-frame stopping, replayed as a CUDA graph.
 *
 * Two tilings decode the same batch with identical results:
 *
 *   DRX_TILING_ONE_LAUNCH  one persistent launch over every frame, one frame
 *       per CTA; frames are ordered longest-work first (normal before short,
 *       then by Tanner-graph edges, frames of one code together) and the
 *       CTAs pull them from one counter, restaging the code tables in shared
 *       memory when the code changes.  Its kernel is compiled for the largest
 *       check degree of the mix.
 *   DRX_TILING_PER_CODE    one persistent launch per code with the code's
 *       own kernel (the frame-pair kernel, two frames per CTA, where it
 *       applies), spread over concurrent streams that the CUDA graph runs as
 *       parallel branches, so that the tail of one code's launch overlaps the
 *       next code's.
 *
 * drx_ldpc_mix_tune times both graphs on the planned batch and keeps the
 * faster: the choice between one frame per CTA and two frames per CTA, and
 * between one launch and per-code launches, is measured, not assumed.
 */
#include <cuda_runtime.h>
#include <string.h>

#include <algorithm>
#include <numeric>
#include <string>
#include <vector>

#include "handle.h"
#include "mixpair.h"

using namespace drxg;

namespace {

constexpr int kSideStreams = 4;

}  // namespace

struct drx_ldpc_mix {
    std::vector<drx_ldpc*> codes;
    const DevCode** d_codes = nullptr; /* device array of the codes' descriptors */
    int dclass_max = 0;
    size_t mix_smem = 0;
    int mix_ctas = 0; /* resident CTAs of the one-launch kernel */
    int sms = 0;
    cudaStream_t capture = nullptr;
    cudaStream_t side[kSideStreams] = {};
    cudaEvent_t fork = nullptr, join[kSideStreams] = {};
    /* plan */
    int nframes = 0;
    int32_t* d_frame_code = nullptr;
    int32_t* d_order = nullptr;
    unsigned* d_work = nullptr; /* one counter per code, then one for the one-launch kernel */
    void* d_msg = nullptr;
    /* learned plans: per-code learned tables (device pointer arrays), the
     * failing rows of the learned pass (nframes + a count) and flags */
    const uint32_t** d_learn = nullptr;
    const int8_t** d_learn_cls = nullptr;
    int* d_learn_iters = nullptr;
    int32_t* d_fb_rows = nullptr;
    uint8_t* d_fb_ok = nullptr;
    /* one launch, two frames per CTA: per code start, count, shape, weight,
     * then the first code of every CTA; one counter per code */
    int* d_pair = nullptr;
    unsigned* d_pair_work = nullptr;
    cudaGraphExec_t exec[4] = {};
    int tiling = DRX_TILING_ONE_LAUNCH;
    float tuned_ms[4] = {};
};

namespace {

void release_plan(drx_ldpc_mix* m)
{
    for (auto& e : m->exec)
        if (e) {
            cudaGraphExecDestroy(e);
            e = nullptr;
        }
    cudaFree(m->d_frame_code);
    cudaFree(m->d_order);
    cudaFree(m->d_work);
    cudaFree(m->d_msg);
    cudaFree(m->d_learn);
    cudaFree(m->d_learn_cls);
    cudaFree(m->d_learn_iters);
    cudaFree(m->d_fb_rows);
    cudaFree(m->d_fb_ok);
    cudaFree(m->d_pair);
    cudaFree(m->d_pair_work);
    m->d_pair = nullptr;
    m->d_pair_work = nullptr;
    m->d_learn = nullptr;
    m->d_learn_cls = nullptr;
    m->d_learn_iters = nullptr;
    m->d_fb_rows = nullptr;
    m->d_fb_ok = nullptr;
    m->d_frame_code = m->d_order = nullptr;
    m->d_work = nullptr;
    m->d_msg = nullptr;
    m->nframes = 0;
}

bool pair_runs(const drx_ldpc* h) { return h->variant != DRX_VARIANT_FRAME && h->pair_ctas_per_sm > 0; }

constexpr int kCompactThreads = 1024;

/* The rows of `order` whose flag in ok is 0, in `order`'s sequence (so a
 * code's frames stay together), into rows; their number into *count and a
 * flag per row into fallback (may be null).  One block: each thread scans a
 * contiguous chunk, a block-wide exclusive scan places the chunks. */
__global__ void __launch_bounds__(kCompactThreads) k_compact_failing(const int32_t* __restrict__ order,
                                                                     const uint8_t* __restrict__ ok, int n,
                                                                     int32_t* __restrict__ rows, int* count,
                                                                     uint8_t* __restrict__ fallback)
{
    __shared__ int warp_sum[kCompactThreads / 32];
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    const int chunk = (n + kCompactThreads - 1) / kCompactThreads;
    const int b = min(n, t * chunk), e = min(n, b + chunk);
    int mine = 0;
    for (int k = b; k < e; k++) {
        const int r = order[k];
        const bool fail = ok[r] == 0;
        if (fallback)
            fallback[r] = fail ? 1 : 0;
        mine += fail;
    }
    int x = mine; /* inclusive scan in the warp */
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xFFFFFFFFu, x, o);
        if (lane >= o)
            x += y;
    }
    if (lane == 31)
        warp_sum[w] = x;
    __syncthreads();
    if (w == 0) {
        int s = lane < kCompactThreads / 32 ? warp_sum[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xFFFFFFFFu, s, o);
            if (lane >= o)
                s += y;
        }
        if (lane < kCompactThreads / 32)
            warp_sum[lane] = s; /* inclusive over warps */
    }
    __syncthreads();
    int pos = x - mine + (w > 0 ? warp_sum[w - 1] : 0);
    for (int k = b; k < e; k++) {
        const int r = order[k];
        if (ok[r] == 0)
            rows[pos++] = r;
    }
    if (t == kCompactThreads - 1)
        *count = pos;
}

}  // namespace

extern "C" {

drx_ldpc_mix* drx_ldpc_mix_new(int ncodes, const drx_fec_params* params, const char* const* rates)
{
    if (ncodes <= 0 || !params || !rates) {
        set_error("drx_ldpc_mix_new: no codes");
        return nullptr;
    }
    drx_ldpc_mix* m = new drx_ldpc_mix();
    for (int c = 0; c < ncodes; c++) {
        drx_ldpc* h = drx_ldpc_new(&params[c], rates[c]);
        if (!h) {
            drx_ldpc_mix_free(m);
            return nullptr;
        }
        m->codes.push_back(h);
        m->dclass_max = std::max(m->dclass_max, h->code.dclass);
        m->mix_smem = std::max(m->mix_smem, h->smem);
    }
    m->sms = m->codes[0]->sms;
    std::vector<const DevCode*> ptrs;
    for (auto* h : m->codes)
        ptrs.push_back(h->dcode);
    bool ok = cuda_check(drxg::dev_malloc(&m->d_codes, sizeof(DevCode*) * ncodes), "cudaMalloc") &&
              cuda_check(cudaMemcpy(m->d_codes, ptrs.data(), sizeof(DevCode*) * ncodes, cudaMemcpyHostToDevice),
                         "cudaMemcpy") &&
              cuda_check(cudaStreamCreateWithFlags(&m->capture, cudaStreamNonBlocking), "cudaStreamCreate") &&
              cuda_check(cudaEventCreateWithFlags(&m->fork, cudaEventDisableTiming), "cudaEventCreate");
    for (int k = 0; ok && k < kSideStreams; k++)
        ok = cuda_check(cudaStreamCreateWithFlags(&m->side[k], cudaStreamNonBlocking), "cudaStreamCreate") &&
             cuda_check(cudaEventCreateWithFlags(&m->join[k], cudaEventDisableTiming), "cudaEventCreate");
    if (ok) {
        m->mix_ctas = decode_mix_ctas_per_sm(m->dclass_max, m->mix_smem);
        ok = m->mix_ctas > 0;
        if (!ok)
            set_error("drx_ldpc_mix_new: the mixed kernel does not fit on this device");
    }
    if (!ok) {
        drx_ldpc_mix_free(m);
        return nullptr;
    }
    return m;
}

void drx_ldpc_mix_free(drx_ldpc_mix* m)
{
    if (!m)
        return;
    if (m->capture)
        cudaStreamSynchronize(m->capture);
    for (int k = 0; k < kSideStreams; k++)
        if (m->side[k])
            cudaStreamSynchronize(m->side[k]);
    release_plan(m);
    cudaFree(m->d_codes);
    for (int k = 0; k < kSideStreams; k++) {
        if (m->side[k])
            cudaStreamDestroy(m->side[k]);
        if (m->join[k])
            cudaEventDestroy(m->join[k]);
    }
    if (m->fork)
        cudaEventDestroy(m->fork);
    if (m->capture)
        cudaStreamDestroy(m->capture);
    for (auto* h : m->codes)
        drx_ldpc_free(h);
    delete m;
}

}  // extern "C"

namespace {

/* Plan (capture) both tilings of a mixed batch.  learned: the first pass
 * runs every code's learned table for at most max_iter iterations, then the
 * failing rows are gathered on the device and decoded again by the plain
 * decoder (at most plain_max_iter iterations; none if <= 0): in one launch
 * for the one-launch tiling, per code right after its learned pass for the
 * per-code tiling. */
int plan_mix(drx_ldpc_mix* m, int nframes, const int32_t* code, const int8_t* llr, size_t llr_stride,
             uint8_t* out, size_t out_stride, int32_t* iters, uint8_t* ok, int max_iter, bool learned,
             int plain_max_iter, uint8_t* fallback)
{
    if (!m || nframes <= 0 || !code || !llr || !out) {
        set_error("drx_ldpc_mix_plan: bad arguments");
        return -1;
    }
    const int ncodes = (int)m->codes.size();
    size_t maxN = 0, maxbytes = 0;
    for (auto* h : m->codes) {
        maxN = std::max(maxN, (size_t)h->code.N);
        maxbytes = std::max(maxbytes, (size_t)h->nbytes);
    }
    if (llr_stride < maxN || out_stride < maxbytes) {
        set_error("drx_ldpc_mix_plan: row stride below the largest frame of the mix");
        return -1;
    }
    std::vector<int> count(ncodes, 0);
    for (int f = 0; f < nframes; f++) {
        if (code[f] < 0 || code[f] >= ncodes) {
            set_error("drx_ldpc_mix_plan: code index out of range");
            return -1;
        }
        count[code[f]]++;
    }
    if (max_iter < 0)
        max_iter = 0;
    if (learned)
        for (int c = 0; c < ncodes; c++)
            if (count[c] && m->codes[c]->learn_iters <= 0) {
                set_error("drx_ldpc_mix_plan_learned: a code of the batch has no learned table");
                return -1;
            }
    release_plan(m);
    /* longest work first: normal frames, then by edges; a code's frames together */
    std::vector<int> corder(ncodes);
    std::iota(corder.begin(), corder.end(), 0);
    std::stable_sort(corder.begin(), corder.end(), [&](int a, int b) {
        const Code &ca = m->codes[a]->code, &cb = m->codes[b]->code;
        if (ca.N != cb.N)
            return ca.N > cb.N;
        return ca.edges > cb.edges;
    });
    std::vector<int> start(ncodes, 0);
    int pos = 0;
    for (int c : corder) {
        start[c] = pos;
        pos += count[c];
    }
    std::vector<int32_t> order(nframes);
    std::vector<int> fill(start);
    for (int f = 0; f < nframes; f++)
        order[fill[code[f]]++] = f;

    /* scratch: per side stream, the largest slab x grid of its codes; the
     * one-launch kernel reuses the same memory (the graphs never overlap) */
    std::vector<size_t> side_bytes(kSideStreams, 0);
    std::vector<size_t> side_off(kSideStreams, 0);
    std::vector<int> code_side(ncodes, 0);
    std::vector<int> code_grid(ncodes, 0);
    std::vector<size_t> code_slab(ncodes, 0);
    int k = 0;
    for (int c : corder) {
        if (!count[c])
            continue;
        drx_ldpc* h = m->codes[c];
        const bool pair = pair_runs(h);
        code_slab[c] = pair ? decode_pair_msg_bytes(h->code.R, h->pair_kid) : decode_msg_bytes(h->code.R, h->code.dclass);
        code_grid[c] = pair ? std::min((count[c] + 1) / 2, h->pair_ctas_per_sm * h->sms)
                            : std::min(count[c], h->ctas_per_sm * h->sms);
        code_side[c] = k;
        side_bytes[k] = std::max(side_bytes[k], code_slab[c] * (size_t)code_grid[c]);
        k = (k + 1) % kSideStreams;
    }
    size_t total = 0;
    for (int s = 0; s < kSideStreams; s++) {
        side_off[s] = total;
        total += (side_bytes[s] + 255) & ~(size_t)255;
    }
    const size_t mix_slab = decode_msg_bytes(
        std::max_element(m->codes.begin(), m->codes.end(), [](drx_ldpc* a, drx_ldpc* b) { return a->code.R < b->code.R; })[0]->code.R,
        m->dclass_max);
    const int mix_grid = std::min(nframes, m->mix_ctas * m->sms);
    total = std::max(total, mix_slab * (size_t)mix_grid);

    /* one launch, two frames per CTA (plain plans, every code of the batch
     * with a shape in the mixed kernel): shared memory and slab of the
     * largest code, CTAs spread over the codes by their work */
    bool pair_plan = !learned;
    std::vector<int> shape(ncodes, -1), weight(ncodes, 0);
    size_t pair_smem = 0, pair_slab = 0;
    for (int c = 0; c < ncodes && pair_plan; c++) {
        if (!count[c])
            continue;
        drx_ldpc* h = m->codes[c];
        const int kid = pair_runs(h) ? pair_kernel_id(h->code) : -1;
        int a, b, g, ls, pm;
        if (kid < 0 || !pair_kernel_shape(kid, &a, &b, &g, &ls, &pm) || (shape[c] = mix_pair_shape(a, b, g, ls)) < 0) {
            pair_plan = false;
            break;
        }
        weight[c] = (int)std::min<long long>(h->code.edges, 1 << 30);
        pair_smem = std::max(pair_smem, decode_pair_smem_bytes(h->code.N, h->code.K, (int)h->code.ent.size() / 2,
                                                               (int)h->code.steps.size(), h->code.q, kid));
        pair_slab = std::max(pair_slab, decode_pair_msg_bytes(h->code.R, kid));
    }
    int pair_grid = 0;
    std::vector<int> pair_host;
    if (pair_plan) {
        pair_grid = std::min(decode_mix_pair_ctas_per_sm(pair_smem) * m->sms, (nframes + 1) / 2);
        pair_plan = pair_grid > 0;
    }
    if (pair_plan) {
        pair_host.assign(4 * (size_t)ncodes + pair_grid, 0);
        double wsum = 0;
        for (int c = 0; c < ncodes; c++) {
            pair_host[c] = start[c];
            pair_host[ncodes + c] = count[c];
            pair_host[2 * ncodes + c] = shape[c];
            pair_host[3 * ncodes + c] = weight[c];
            wsum += (double)count[c] * weight[c];
        }
        /* CTA k starts on the code whose share of the work covers (k + 1/2) / grid */
        double acc = 0;
        int ci = 0;
        for (int k = 0; k < pair_grid; k++) {
            const double at = (k + 0.5) / pair_grid * wsum;
            while (ci < ncodes && acc + (double)count[corder[ci]] * weight[corder[ci]] < at) {
                acc += (double)count[corder[ci]] * weight[corder[ci]];
                ci++;
            }
            pair_host[4 * (size_t)ncodes + k] = corder[std::min(ci, ncodes - 1)];
        }
        total = std::max(total, pair_slab * (size_t)pair_grid);
    }
    if (!cuda_check(drxg::dev_malloc(&m->d_frame_code, sizeof(int32_t) * nframes), "cudaMalloc") ||
        !cuda_check(drxg::dev_malloc(&m->d_order, sizeof(int32_t) * nframes), "cudaMalloc") ||
        !cuda_check(drxg::dev_malloc(&m->d_work, sizeof(unsigned) * (2 * ncodes + 1)), "cudaMalloc") ||
        !cuda_check(drxg::dev_malloc(&m->d_msg, total), "cudaMalloc") ||
        !cuda_check(cudaMemcpy(m->d_frame_code, code, sizeof(int32_t) * nframes, cudaMemcpyHostToDevice), "cudaMemcpy") ||
        !cuda_check(cudaMemcpy(m->d_order, order.data(), sizeof(int32_t) * nframes, cudaMemcpyHostToDevice), "cudaMemcpy") ||
        (pair_plan &&
         (!cuda_check(drxg::dev_malloc(&m->d_pair, sizeof(int) * pair_host.size()), "cudaMalloc") ||
          !cuda_check(drxg::dev_malloc(&m->d_pair_work, sizeof(unsigned) * ncodes), "cudaMalloc") ||
          !cuda_check(cudaMemcpy(m->d_pair, pair_host.data(), sizeof(int) * pair_host.size(), cudaMemcpyHostToDevice),
                      "cudaMemcpy")))) {
        release_plan(m);
        return -1;
    }
    if (learned) {
        std::vector<const uint32_t*> lt(ncodes, nullptr);
        std::vector<const int8_t*> lc(ncodes, nullptr);
        std::vector<int> li(ncodes, 0);
        for (int c = 0; c < ncodes; c++) {
            drx_ldpc* h = m->codes[c];
            if (h->learn_iters > 0) {
                lt[c] = h->learn;
                lc[c] = (const int8_t*)((const char*)h->learn + sizeof(uint32_t) * kLearnMaxIters * kLearnClasses);
                li[c] = h->learn_iters;
            }
        }
        if (!cuda_check(drxg::dev_malloc(&m->d_learn, sizeof(void*) * ncodes), "cudaMalloc") ||
            !cuda_check(drxg::dev_malloc(&m->d_learn_cls, sizeof(void*) * ncodes), "cudaMalloc") ||
            !cuda_check(drxg::dev_malloc(&m->d_learn_iters, sizeof(int) * ncodes), "cudaMalloc") ||
            !cuda_check(drxg::dev_malloc(&m->d_fb_rows, sizeof(int32_t) * (nframes + 4 + ncodes)), "cudaMalloc") ||
            !cuda_check(drxg::dev_malloc(&m->d_fb_ok, nframes), "cudaMalloc") ||
            !cuda_check(cudaMemcpy(m->d_learn, lt.data(), sizeof(void*) * ncodes, cudaMemcpyHostToDevice), "cudaMemcpy") ||
            !cuda_check(cudaMemcpy(m->d_learn_cls, lc.data(), sizeof(void*) * ncodes, cudaMemcpyHostToDevice), "cudaMemcpy") ||
            !cuda_check(cudaMemcpy(m->d_learn_iters, li.data(), sizeof(int) * ncodes, cudaMemcpyHostToDevice), "cudaMemcpy")) {
            release_plan(m);
            return -1;
        }
        if (!ok)
            ok = m->d_fb_ok;
    }
    m->nframes = nframes;
    /* kernel attributes are set before capture (not a stream operation) */
    decode_mix_ctas_per_sm(m->dclass_max, m->mix_smem);
    if (pair_plan)
        decode_mix_pair_ctas_per_sm(pair_smem);
    for (auto* h : m->codes) {
        decode_ctas_per_sm(h->code.dclass, h->smem);
        if (h->pair_ctas_per_sm > 0)
            decode_pair_ctas_per_sm(h->pair_kid, h->pair_smem);
    }

    for (int t = DRX_TILING_ONE_LAUNCH; t <= DRX_TILING_ONE_LAUNCH_PAIR; t++) {
        if (t == DRX_TILING_ONE_LAUNCH_PAIR && !pair_plan)
            continue;
        cudaGraph_t g = nullptr;
        if (!cuda_check(cudaStreamBeginCapture(m->capture, cudaStreamCaptureModeRelaxed), "cudaStreamBeginCapture")) {
            release_plan(m);
            return -1;
        }
        cudaError_t e = cudaSuccess;
        if (t == DRX_TILING_ONE_LAUNCH) {
            MixParams p{};
            p.codes = m->d_codes;
            p.frame_code = m->d_frame_code;
            p.order = m->d_order;
            p.llr = llr;
            p.llr_stride = llr_stride;
            p.out = out;
            p.out_stride = out_stride;
            p.iters = iters;
            p.ok = ok;
            p.nframes = nframes;
            p.max_iter = max_iter;
            p.work = m->d_work + ncodes;
            p.msg = m->d_msg;
            p.msg_stride = mix_slab;
            if (learned) {
                p.learn = m->d_learn;
                p.learn_class = m->d_learn_cls;
                p.learn_iters = m->d_learn_iters;
            }
            e = cudaMemsetAsync(p.work, 0, sizeof(unsigned), m->capture);
            if (e == cudaSuccess)
                e = launch_decode_mix(p, m->dclass_max, m->mix_smem, mix_grid, m->capture);
        } else if (t == DRX_TILING_ONE_LAUNCH_PAIR) {
            MixPairParams p{};
            p.base.codes = m->d_codes;
            p.base.frame_code = m->d_frame_code;
            p.base.order = m->d_order;
            p.base.llr = llr;
            p.base.llr_stride = llr_stride;
            p.base.out = out;
            p.base.out_stride = out_stride;
            p.base.iters = iters;
            p.base.ok = ok;
            p.base.nframes = nframes;
            p.base.max_iter = max_iter;
            p.base.msg = m->d_msg;
            p.base.msg_stride = pair_slab;
            p.code_start = m->d_pair;
            p.code_count = m->d_pair + ncodes;
            p.code_shape = m->d_pair + 2 * ncodes;
            p.code_weight = m->d_pair + 3 * ncodes;
            p.cta_code = m->d_pair + 4 * ncodes;
            p.code_work = m->d_pair_work;
            p.ncodes = ncodes;
            e = cudaMemsetAsync(m->d_pair_work, 0, sizeof(unsigned) * ncodes, m->capture);
            if (e == cudaSuccess)
                e = launch_decode_mix_pair(p, pair_smem, pair_grid, m->capture);
        } else {
            e = cudaEventRecord(m->fork, m->capture);
            for (int s = 0; s < kSideStreams && e == cudaSuccess; s++)
                e = cudaStreamWaitEvent(m->side[s], m->fork, 0);
            for (int c : corder) {
                if (!count[c] || e != cudaSuccess)
                    continue;
                drx_ldpc* h = m->codes[c];
                cudaStream_t s = m->side[code_side[c]];
                DecodeParams p{};
                p.code = h->dcode;
                p.llr = llr;
                p.llr_stride = llr_stride;
                p.out = out;
                p.out_stride = out_stride;
                p.iters = iters;
                p.ok = ok;
                p.nframes = count[c];
                p.max_iter = max_iter;
                p.err = h->err;
                p.rows = m->d_order + start[c];
                p.work = m->d_work + c;
                p.msg = (char*)m->d_msg + side_off[code_side[c]];
                p.msg_stride = code_slab[c];
                if (learned) {
                    p.learn = h->learn;
                    p.learn_class = (const int8_t*)((const char*)h->learn +
                                                    sizeof(uint32_t) * kLearnMaxIters * kLearnClasses);
                    p.learn_iters = h->learn_iters;
                }
                e = cudaMemsetAsync(p.work, 0, sizeof(unsigned), s);
                if (e == cudaSuccess)
                    e = pair_runs(h) ? launch_decode_pair(p, h->pair_kid, h->pair_smem, code_grid[c], s)
                                     : launch_decode(p, h->code.dclass, h->smem, code_grid[c], s);
                if (learned && e == cudaSuccess) {
                    /* fallback of this code, on its stream: its failing rows through its own
                     * plain kernel (the count read on the device) */
                    int* cnt = (int*)(m->d_fb_rows + nframes + 4) + c;
                    k_compact_failing<<<1, kCompactThreads, 0, s>>>(m->d_order + start[c], ok, count[c],
                                                                    m->d_fb_rows + start[c], cnt, fallback);
                    e = cudaGetLastError();
                    if (e == cudaSuccess && plain_max_iter > 0) {
                        DecodeParams q = p;
                        q.learn = nullptr;
                        q.learn_class = nullptr;
                        q.learn_iters = 0;
                        q.rows = m->d_fb_rows + start[c];
                        q.nframes_dev = cnt;
                        q.max_iter = plain_max_iter;
                        q.work = m->d_work + ncodes + 1 + c;
                        e = cudaMemsetAsync(q.work, 0, sizeof(unsigned), s);
                        if (e == cudaSuccess)
                            e = pair_runs(h) ? launch_decode_pair(q, h->pair_kid, h->pair_smem, code_grid[c], s)
                                             : launch_decode(q, h->code.dclass, h->smem, code_grid[c], s);
                    }
                }
            }
            for (int s = 0; s < kSideStreams; s++) {
                if (e == cudaSuccess)
                    e = cudaEventRecord(m->join[s], m->side[s]);
                if (e == cudaSuccess)
                    e = cudaStreamWaitEvent(m->capture, m->join[s], 0);
            }
        }
        if (learned && t == DRX_TILING_ONE_LAUNCH && e == cudaSuccess) {
            /* fallback: the failing rows, in processing order, through the plain one-launch kernel */
            int* cnt = (int*)(m->d_fb_rows + nframes);
            k_compact_failing<<<1, kCompactThreads, 0, m->capture>>>(m->d_order, ok, nframes, m->d_fb_rows, cnt,
                                                                     fallback);
            e = cudaGetLastError();
            if (e == cudaSuccess && plain_max_iter > 0) {
                MixParams p{};
                p.codes = m->d_codes;
                p.frame_code = m->d_frame_code;
                p.order = m->d_fb_rows;
                p.llr = llr;
                p.llr_stride = llr_stride;
                p.out = out;
                p.out_stride = out_stride;
                p.iters = iters;
                p.ok = ok;
                p.nframes = nframes;
                p.nframes_dev = cnt;
                p.max_iter = plain_max_iter;
                p.work = m->d_work + ncodes;
                p.msg = m->d_msg;
                p.msg_stride = mix_slab;
                e = cudaMemsetAsync(p.work, 0, sizeof(unsigned), m->capture);
                if (e == cudaSuccess)
                    e = launch_decode_mix(p, m->dclass_max, m->mix_smem, mix_grid, m->capture);
            }
        }
        const cudaError_t e2 = cudaStreamEndCapture(m->capture, &g);
        if (e == cudaSuccess)
            e = e2;
        if (e == cudaSuccess)
            e = cudaGraphInstantiate(&m->exec[t], g, 0);
        if (g)
            cudaGraphDestroy(g);
        if (!cuda_check(e, "mixed-batch graph")) {
            release_plan(m);
            return -1;
        }
    }
    return 0;
}

}  // namespace

extern "C" {

int drx_ldpc_mix_plan(drx_ldpc_mix* m, int nframes, const int32_t* code, const int8_t* llr, size_t llr_stride,
                      uint8_t* out, size_t out_stride, int32_t* iters, uint8_t* ok, int max_iter)
{
    return plan_mix(m, nframes, code, llr, llr_stride, out, out_stride, iters, ok, max_iter, false, 0, nullptr);
}

int drx_ldpc_mix_plan_learned(drx_ldpc_mix* m, int nframes, const int32_t* code, const int8_t* llr,
                              size_t llr_stride, uint8_t* out, size_t out_stride, int32_t* iters, uint8_t* ok,
                              uint8_t* fallback, int learned_iters, int plain_max_iter)
{
    return plan_mix(m, nframes, code, llr, llr_stride, out, out_stride, iters, ok, learned_iters, true,
                    plain_max_iter, fallback);
}

int drx_ldpc_mix_set_learned(drx_ldpc_mix* m, int code_index, int iters, int nclass, const int8_t* class_of_degree,
                             const float* scale, const float* offset)
{
    if (!m || code_index < 0 || code_index >= (int)m->codes.size()) {
        set_error("drx_ldpc_mix_set_learned: code index out of range");
        return -1;
    }
    return drx_ldpc_set_learned(m->codes[code_index], iters, nclass, class_of_degree, scale, offset);
}

int drx_ldpc_mix_set_tiling(drx_ldpc_mix* m, int tiling)
{
    if (!m || tiling < DRX_TILING_ONE_LAUNCH || tiling > DRX_TILING_ONE_LAUNCH_PAIR) {
        set_error("drx_ldpc_mix_set_tiling: unknown tiling");
        return -1;
    }
    if (m->nframes && !m->exec[tiling]) {
        set_error("drx_ldpc_mix_set_tiling: the plan has no such tiling (two frames per CTA in one launch needs "
                  "a plain plan of DVB-S2 codes)");
        return -1;
    }
    m->tiling = tiling;
    return tiling;
}

int drx_ldpc_mix_run(drx_ldpc_mix* m, void* stream)
{
    if (!m || !m->nframes || !m->exec[m->tiling]) {
        set_error("drx_ldpc_mix_run: no plan");
        return -1;
    }
    return cuda_check(cudaGraphLaunch(m->exec[m->tiling], stream ? (cudaStream_t)stream : m->capture),
                      "cudaGraphLaunch") ? 0 : -1;
}

int drx_ldpc_mix_tune(drx_ldpc_mix* m, void* stream, float* ms_one_launch, float* ms_per_code)
{
    if (!m || !m->nframes) {
        set_error("drx_ldpc_mix_tune: no plan");
        return -1;
    }
    cudaStream_t s = stream ? (cudaStream_t)stream : m->capture;
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    float best = 0;
    int choice = DRX_TILING_ONE_LAUNCH;
    for (int t = DRX_TILING_ONE_LAUNCH; t <= DRX_TILING_ONE_LAUNCH_PAIR; t++) {
        m->tuned_ms[t] = 0;
        if (!m->exec[t])
            continue;
        float tmin = 1e30f;
        cudaGraphLaunch(m->exec[t], s); /* warm-up */
        for (int r = 0; r < 2; r++) {
            cudaEventRecord(a, s);
            cudaGraphLaunch(m->exec[t], s);
            cudaEventRecord(b, s);
            if (!cuda_check(cudaEventSynchronize(b), "drx_ldpc_mix_tune")) {
                cudaEventDestroy(a);
                cudaEventDestroy(b);
                return -1;
            }
            float ms = 0;
            cudaEventElapsedTime(&ms, a, b);
            tmin = std::min(tmin, ms);
        }
        m->tuned_ms[t] = tmin;
        if (t == DRX_TILING_ONE_LAUNCH || tmin < best) {
            best = tmin;
            choice = t;
        }
    }
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (ms_one_launch)
        *ms_one_launch = m->tuned_ms[DRX_TILING_ONE_LAUNCH];
    if (ms_per_code)
        *ms_per_code = m->tuned_ms[DRX_TILING_PER_CODE];
    m->tiling = choice;
    return choice;
}

float drx_ldpc_mix_tuned_ms(const drx_ldpc_mix* m, int tiling)
{
    if (!m || tiling < DRX_TILING_ONE_LAUNCH || tiling > DRX_TILING_ONE_LAUNCH_PAIR)
        return -1.0f;
    return m->exec[tiling] ? m->tuned_ms[tiling] : -1.0f;
}

}  // extern "C"
