/*
 * extern "C" entry points of libdvbrx_b200.so (declared in include/dvbrx_b200.h).
 *
 * A handle holds one compiled code (its tables in device memory), a CUDA
 * stream, the per-CTA message scratch, the group-barrier counters and the
 * pinned staging buffers of the host-pointer calls.
 */
#include <cuda_runtime.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/dvbrx_b200.h"
#include <math.h>

#include "channel.h"
#include "codes.h"
#include "codes_gen.h"
#include "handle.h"
#include "ldpc_device.h"

using namespace drxg;

namespace {

thread_local std::string g_err;

void set_err(const std::string& s) { g_err = s; }

bool cuda_ok(cudaError_t e, const char* what)
{
    if (e == cudaSuccess)
        return true;
    set_err(std::string(what) + ": " + cudaGetErrorString(e));
    return false;
}

constexpr int kLanes = 64;

}  // namespace


namespace {

void release_stage(drx_ldpc* d)
{
    cudaFreeHost(d->h_llr);
    cudaFreeHost(d->h_out);
    cudaFreeHost(d->h_it);
    cudaFreeHost(d->h_ok);
    cudaFree(d->d_llr);
    cudaFree(d->d_out);
    cudaFree(d->d_it);
    cudaFree(d->d_ok);
    d->h_llr = nullptr;
    d->h_out = nullptr;
    d->h_it = nullptr;
    d->h_ok = nullptr;
    d->d_llr = nullptr;
    d->d_out = nullptr;
    d->d_it = nullptr;
    d->d_ok = nullptr;
    d->stage_frames = 0;
}

bool ensure_stage(drx_ldpc* d, size_t nframes)
{
    if (d->stage_frames >= nframes)
        return true;
    cudaStreamSynchronize(d->stream);
    release_stage(d);
    const size_t N = d->code.N, nb = d->nbytes;
    if (!cuda_ok(cudaMallocHost(&d->h_llr, nframes * N), "cudaMallocHost") ||
        !cuda_ok(cudaMallocHost(&d->h_out, nframes * nb), "cudaMallocHost") ||
        !cuda_ok(cudaMallocHost(&d->h_it, nframes * 4), "cudaMallocHost") ||
        !cuda_ok(cudaMallocHost(&d->h_ok, nframes), "cudaMallocHost") ||
        !cuda_ok(drxg::dev_malloc(&d->d_llr, nframes * N), "cudaMalloc") ||
        !cuda_ok(drxg::dev_malloc(&d->d_out, nframes * nb), "cudaMalloc") ||
        !cuda_ok(drxg::dev_malloc(&d->d_it, nframes * 4), "cudaMalloc") ||
        !cuda_ok(drxg::dev_malloc(&d->d_ok, nframes), "cudaMalloc")) {
        release_stage(d);
        return false;
    }
    d->stage_frames = nframes;
    return true;
}

bool ensure_scratch(drx_ldpc* d, size_t need)
{
    if (d->msg_cap >= need)
        return true;
    cudaStreamSynchronize(d->stream);
    cudaFree(d->msg);
    d->msg = nullptr;
    d->msg_cap = 0;
    if (!cuda_ok(drxg::dev_malloc(&d->msg, need), "cudaMalloc(messages)"))
        return false;
    d->msg_cap = need;
    return true;
}

/* The frame-pair kernel decodes per-frame batches of codes it supports,
 * unless the handle is pinned to the one-frame kernel. */
bool use_pair(const drx_ldpc* d)
{
    if (d->variant == DRX_VARIANT_FRAME)
        return false;
    return d->pair_ctas_per_sm > 0;
}

bool ensure_msg(drx_ldpc* d, int grid)
{
    const size_t need = decode_msg_bytes(d->code.R, d->code.dclass) * (size_t)grid;
    if (d->msg_cap >= need)
        return true;
    cudaStreamSynchronize(d->stream);
    cudaFree(d->msg);
    d->msg = nullptr;
    d->msg_cap = 0;
    if (!cuda_ok(drxg::dev_malloc(&d->msg, need), "cudaMalloc(messages)"))
        return false;
    d->msg_cap = need;
    return true;
}

bool ensure_sync(drx_ldpc* d, size_t words)
{
    if (d->sync_cap >= words)
        return true;
    cudaStreamSynchronize(d->stream);
    cudaFree(d->sync);
    d->sync = nullptr;
    d->sync_cap = 0;
    if (!cuda_ok(drxg::dev_malloc(&d->sync, words * sizeof(unsigned)), "cudaMalloc(sync)"))
        return false;
    d->sync_cap = words;
    return true;
}

/* Upload a compiled code: DevCode, then its tables. */
bool upload_code(drx_ldpc* d)
{
    const Code& c = d->code;
    auto a16 = [](size_t v) { return (v + 15) & ~(size_t)15; };
    const size_t o_ent = a16(sizeof(DevCode));
    const size_t o_eoff = o_ent + a16(c.ent.size() * sizeof(int32_t));
    const size_t o_steps = o_eoff + a16(c.eoff.size() * sizeof(uint16_t));
    const size_t o_perm = o_steps + a16(c.steps.size() * sizeof(uint32_t));
    const size_t o_lmeta = o_perm + a16(c.perm.size() * sizeof(uint16_t));
    const size_t o_nlev = o_lmeta + a16(c.lmeta.size() * sizeof(uint64_t));
    const size_t total = o_nlev + a16(c.nlev.size());
    std::vector<char> host(total, 0);
    if (!cuda_ok(drxg::dev_malloc(&d->blob, total), "cudaMalloc(code)"))
        return false;
    char* base = (char*)d->blob;
    DevCode dc{};
    dc.N = c.N;
    dc.K = c.K;
    dc.R = c.R;
    dc.q = c.q;
    dc.kldpc = d->params.kldpc;
    dc.nbytes = d->nbytes;
    dc.nent = (int)c.ent.size() / 2;
    dc.nsteps = (int)c.steps.size();
    dc.dclass = c.dclass;
    dc.ent = (const int2*)(base + o_ent);
    dc.eoff = (const uint16_t*)(base + o_eoff);
    dc.steps = (const uint32_t*)(base + o_steps);
    dc.perm = (const uint16_t*)(base + o_perm);
    dc.lmeta = (const unsigned long long*)(base + o_lmeta);
    dc.nlev = (const uint8_t*)(base + o_nlev);
    memcpy(host.data(), &dc, sizeof(dc));
    memcpy(host.data() + o_lmeta, c.lmeta.data(), c.lmeta.size() * sizeof(uint64_t));
    memcpy(host.data() + o_nlev, c.nlev.data(), c.nlev.size());
    memcpy(host.data() + o_ent, c.ent.data(), c.ent.size() * sizeof(int32_t));
    memcpy(host.data() + o_eoff, c.eoff.data(), c.eoff.size() * sizeof(uint16_t));
    memcpy(host.data() + o_steps, c.steps.data(), c.steps.size() * sizeof(uint32_t));
    memcpy(host.data() + o_perm, c.perm.data(), c.perm.size() * sizeof(uint16_t));
    if (!cuda_ok(cudaMemcpy(d->blob, host.data(), total, cudaMemcpyHostToDevice), "cudaMemcpy(code)"))
        return false;
    d->dcode = (DevCode*)d->blob;
    d->smem = decode_smem_bytes(c.N, dc.nent, dc.nsteps, c.q);
    return true;
}

/* Per-frame extras of a launch: learned check nodes, a row list and a
 * frame count read on the device (nframes is then an upper bound). */
struct Extra {
    const uint32_t* learn = nullptr;
    const int8_t* learn_class = nullptr;
    int learn_iters = 0;
    const int32_t* rows = nullptr;
    const int* nframes_dev = nullptr;
    unsigned* work = nullptr; /* frame counter (default: the handle's) */
    void* msg = nullptr;      /* message scratch of the caller's, large enough (default: the handle's) */
};

/* Queue one decode of nframes device-resident frames. */
int enqueue(drx_ldpc* d, const int8_t* llr, size_t llr_stride, uint8_t* out, size_t out_stride,
            int32_t* iters, uint8_t* ok, int nframes, int max_iter, int stop, cudaStream_t s,
            const Extra* x = nullptr)
{
    if (nframes <= 0)
        return 0;
    if (max_iter < 0) /* the reference's loop runs no iteration then (ldpc.c:628) */
        max_iter = 0;
    if (stop < 0) {
        set_err("stop must be DRX_STOP_FRAME or a group size > 0");
        return -1;
    }
    if (llr_stride < (size_t)d->code.N || out_stride < (size_t)d->nbytes) {
        set_err("row stride below the frame size");
        return -1;
    }
    const int capacity = d->ctas_per_sm * d->sms;
    if (capacity <= 0) {
        set_err("decoder kernel cannot be resident on this device");
        return -1;
    }
    DecodeParams p{};
    p.code = d->dcode;
    p.llr = llr;
    p.llr_stride = llr_stride;
    p.out = out;
    p.out_stride = out_stride;
    p.iters = iters;
    p.ok = ok;
    p.nframes = nframes;
    p.max_iter = max_iter;
    p.err = d->err;
    p.wait_limit = d->wait_limit;
    p.skip_vote = d->test_skip_vote;
    if (x) {
        if (stop != 0) {
            set_err("learned check nodes and row lists need per-frame stopping");
            return -1;
        }
        p.learn = x->learn;
        p.learn_class = x->learn_class;
        p.learn_iters = x->learn_iters;
        p.rows = x->rows;
        p.nframes_dev = x->nframes_dev;
    }
    unsigned* work = x && x->work ? x->work : d->work;
    int grid;
    if (stop == 0 && use_pair(d)) {
        /* two frames per CTA */
        grid = std::min((nframes + 1) / 2, d->pair_ctas_per_sm * d->sms);
        p.group = 0;
        p.work = work;
        if (!cuda_ok(cudaMemsetAsync(work, 0, sizeof(unsigned), s), "cudaMemsetAsync"))
            return -1;
        const size_t slab = decode_pair_msg_bytes(d->code.R, d->pair_kid);
        if (!(x && x->msg) && !ensure_scratch(d, slab * (size_t)grid))
            return -1;
        p.msg = x && x->msg ? x->msg : d->msg;
        p.msg_stride = slab;
        return cuda_ok(launch_decode_pair(p, d->pair_kid, d->pair_smem, grid, s), "decoder launch") ? 0 : -1;
    }
    const int pair_capacity = d->pair_ctas_per_sm * d->sms;
    if (stop > 0 && use_pair(d) && (stop + 1) / 2 <= pair_capacity) {
        /* groups of G frames on teams of ceil(G / 2) co-resident CTAs */
        const int G = stop, M = (G + 1) / 2;
        const int ngroups = (nframes + G - 1) / G;
        const int nteams = std::min(ngroups, pair_capacity / M);
        const int per_team = (ngroups + nteams - 1) / nteams;
        const size_t words = 2 * (size_t)(max_iter + 1) * (size_t)nteams * per_team;
        if (!ensure_sync(d, words))
            return -1;
        if (!cuda_ok(cudaMemsetAsync(d->sync, 0, words * sizeof(unsigned), s), "cudaMemsetAsync"))
            return -1;
        grid = nteams * M;
        p.group = G;
        p.nteams = nteams;
        p.team_sync = d->sync;
        const size_t slab = decode_pair_msg_bytes(d->code.R, d->pair_kid);
        if (!ensure_scratch(d, slab * (size_t)grid))
            return -1;
        p.msg = d->msg;
        p.msg_stride = slab;
        return cuda_ok(launch_decode_pair(p, d->pair_kid, d->pair_smem, grid, s), "decoder launch") ? 0 : -1;
    }
    if (stop == 0) {
        grid = std::min(nframes, capacity);
        p.group = 0;
        p.work = work;
        if (!cuda_ok(cudaMemsetAsync(work, 0, sizeof(unsigned), s), "cudaMemsetAsync"))
            return -1;
    } else {
        const int G = stop;
        if (G > capacity) {
            set_err("group larger than the resident CTAs of this device");
            return -1;
        }
        const int ngroups = (nframes + G - 1) / G;
        const int nteams = std::min(ngroups, capacity / G);
        const int per_team = (ngroups + nteams - 1) / nteams;
        const size_t words = 2 * (size_t)(std::max(max_iter, 0) + 1) * (size_t)nteams * per_team;
        if (!ensure_sync(d, words))
            return -1;
        if (!cuda_ok(cudaMemsetAsync(d->sync, 0, words * sizeof(unsigned), s), "cudaMemsetAsync"))
            return -1;
        grid = nteams * G;
        p.group = G;
        p.nteams = nteams;
        p.team_sync = d->sync;
    }
    if (!(x && x->msg) && !ensure_msg(d, grid))
        return -1;
    p.msg = x && x->msg ? x->msg : d->msg;
    p.msg_stride = decode_msg_bytes(d->code.R, d->code.dclass);
    return cuda_ok(launch_decode(p, d->code.dclass, d->smem, grid, s), "decoder launch") ? 0 : -1;
}

/* Rows whose learned decode failed: appended to rows (count in *count,
 * zeroed by the caller), flagged in fallback (may be null). */
__global__ void k_fallback_rows(const uint8_t* __restrict__ ok, int n, int32_t* __restrict__ rows, int* count,
                                uint8_t* __restrict__ fallback)
{
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < n; f += gridDim.x * blockDim.x) {
        const bool fail = ok[f] == 0;
        if (fallback)
            fallback[f] = fail ? 1 : 0;
        if (fail)
            rows[atomicAdd(count, 1)] = f;
    }
}

/* Streams, events, frame counters of the pipelined host call. */
bool ensure_pipe(drx_ldpc* d)
{
    if (d->copy)
        return true;
    bool ok = cuda_ok(cudaStreamCreateWithFlags(&d->pipe[0], cudaStreamNonBlocking), "cudaStreamCreate") &&
              cuda_ok(cudaStreamCreateWithFlags(&d->pipe[1], cudaStreamNonBlocking), "cudaStreamCreate") &&
              cuda_ok(drxg::dev_malloc(&d->chunk_work, kMaxChunks * sizeof(unsigned)), "cudaMalloc");
    for (int k = 0; ok && k < kChunkEvents; k++)
        ok = cuda_ok(cudaEventCreateWithFlags(&d->chunk_ev[k], cudaEventDisableTiming), "cudaEventCreate");
    if (ok)
        ok = cuda_ok(cudaStreamCreateWithFlags(&d->copy, cudaStreamNonBlocking), "cudaStreamCreate");
    return ok;
}

/* Message scratch of the largest per-frame launch of this handle. */
size_t launch_msg_bytes(const drx_ldpc* d)
{
    size_t a = decode_msg_bytes(d->code.R, d->code.dclass) * (size_t)(d->ctas_per_sm * d->sms);
    if (d->pair_ctas_per_sm > 0)
        a = std::max(a, decode_pair_msg_bytes(d->code.R, d->pair_kid) * (size_t)(d->pair_ctas_per_sm * d->sms));
    return a;
}

bool ensure_msg2(drx_ldpc* d, size_t need)
{
    if (d->msg2_cap >= need)
        return true;
    cudaFree(d->msg2);
    d->msg2 = nullptr;
    d->msg2_cap = 0;
    if (!cuda_ok(drxg::dev_malloc(&d->msg2, need), "cudaMalloc(messages)"))
        return false;
    d->msg2_cap = need;
    return true;
}

/* Per-frame stopping on host rows, pipelined: the batch is cut into chunks;
 * chunk c is copied into pinned memory, sent to the device on the copy
 * stream, and decoded on decode stream c % 2 once its copy is done (its own
 * frame counter, the stream's own message slab), its results returned on
 * the same stream.  Copies of later chunks overlap earlier decodes, and the
 * CTAs of chunk c + 1 take the SMs that chunk c's tail leaves. */
/* memcpy on up to 8 host threads for large copies (the staging copies of a
 * host call run at the speed of one core otherwise) */
void par_memcpy(void* dst, const void* src, size_t n)
{
    const size_t kMin = (size_t)4 << 20;
    const unsigned hw = std::thread::hardware_concurrency();
    const int nt = (int)std::min<size_t>(std::min(8u, hw ? hw : 1u), n / kMin);
    if (nt <= 1) {
        memcpy(dst, src, n);
        return;
    }
    const size_t part = (n / nt + 63) & ~(size_t)63;
    std::vector<std::thread> th;
    for (int k = 1; k < nt; k++) {
        const size_t a = part * k;
        if (a >= n)
            break;
        const size_t len = std::min(part, n - a);
        th.emplace_back([=] { memcpy((char*)dst + a, (const char*)src + a, len); });
    }
    memcpy(dst, src, std::min(part, n));
    for (auto& t : th)
        t.join();
}

/* True if p is page-locked host memory (cudaMallocHost, cudaHostAlloc,
 * cudaHostRegister), which the copy engines read and write directly. */
bool host_pinned(const void* p)
{
    if (!p)
        return true;
    cudaPointerAttributes at{};
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError(); /* not a pointer the runtime knows: pageable */
        return false;
    }
    return at.type == cudaMemoryTypeHost;
}

/*
 * Host batch, pipelined: the batch goes in chunks, each staged into pinned
 * memory on the host (unless the caller's rows are pinned already: then the
 * copy engine reads them directly), copied in on the copy stream and decoded
 * on one of two alternating streams (each with its own message slab), so
 * that copies overlap decodes and a chunk's tail overlaps the next chunk.
 * The first chunk is one wave of the decoder (every CTA busy once), so that
 * the GPU starts early; chunks then double.  Each chunk's results are copied
 * back on its decode stream (into the caller's arrays if they are pinned)
 * and out of the staging memory while later chunks decode.
 */
int decode_host_pipelined(drx_ldpc* d, const int8_t* llr, uint8_t* out, int32_t* iters, uint8_t* ok, int nframes,
                          int max_iter)
{
    const size_t N = d->code.N, nb = d->nbytes;
    const size_t mb = launch_msg_bytes(d);
    if (!ensure_stage(d, nframes) || !ensure_pipe(d) || !ensure_scratch(d, mb) || !ensure_msg2(d, mb))
        return -1;
    /* chunk sizes: one wave, then doubling, at most kMaxChunks chunks */
    const int wave = use_pair(d) ? 2 * d->pair_ctas_per_sm * d->sms : d->ctas_per_sm * d->sms;
    std::vector<int> first, size;
    int f0 = 0, sz = std::max(2, wave & ~1);
    while (f0 < nframes) {
        const int left = kMaxChunks - (int)size.size();
        int n = std::min(sz, nframes - f0);
        if (left == 1)
            n = nframes - f0;
        else
            n = std::max(n, std::min(nframes - f0, (nframes - f0 + left - 1) / left));
        first.push_back(f0);
        size.push_back(n);
        f0 += n;
        if (size.size() > 1)
            sz *= 2;
    }
    const int nch = (int)size.size();
    cudaEvent_t* in_ev = d->chunk_ev;
    cudaEvent_t* out_ev = d->chunk_ev + kMaxChunks;
    cudaEvent_t start = d->chunk_ev[2 * kMaxChunks];
    /* work queued on the handle's stream goes first (it may use the scratch) */
    if (!cuda_ok(cudaEventRecord(start, d->stream), "cudaEventRecord") ||
        !cuda_ok(cudaStreamWaitEvent(d->copy, start, 0), "cudaStreamWaitEvent") ||
        !cuda_ok(cudaStreamWaitEvent(d->pipe[0], start, 0), "cudaStreamWaitEvent") ||
        !cuda_ok(cudaStreamWaitEvent(d->pipe[1], start, 0), "cudaStreamWaitEvent"))
        return -1;
    const bool in_pinned = host_pinned(llr);
    const bool out_pinned = host_pinned(out) && host_pinned(iters) && host_pinned(ok);
    const int8_t* h_in = in_pinned ? llr : d->h_llr;
    uint8_t* h_out = out_pinned ? out : d->h_out;
    int32_t* h_it = out_pinned ? iters : d->h_it;
    uint8_t* h_ok = out_pinned ? ok : d->h_ok;
    int rc = 0, queued = 0;
    for (int c = 0; c < nch && rc == 0; c++, queued++) {
        const size_t a = (size_t)first[c];
        const int n = size[c];
        if (!in_pinned)
            par_memcpy(d->h_llr + a * N, llr + a * N, (size_t)n * N);
        cudaStream_t ks = d->pipe[c & 1];
        Extra x;
        x.work = d->chunk_work + c;
        x.msg = (c & 1) ? d->msg2 : d->msg;
        bool good = cuda_ok(cudaMemcpyAsync(d->d_llr + a * N, h_in + a * N, (size_t)n * N, cudaMemcpyHostToDevice,
                                            d->copy),
                            "cudaMemcpyAsync") &&
                    cuda_ok(cudaEventRecord(in_ev[c], d->copy), "cudaEventRecord") &&
                    cuda_ok(cudaStreamWaitEvent(ks, in_ev[c], 0), "cudaStreamWaitEvent") &&
                    !enqueue(d, d->d_llr + a * N, N, d->d_out + a * nb, nb, d->d_it + a, d->d_ok + a, n, max_iter,
                             0, ks, &x) &&
                    cuda_ok(cudaMemcpyAsync(h_out + a * nb, d->d_out + a * nb, (size_t)n * nb,
                                            cudaMemcpyDeviceToHost, ks),
                            "cudaMemcpyAsync");
        if (good && h_it)
            good = cuda_ok(cudaMemcpyAsync(h_it + a, d->d_it + a, (size_t)n * 4, cudaMemcpyDeviceToHost, ks),
                           "cudaMemcpyAsync");
        if (good && h_ok)
            good = cuda_ok(cudaMemcpyAsync(h_ok + a, d->d_ok + a, (size_t)n, cudaMemcpyDeviceToHost, ks),
                           "cudaMemcpyAsync");
        if (!good || !cuda_ok(cudaEventRecord(out_ev[c], ks), "cudaEventRecord"))
            rc = -1;
    }
    /* results out of the staging memory, chunk by chunk, as they arrive */
    for (int c = 0; c < queued && rc == 0 && !out_pinned; c++) {
        if (!cuda_ok(cudaEventSynchronize(out_ev[c]), "decode")) {
            rc = -1;
            break;
        }
        const size_t a = (size_t)first[c];
        const int n = size[c];
        par_memcpy(out + a * nb, d->h_out + a * nb, (size_t)n * nb);
        if (iters)
            memcpy(iters + a, d->h_it + a, (size_t)n * 4);
        if (ok)
            memcpy(ok + a, d->h_ok + a, (size_t)n);
    }
    const bool s0 = cuda_ok(cudaStreamSynchronize(d->pipe[0]), "decode");
    const bool s1 = cuda_ok(cudaStreamSynchronize(d->pipe[1]), "decode");
    const bool s2 = cuda_ok(cudaStreamSynchronize(d->copy), "copy");
    return rc || !s0 || !s1 || !s2 ? -1 : 0;
}

bool ensure_fallback(drx_ldpc* d, size_t nframes)
{
    if (d->fb_cap >= nframes)
        return true;
    cudaStreamSynchronize(d->stream);
    cudaFree(d->fb_rows);
    cudaFree(d->fb_ok);
    d->fb_rows = nullptr;
    d->fb_ok = nullptr;
    d->fb_cap = 0;
    if (!cuda_ok(drxg::dev_malloc(&d->fb_rows, nframes * sizeof(int32_t) + 16), "cudaMalloc(fallback rows)") ||
        !cuda_ok(drxg::dev_malloc(&d->fb_ok, nframes), "cudaMalloc(fallback flags)"))
        return false;
    d->fb_cap = nframes;
    return true;
}

/* allocation-failure test hook: allocations left before one fails (-1: off) */
std::atomic<long> g_alloc_countdown{ -1 };

}  // namespace

namespace drxg {

bool alloc_fails_now()
{
    long v = g_alloc_countdown.load();
    while (v >= 0) {
        if (g_alloc_countdown.compare_exchange_weak(v, v - 1))
            return v == 0;
    }
    return false;
}

}  // namespace drxg

extern "C" {

const char* drx_ldpc_last_error(void) { return g_err.c_str(); }

void drx_test_fail_device_alloc(int after) { g_alloc_countdown.store(after < 0 ? -1 : after); }

int drx_ldpc_set_wait_limit(drx_ldpc* d, int polls)
{
    if (!d || polls < 0) {
        set_err("drx_ldpc_set_wait_limit: NULL handle or negative limit");
        return -1;
    }
    d->wait_limit = polls;
    return 0;
}

int drx_ldpc_test_skip_vote(drx_ldpc* d, int cta)
{
    if (!d || cta < -1) {
        set_err("drx_ldpc_test_skip_vote: NULL handle or CTA below -1");
        return -1;
    }
    d->test_skip_vote = cta + 1;
    return 0;
}

int drx_fec_lookup(int short_frame, const char* rate, drx_fec_params* p)
{
    if (!rate || !p)
        return -1;
    const cg_fec* rows = short_frame ? cg_fec_short : cg_fec_normal;
    const int n = short_frame ? (int)(sizeof(cg_fec_short) / sizeof(*cg_fec_short))
                              : (int)(sizeof(cg_fec_normal) / sizeof(*cg_fec_normal));
    for (int i = 0; i < n; i++) {
        if (strcmp(rows[i].rate, rate) == 0) {
            p->short_frame = short_frame;
            p->nldpc = short_frame ? 16200 : 64800;
            p->kldpc = rows[i].nbch;
            p->kbch = rows[i].kbch;
            p->t = rows[i].t;
            return 0;
        }
    }
    return -1;
}

int drx_ldpc_lanes(void) { return kLanes; }

drx_ldpc* drx_ldpc_new(const drx_fec_params* p, const char* rate)
{
    if (!p || !rate) {
        set_err("NULL argument");
        return nullptr;
    }
    const int table = find_table(p->short_frame, rate);
    if (table < 0) {
        set_err(std::string("no LDPC table for rate ") + rate);
        return nullptr;
    }
    drx_ldpc* d = new drx_ldpc();
    std::string err;
    if (!compile_code(table, &d->code, &err)) {
        set_err(err);
        delete d;
        return nullptr;
    }
    d->params = *p;
    if (d->params.kldpc <= 0 || d->params.kldpc > d->code.K)
        d->params.kldpc = d->code.K;
    d->nbytes = (d->params.kldpc + 7) / 8;
    if (!cuda_ok(cudaGetDevice(&d->device), "cudaGetDevice") ||
        !cuda_ok(cudaDeviceGetAttribute(&d->sms, cudaDevAttrMultiProcessorCount, d->device),
                 "cudaDeviceGetAttribute") ||
        !cuda_ok(cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking), "cudaStreamCreate") ||
        !upload_code(d) || !cuda_ok(drxg::dev_malloc(&d->work, 256), "cudaMalloc") ||
        !cuda_ok(drxg::dev_malloc(&d->err, sizeof(int)), "cudaMalloc") ||
        !cuda_ok(cudaMemset(d->err, 0, sizeof(int)), "cudaMemset")) {
        drx_ldpc_free(d);
        return nullptr;
    }
    d->ctas_per_sm = decode_ctas_per_sm(d->code.dclass, d->smem);
    d->pair_kid = pair_kernel_id(d->code);
    if (d->pair_kid >= 0) {
        auto smem_of = [&](int kid) {
            return decode_pair_smem_bytes(d->code.N, d->code.K, (int)d->code.ent.size() / 2,
                                          (int)d->code.steps.size(), d->code.q, kid);
        };
        d->pair_smem = smem_of(d->pair_kid);
        d->pair_ctas_per_sm = decode_pair_ctas_per_sm(d->pair_kid, d->pair_smem);
        /* a two-CTA twin when it makes more CTAs resident: all posteriors in
         * shared memory if they leave room, else the parity-out one */
        const int base = d->pair_kid;
        for (int pm = 1; pm <= 2; pm++) {
            const int tw = pair_kernel_twin(base, pm);
            if (tw < 0)
                continue;
            const size_t sm = smem_of(tw);
            const int n = decode_pair_ctas_per_sm(tw, sm);
            if (n > d->pair_ctas_per_sm) {
                d->pair_kid = tw;
                d->pair_smem = sm;
                d->pair_ctas_per_sm = n;
                break;
            }
        }
    }
    if (d->ctas_per_sm <= 0) {
        set_err("decoder kernel does not fit on this device");
        drx_ldpc_free(d);
        return nullptr;
    }
    return d;
}

void drx_ldpc_free(drx_ldpc* d)
{
    if (!d)
        return;
    if (d->stream)
        cudaStreamSynchronize(d->stream);
    release_stage(d);
    cudaFree(d->msg);
    cudaFree(d->msg2);
    cudaFree(d->chunk_work);
    for (int k = 0; k < kChunkEvents; k++)
        if (d->chunk_ev[k])
            cudaEventDestroy(d->chunk_ev[k]);
    for (int k = 0; k < 2; k++)
        if (d->pipe[k]) {
            cudaStreamSynchronize(d->pipe[k]);
            cudaStreamDestroy(d->pipe[k]);
        }
    if (d->copy) {
        cudaStreamSynchronize(d->copy);
        cudaStreamDestroy(d->copy);
    }
    cudaFree(d->fb_rows);
    cudaFree(d->fb_ok);
    cudaFree(d->learn);
    cudaFree(d->sync);
    cudaFree(d->work);
    cudaFree(d->err);
    cudaFree(d->blob);
    if (d->stream)
        cudaStreamDestroy(d->stream);
    delete d;
}

int drx_ldpc_get_info(const drx_ldpc* d, drx_ldpc_info* info)
{
    if (!d || !info)
        return -1;
    info->nldpc = d->code.N;
    info->kldpc = d->params.kldpc;
    info->K = d->code.K;
    info->R = d->code.R;
    info->q = d->code.q;
    info->edges = d->code.edges;
    info->steps = (int)d->code.steps.size();
    info->deg_max = d->code.deg_max;
    info->levelled = d->code.levelled ? 1 : 0;
    return 0;
}

int drx_ldpc_set_variant(drx_ldpc* d, int variant)
{
    if (!d || (variant != DRX_VARIANT_AUTO && variant != DRX_VARIANT_FRAME && variant != DRX_VARIANT_PAIR)) {
        set_err("unknown variant");
        return -1;
    }
    if (variant == DRX_VARIANT_PAIR && d->pair_ctas_per_sm <= 0) {
        set_err("the frame-pair kernel does not run this code");
        return -1;
    }
    d->variant = variant;
    return use_pair(d) ? DRX_VARIANT_PAIR : DRX_VARIANT_FRAME;
}

int drx_ldpc_code_info(int short_frame, const char* rate, drx_ldpc_info* info)
{
    if (!rate || !info)
        return -1;
    const int table = find_table(short_frame, rate);
    if (table < 0) {
        set_err(std::string("no LDPC table for rate ") + rate);
        return -1;
    }
    Code c;
    std::string err;
    if (!compile_code(table, &c, &err)) {
        set_err(err);
        return -1;
    }
    drx_fec_params p{};
    info->kldpc = drx_fec_lookup(short_frame, rate, &p) == 0 ? p.kldpc : c.K;
    info->nldpc = c.N;
    info->K = c.K;
    info->R = c.R;
    info->q = c.q;
    info->edges = c.edges;
    info->steps = (int)c.steps.size();
    info->deg_max = c.deg_max;
    info->levelled = c.levelled ? 1 : 0;
    return 0;
}

int drx_ldpc_device_error(drx_ldpc* d)
{
    if (!d)
        return -1;
    int v = 0;
    cudaStreamSynchronize(d->stream);
    cudaMemcpy(&v, d->err, sizeof(int), cudaMemcpyDeviceToHost);
    cudaMemset(d->err, 0, sizeof(int));
    return v;
}

int drx_ldpc_decode_device(drx_ldpc* d, const int8_t* llr, size_t llr_stride, uint8_t* out,
                           size_t out_stride, int32_t* iters, uint8_t* ok, int nframes,
                           int max_iter, int stop, void* stream)
{
    if (!d || (nframes > 0 && (!llr || !out))) {
        set_err("NULL argument");
        return -1;
    }
    return enqueue(d, llr, llr_stride, out, out_stride, iters, ok, nframes, max_iter, stop,
                   stream ? (cudaStream_t)stream : d->stream);
}

int drx_ldpc_set_learned(drx_ldpc* d, int iters, int nclass, const int8_t* class_of_degree,
                         const float* scale, const float* offset)
{
    if (!d) {
        set_err("NULL handle");
        return -1;
    }
    if (iters == 0) {
        d->learn_iters = 0;
        return 0;
    }
    if (iters < 0 || iters > kLearnMaxIters || nclass < 1 || nclass > kLearnClasses || !class_of_degree ||
        !scale || !offset) {
        set_err("learned table: 1..32 iterations, 1..8 classes and all arrays are required");
        return -1;
    }
    for (int k = 0; k <= 32; k++)
        if (class_of_degree[k] < 0 || class_of_degree[k] >= nclass) {
            set_err("learned table: class of a degree out of range");
            return -1;
        }
    std::vector<uint32_t> tab((size_t)iters * kLearnClasses, 0);
    for (int t = 0; t < iters; t++)
        for (int k = 0; k < nclass; k++) {
            const float b = scale[t * nclass + k], a = offset[t * nclass + k];
            if (!(b == b) || !(a == a)) {
                set_err("learned table: NaN parameter");
                return -1;
            }
            const long bq = std::min(std::max(lrintf(b * 256.0f), 0L), 65535L);
            const long aq = std::min(std::max(lrintf(a * 256.0f), -32768L), 32767L);
            tab[(size_t)t * kLearnClasses + k] = (uint32_t)bq | (uint32_t)(uint16_t)(int16_t)aq << 16;
        }
    if (!d->learn) {
        if (!cuda_ok(drxg::dev_malloc(&d->learn, sizeof(uint32_t) * kLearnMaxIters * kLearnClasses + 64),
                     "cudaMalloc(learned table)"))
            return -1;
    }
    cudaStreamSynchronize(d->stream);
    if (!cuda_ok(cudaMemcpy(d->learn, tab.data(), tab.size() * sizeof(uint32_t), cudaMemcpyHostToDevice),
                 "cudaMemcpy(learned table)") ||
        !cuda_ok(cudaMemcpy((char*)d->learn + sizeof(uint32_t) * kLearnMaxIters * kLearnClasses,
                            class_of_degree, 33, cudaMemcpyHostToDevice),
                 "cudaMemcpy(learned classes)"))
        return -1;
    d->learn_iters = iters;
    return 0;
}

int drx_ldpc_decode_learned_device(drx_ldpc* d, const int8_t* llr, size_t llr_stride, uint8_t* out,
                                   size_t out_stride, int32_t* iters, uint8_t* ok, uint8_t* fallback,
                                   int nframes, int learned_iters, int plain_max_iter, void* stream)
{
    if (!d || (nframes > 0 && (!llr || !out))) {
        set_err("NULL argument");
        return -1;
    }
    if (d->learn_iters <= 0) {
        set_err("no learned table on this handle (drx_ldpc_set_learned)");
        return -1;
    }
    if (nframes <= 0)
        return 0;
    cudaStream_t s = stream ? (cudaStream_t)stream : d->stream;
    if (!ensure_fallback(d, (size_t)nframes))
        return -1;
    uint8_t* okb = ok ? ok : d->fb_ok;
    Extra x;
    x.learn = d->learn;
    x.learn_class = (const int8_t*)((const char*)d->learn + sizeof(uint32_t) * kLearnMaxIters * kLearnClasses);
    x.learn_iters = d->learn_iters;
    if (enqueue(d, llr, llr_stride, out, out_stride, iters, okb, nframes, learned_iters, 0, s, &x))
        return -1;
    if (plain_max_iter <= 0) {
        if (fallback && !cuda_ok(cudaMemsetAsync(fallback, 0, (size_t)nframes, s), "cudaMemsetAsync"))
            return -1;
        return 0;
    }
    int* count = (int*)(d->fb_rows + d->fb_cap);
    if (!cuda_ok(cudaMemsetAsync(count, 0, sizeof(int), s), "cudaMemsetAsync"))
        return -1;
    const int blocks = std::min((nframes + 255) / 256, 4 * d->sms);
    k_fallback_rows<<<blocks, 256, 0, s>>>(okb, nframes, d->fb_rows, count, fallback);
    if (!cuda_ok(cudaGetLastError(), "fallback rows"))
        return -1;
    Extra y;
    y.rows = d->fb_rows;
    y.nframes_dev = count;
    return enqueue(d, llr, llr_stride, out, out_stride, iters, okb, nframes, plain_max_iter, 0, s, &y);
}

int drx_ldpc_decode_host(drx_ldpc* d, const int8_t* llr, uint8_t* out, int32_t* iters,
                         uint8_t* ok, int nframes, int max_iter, int stop)
{
    if (!d || (nframes > 0 && (!llr || !out))) {
        set_err("NULL argument");
        return -1;
    }
    if (nframes <= 0)
        return 0;
    if (stop == 0 && nframes >= 512)
        return decode_host_pipelined(d, llr, out, iters, ok, nframes, max_iter);
    const size_t N = d->code.N, nb = d->nbytes;
    cudaStream_t s = d->stream;
    if (!ensure_stage(d, nframes))
        return -1;
    memcpy(d->h_llr, llr, (size_t)nframes * N);
    if (!cuda_ok(cudaMemcpyAsync(d->d_llr, d->h_llr, (size_t)nframes * N, cudaMemcpyHostToDevice, s),
                 "cudaMemcpyAsync"))
        return -1;
    if (enqueue(d, d->d_llr, N, d->d_out, nb, d->d_it, d->d_ok, nframes, max_iter, stop, s))
        return -1;
    if (!cuda_ok(cudaMemcpyAsync(d->h_out, d->d_out, (size_t)nframes * nb, cudaMemcpyDeviceToHost, s),
                 "cudaMemcpyAsync") ||
        !cuda_ok(cudaMemcpyAsync(d->h_it, d->d_it, (size_t)nframes * 4, cudaMemcpyDeviceToHost, s),
                 "cudaMemcpyAsync") ||
        !cuda_ok(cudaMemcpyAsync(d->h_ok, d->d_ok, (size_t)nframes, cudaMemcpyDeviceToHost, s),
                 "cudaMemcpyAsync") ||
        !cuda_ok(cudaStreamSynchronize(s), "decode"))
        return -1;
    memcpy(out, d->h_out, (size_t)nframes * nb);
    if (iters)
        memcpy(iters, d->h_it, (size_t)nframes * 4);
    if (ok)
        memcpy(ok, d->h_ok, (size_t)nframes);
    return 0;
}

int drx_channel_generate(drx_ldpc* d, const char* constellation, const char* const_rate, int nframes,
                         float esn0_db, unsigned long long seed, int8_t* llr, size_t llr_stride,
                         void* llr_f16, size_t llr_f16_stride, uint8_t* info, size_t info_stride,
                         void* stream)
{
    if (!d || !constellation || !const_rate) {
        set_err("NULL argument");
        return -1;
    }
    if (nframes <= 0)
        return 0;
    const int short_frame = d->code.N == 16200 ? 1 : 0;
    const cg_const* row = nullptr;
    for (int i = 0; i < CG_NCONSTS; i++)
        if (!strcmp(cg_consts[i].name, constellation) && !strcmp(cg_consts[i].rate, const_rate) &&
            cg_consts[i].short_frame == short_frame)
            row = &cg_consts[i];
    if (!row) {
        set_err(std::string("no constellation ") + constellation + " " + const_rate);
        return -1;
    }
    if ((llr && llr_stride < (size_t)d->code.N) || (llr_f16 && llr_f16_stride < (size_t)d->code.N) ||
        (info && info_stride < (size_t)d->nbytes)) {
        set_err("row stride below the frame size");
        return -1;
    }
    ChannelParams p{};
    p.code = d->dcode;
    p.seed = seed;
    p.n0 = powf(10.0f, -esn0_db / 10.0f);
    p.bits = row->bits;
    p.qpsk = row->order[0] < 0;
    const int np = 1 << row->bits;
    double e = 0;
    for (int i = 0; i < np; i++)
        e += (double)row->points[2 * i] * row->points[2 * i] + (double)row->points[2 * i + 1] * row->points[2 * i + 1];
    const float g = (float)(1.0 / sqrt(e / np)); /* unit average energy, as demap.c:183-187 */
    for (int i = 0; i < np; i++) {
        p.re[i] = row->points[2 * i] * g;
        p.im[i] = row->points[2 * i + 1] * g;
        p.e[i] = p.re[i] * p.re[i] + p.im[i] * p.im[i];
    }
    for (int b = 0; b < 8; b++)
        p.order[b] = row->order[b] < 0 ? 0 : row->order[b];
    p.llr = llr;
    p.llr_stride = llr_stride;
    p.llr_f16 = (__half*)llr_f16;
    p.llr_f16_stride = llr_f16_stride;
    p.info = info;
    p.info_stride = info_stride;
    return cuda_ok(launch_channel(p, nframes, d->code.N, stream ? (cudaStream_t)stream : d->stream),
                   "channel launch") ? 0 : -1;
}

int drx_ldpc_decode(drx_ldpc* d, const int8_t* const* llr, uint8_t* const* out, int nframes,
                    int max_iter)
{
    if (!d) {
        set_err("NULL handle");
        return -1;
    }
    if (nframes > kLanes) /* ldpc.c:620-621 */
        return -1;
    if (nframes <= 0) /* every lane padded: the syndrome passes at once */
        return 0;
    if (!llr || !out) {
        set_err("NULL argument");
        return -1;
    }
    const size_t N = d->code.N, nb = d->nbytes;
    cudaStream_t s = d->stream;
    if (!ensure_stage(d, kLanes))
        return -1;
    for (int f = 0; f < nframes; f++)
        memcpy(d->h_llr + (size_t)f * N, llr[f], N);
    if (!cuda_ok(cudaMemcpyAsync(d->d_llr, d->h_llr, (size_t)nframes * N, cudaMemcpyHostToDevice, s),
                 "cudaMemcpyAsync"))
        return -1;
    if (enqueue(d, d->d_llr, N, d->d_out, nb, d->d_it, d->d_ok, nframes, max_iter, nframes, s))
        return -1;
    if (!cuda_ok(cudaMemcpyAsync(d->h_out, d->d_out, (size_t)nframes * nb, cudaMemcpyDeviceToHost, s),
                 "cudaMemcpyAsync") ||
        !cuda_ok(cudaMemcpyAsync(d->h_it, d->d_it, (size_t)nframes * 4, cudaMemcpyDeviceToHost, s),
                 "cudaMemcpyAsync") ||
        !cuda_ok(cudaMemcpyAsync(d->h_ok, d->d_ok, (size_t)nframes, cudaMemcpyDeviceToHost, s),
                 "cudaMemcpyAsync") ||
        !cuda_ok(cudaStreamSynchronize(s), "decode"))
        return -1;
    for (int f = 0; f < nframes; f++)
        memcpy(out[f], d->h_out + (size_t)f * nb, nb);
    int all = 1;
    for (int f = 0; f < nframes; f++)
        all &= d->h_ok[f];
    return all ? d->h_it[0] : -1;
}

}  // extern "C"

namespace drxg {

/* Read-only view of a handle for the allocation-free entry point (noalloc.cu). */
const DevCode* handle_code(const drx_ldpc* d, int* R, int* dclass, int* N, int* nbytes, int* capacity,
                           size_t* smem, cudaStream_t* stream)
{
    *R = d->code.R;
    *dclass = d->code.dclass;
    *N = d->code.N;
    *nbytes = d->nbytes;
    *capacity = d->ctas_per_sm * d->sms;
    *smem = d->smem;
    *stream = d->stream;
    return d->dcode;
}

/* The frame-pair kernel of a handle's per-frame calls (-1: the one-frame
 * kernel), its dynamic shared memory and resident CTAs. */
int handle_pair(const drx_ldpc* d, size_t* smem, int* capacity)
{
    if (!use_pair(d))
        return -1;
    *smem = d->pair_smem;
    *capacity = d->pair_ctas_per_sm * d->sms;
    return d->pair_kid;
}

void handle_set_error(const char* msg) { set_err(msg); }

}  // namespace drxg

namespace drxg {

void set_error(const std::string& s) { set_err(s); }
bool cuda_check(cudaError_t e, const char* what) { return cuda_ok(e, what); }

}  // namespace drxg
