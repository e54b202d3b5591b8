/*
 * The receiver's FEC stage on the GPU.
 *
 * drx_fec_decode_device: LDPC then BCH of device rows on one stream, the FEC
 * path of the reference's DVB-T2 receiver (libdvbrx/src/dvbt2.c:2386-2396:
 * drx_ldpc_decode on batches of drx_ldpc_lanes() blocks, then drx_bch_decode
 * of every block, also when the LDPC batch did not converge).
 *
 * drx_rxq: the LDPC stage of the reference's multi-threaded receiver
 * (libdvbrx/src/rxmt.c) as one queue in front of the GPU.  Frames arrive one
 * at a time with their code; as in batch_for / on_plframe
 * (rxmt.c:214-275), each code has at most one open batch, at most max_open
 * batches are open at once (a frame of another code sends the oldest), and a
 * batch is sent when it holds batch_frames frames, or when it has been open
 * longer than the latency bound (rxmt.c:476-480), or on a flush.  A sent
 * batch goes to the GPU on its code's stream: host-to-device copy, LDPC
 * decode (per-frame stopping, or the batch as one group: the reference's
 * drx_ldpc_decode on the batch, rxmt.c:514-536), BCH decode, results back
 * to page-locked memory.  Batches of different codes overlap on the GPU;
 * frames leave the queue in arrival order (the sequence numbers of
 * out_thread, rxmt.c:570-606), each as soon as its batch is done.
 */
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <chrono>
#include <deque>
#include <string>
#include <vector>

#include "../../include/dvbrx_b200.h"
#include "handle.h"

using drxg::cuda_check;
using drxg::set_error;

extern "C" int drx_fec_decode_device(drx_ldpc* d, drx_bch* b, const int8_t* llr, size_t llr_stride, uint8_t* cw,
                                     size_t cw_stride, int32_t* iters, uint8_t* ok, int32_t* bch_result,
                                     int nframes, int max_iter, int stop, void* stream)
{
    if (!d || !b) {
        set_error("drx_fec_decode_device: NULL handle");
        return -1;
    }
    if (nframes <= 0)
        return 0;
    /* one stream for both steps: the BCH decode reads what the LDPC decode wrote */
    void* s = stream ? stream : (void*)d->stream;
    if (drx_ldpc_decode_device(d, llr, llr_stride, cw, cw_stride, iters, ok, nframes, max_iter, stop, s))
        return -1;
    return drx_bch_decode_device(b, cw, cw_stride, bch_result, nframes, s);
}

namespace {

using Clock = std::chrono::steady_clock;

struct RxCode {
    drx_fec_params p{};
    std::string rate;
    drx_ldpc* ldpc = nullptr;
    drx_bch* bch = nullptr;
    cudaStream_t stream = nullptr; /* the code's batches run in order on it (its handles' scratch) */
    int N = 0, nbytes = 0;
};

struct RxBatch {
    int code = -1;
    int n = 0, emitted = 0;
    bool sent = false;
    Clock::time_point start;
    std::vector<uint64_t> fseq;
    int8_t* h_llr = nullptr;
    uint8_t* h_cw = nullptr;
    int32_t* h_it = nullptr;
    uint8_t* h_ok = nullptr;
    int32_t* h_bch = nullptr;
    int8_t* d_llr = nullptr;
    uint8_t* d_cw = nullptr;
    int32_t* d_it = nullptr;
    uint8_t* d_ok = nullptr;
    int32_t* d_bch = nullptr;
    cudaEvent_t done = nullptr;
};

constexpr int kMaxN = 64800;
constexpr int kMaxBytes = 64800 / 8;

}  // namespace

struct drx_rxq {
    int batch_frames = 64, max_open = 4, max_iter = 30, stop = 0, latency_ms = 0;
    std::vector<RxCode> codes;
    std::vector<RxBatch*> open;                 /* by age, oldest first */
    std::deque<std::pair<RxBatch*, int>> order; /* every queued frame, in arrival order */
    std::vector<RxBatch*> pool;                 /* batches not in use */
    std::vector<RxBatch*> all;
    uint64_t next_fseq = 0;
};

namespace {

void free_batch(RxBatch* b)
{
    cudaFreeHost(b->h_llr);
    cudaFreeHost(b->h_cw);
    cudaFreeHost(b->h_it);
    cudaFreeHost(b->h_ok);
    cudaFreeHost(b->h_bch);
    cudaFree(b->d_llr);
    cudaFree(b->d_cw);
    cudaFree(b->d_it);
    cudaFree(b->d_ok);
    cudaFree(b->d_bch);
    if (b->done)
        cudaEventDestroy(b->done);
    delete b;
}

RxBatch* new_batch(int frames)
{
    RxBatch* b = new RxBatch();
    const size_t F = (size_t)frames;
    b->fseq.resize(F);
    const bool ok = cuda_check(cudaMallocHost(&b->h_llr, F * kMaxN), "cudaMallocHost") &&
                    cuda_check(cudaMallocHost(&b->h_cw, F * kMaxBytes), "cudaMallocHost") &&
                    cuda_check(cudaMallocHost(&b->h_it, F * 4), "cudaMallocHost") &&
                    cuda_check(cudaMallocHost(&b->h_ok, F), "cudaMallocHost") &&
                    cuda_check(cudaMallocHost(&b->h_bch, F * 4), "cudaMallocHost") &&
                    cuda_check(drxg::dev_malloc(&b->d_llr, F * kMaxN), "cudaMalloc") &&
                    cuda_check(drxg::dev_malloc(&b->d_cw, F * kMaxBytes), "cudaMalloc") &&
                    cuda_check(drxg::dev_malloc(&b->d_it, F * 4), "cudaMalloc") &&
                    cuda_check(drxg::dev_malloc(&b->d_ok, F), "cudaMalloc") &&
                    cuda_check(drxg::dev_malloc(&b->d_bch, F * 4), "cudaMalloc") &&
                    cuda_check(cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming), "cudaEventCreate");
    if (!ok) {
        free_batch(b);
        return nullptr;
    }
    return b;
}

/* Queue a batch on its code's stream: copy in, LDPC, BCH, copy out. */
bool send_batch(drx_rxq* q, RxBatch* b)
{
    for (size_t i = 0; i < q->open.size(); i++)
        if (q->open[i] == b) {
            q->open.erase(q->open.begin() + (long)i);
            break;
        }
    const RxCode& c = q->codes[(size_t)b->code];
    const size_t n = (size_t)b->n, N = (size_t)c.N, nb = (size_t)c.nbytes;
    cudaStream_t s = c.stream;
    b->sent = true;
    /* on a failure the batch's frames are still popped (in order), with whatever the
     * failed step left; the push or pop that sent it returns -1 */
    return cuda_check(cudaMemcpyAsync(b->d_llr, b->h_llr, n * N, cudaMemcpyHostToDevice, s), "cudaMemcpyAsync") &&
           drx_fec_decode_device(c.ldpc, c.bch, b->d_llr, N, b->d_cw, nb, b->d_it, b->d_ok, b->d_bch, b->n,
                                 q->max_iter, q->stop ? b->n : 0, s) == 0 &&
           cuda_check(cudaMemcpyAsync(b->h_cw, b->d_cw, n * nb, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync") &&
           cuda_check(cudaMemcpyAsync(b->h_it, b->d_it, n * 4, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync") &&
           cuda_check(cudaMemcpyAsync(b->h_ok, b->d_ok, n, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync") &&
           cuda_check(cudaMemcpyAsync(b->h_bch, b->d_bch, n * 4, cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync") &&
           cuda_check(cudaEventRecord(b->done, s), "cudaEventRecord");
}

/* Batches open longer than the latency bound go out (rxmt.c:476-480). */
bool send_late(drx_rxq* q)
{
    if (q->latency_ms <= 0)
        return true;
    const Clock::time_point now = Clock::now();
    for (size_t i = 0; i < q->open.size();) {
        RxBatch* b = q->open[i];
        if (std::chrono::duration_cast<std::chrono::milliseconds>(now - b->start).count() > q->latency_ms) {
            if (!send_batch(q, b))
                return false;
        } else {
            i++;
        }
    }
    return true;
}

}  // namespace

extern "C" {

drx_rxq* drx_rxq_new(int ncodes, const drx_fec_params* params, const char* const* rates, int batch_frames,
                     int max_open, int max_iter, int stop, int max_latency_ms)
{
    if (ncodes < 1 || !params || !rates || batch_frames < 1 || max_open < 1 || (stop != 0 && stop != 1)) {
        set_error("drx_rxq_new: bad arguments");
        return nullptr;
    }
    if (stop == 1 && batch_frames > drx_ldpc_lanes()) {
        /* a group's CTAs wait for each other: the reference's batch of at most lanes frames */
        set_error("drx_rxq_new: group decoding takes batches of at most drx_ldpc_lanes() frames");
        return nullptr;
    }
    drx_rxq* q = new drx_rxq();
    q->batch_frames = batch_frames;
    q->max_open = max_open;
    q->max_iter = max_iter < 0 ? 0 : max_iter;
    q->stop = stop;
    q->latency_ms = max_latency_ms;
    for (int k = 0; k < ncodes; k++) {
        RxCode c;
        c.p = params[k];
        c.rate = rates[k] ? rates[k] : "";
        c.ldpc = drx_ldpc_new(&params[k], c.rate.c_str());
        c.bch = c.ldpc ? drx_bch_new(&params[k]) : nullptr;
        if (!c.ldpc || !c.bch || params[k].nldpc > kMaxN ||
            !cuda_check(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking), "cudaStreamCreate")) {
            drx_bch_free(c.bch);
            drx_ldpc_free(c.ldpc);
            q->codes.push_back(c); /* freed with the others */
            q->codes.back().ldpc = nullptr;
            q->codes.back().bch = nullptr;
            drx_rxq_free(q);
            return nullptr;
        }
        drx_ldpc_info info{};
        drx_ldpc_get_info(c.ldpc, &info);
        c.N = info.nldpc;
        c.nbytes = (info.kldpc + 7) / 8;
        q->codes.push_back(c);
    }
    return q;
}

void drx_rxq_free(drx_rxq* q)
{
    if (!q)
        return;
    for (RxCode& c : q->codes) {
        if (c.stream) {
            cudaStreamSynchronize(c.stream);
            cudaStreamDestroy(c.stream);
        }
        drx_bch_free(c.bch);
        drx_ldpc_free(c.ldpc);
    }
    for (RxBatch* b : q->all)
        free_batch(b);
    delete q;
}

int drx_rxq_push(drx_rxq* q, int code, const int8_t* llr, uint64_t* fseq)
{
    if (!q || !llr || code < 0 || code >= (int)q->codes.size()) {
        set_error("drx_rxq_push: bad arguments");
        return -1;
    }
    /* the open batch of this code, or a new one (the oldest goes out if
     * max_open are open: rxmt.c:214-225) */
    RxBatch* b = nullptr;
    for (RxBatch* o : q->open)
        if (o->code == code)
            b = o;
    if (!b) {
        if ((int)q->open.size() >= q->max_open && !send_batch(q, q->open[0]))
            return -1;
        if (!q->pool.empty()) {
            b = q->pool.back();
            q->pool.pop_back();
        } else {
            b = new_batch(q->batch_frames);
            if (!b)
                return -1;
            q->all.push_back(b);
        }
        b->code = code;
        b->n = b->emitted = 0;
        b->sent = false;
        b->start = Clock::now();
        q->open.push_back(b);
    }
    const RxCode& c = q->codes[(size_t)code];
    memcpy(b->h_llr + (size_t)b->n * (size_t)c.N, llr, (size_t)c.N);
    const uint64_t f = q->next_fseq++;
    b->fseq[(size_t)b->n] = f;
    q->order.emplace_back(b, b->n);
    b->n++;
    if (fseq)
        *fseq = f;
    if (b->n == q->batch_frames && !send_batch(q, b))
        return -1;
    return send_late(q) ? 0 : -1;
}

int drx_rxq_flush(drx_rxq* q)
{
    if (!q) {
        set_error("drx_rxq_flush: NULL queue");
        return -1;
    }
    while (!q->open.empty())
        if (!send_batch(q, q->open[0]))
            return -1;
    return 0;
}

int drx_rxq_pop(drx_rxq* q, int wait, uint64_t* fseq, int* code, uint8_t* cw, int32_t* iters, int32_t* ok,
                int32_t* bch_result)
{
    if (!q) {
        set_error("drx_rxq_pop: NULL queue");
        return -1;
    }
    if (!send_late(q))
        return -1;
    if (q->order.empty())
        return 0;
    RxBatch* b = q->order.front().first;
    const int i = q->order.front().second;
    if (!b->sent) {
        if (!wait)
            return 0;
        if (!send_batch(q, b)) /* the next frame waits in an open batch: send it */
            return -1;
    }
    if (wait) {
        if (!cuda_check(cudaEventSynchronize(b->done), "drx_rxq_pop"))
            return -1;
    } else {
        const cudaError_t e = cudaEventQuery(b->done);
        if (e == cudaErrorNotReady)
            return 0;
        if (!cuda_check(e, "drx_rxq_pop"))
            return -1;
    }
    const RxCode& c = q->codes[(size_t)b->code];
    if (fseq)
        *fseq = b->fseq[(size_t)i];
    if (code)
        *code = b->code;
    if (cw)
        memcpy(cw, b->h_cw + (size_t)i * (size_t)c.nbytes, (size_t)c.nbytes);
    if (iters)
        *iters = b->h_it[i];
    if (ok)
        *ok = b->h_ok[i];
    if (bch_result)
        *bch_result = b->h_bch[i];
    q->order.pop_front();
    if (++b->emitted == b->n)
        q->pool.push_back(b);
    return 1;
}

int drx_rxq_pending(const drx_rxq* q) { return q ? (int)q->order.size() : -1; }

}  // extern "C"
