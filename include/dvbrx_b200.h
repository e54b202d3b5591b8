/*
 * dvbrx_b200: DVB-S2 / S2X / T2 LDPC decoding on an NVIDIA B200 (sm_100a).
 *
 * C ABI of libdvbrx_b200.so.  The first five entry points are the drop-in
 * for the reference receiver's decoder (TrusterBSW/DVB-Rx, libdvbrx): same
 * names, same argument meaning, same return values.  A program built against
 * libdvbrx's ldpc.h and fec.h links against this library unchanged.  The
 * rest are additions for batches that do not fit the reference's 64-lane
 * call: device-resident batches, mixed-code batches and the learned decoder.
 *
 * Plain pointers and sizes only; `stream` arguments are cudaStream_t values
 * passed as void*.  NULL means the handle's own stream; pass
 * cudaStreamLegacy ((void*)1) for the legacy default stream.
 */
#ifndef DVBRX_B200_H
#define DVBRX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- drop-in: reference libdvbrx/include/dvbrx/fec.h, ldpc.h ------------ */

/* Same layout as the reference's drx_fec_params (libdvbrx/include/dvbrx/fec.h:13-19). */
#ifndef DVBRX_FEC_H
typedef struct {
    int short_frame; /* 0: normal (64800 bits), 1: short (16200 bits) */
    int nldpc;       /* LDPC codeword length */
    int kldpc;       /* = nbch */
    int kbch;        /* BBFRAME length */
    int t;           /* BCH error-correcting capability */
} drx_fec_params;
#endif

typedef struct drx_ldpc drx_ldpc;

/* Replaces drx_fec_lookup (libdvbrx/include/dvbrx/fec.h:25, libdvbrx/src/bch.c:25-41):
 * FEC parameters of a rate string ("3_4", "13_45", "1_5_VLSNR_SF2", ...).
 * Returns 0 on success, -1 for an unknown rate. */
int drx_fec_lookup(int short_frame, const char* rate, drx_fec_params* p);

/* Replaces drx_ldpc_lanes (libdvbrx/include/dvbrx/ldpc.h:17, ldpc.c:186): the most
 * frames one drx_ldpc_decode call takes.  64, the size callers give their
 * pointer arrays (libdvbrx/src/rx.c:14, rxmt.c:23). */
int drx_ldpc_lanes(void);

/* Replaces drx_ldpc_new (libdvbrx/include/dvbrx/ldpc.h:20, ldpc.c:199-260).  Returns
 * NULL for an unknown rate or when no CUDA device or memory is available
 * (drx_ldpc_last_error() says which).  The handle owns its GPU memory and
 * stream; like the reference's, it is not thread-safe. */
drx_ldpc* drx_ldpc_new(const drx_fec_params* p, const char* rate);

/* Replaces drx_ldpc_free (libdvbrx/include/dvbrx/ldpc.h:21, ldpc.c:262-273); NULL-safe. */
void drx_ldpc_free(drx_ldpc* d);

/* Replaces drx_ldpc_decode (libdvbrx/include/dvbrx/ldpc.h:32-36, ldpc.c:614-638).
 * llr[f]: nldpc int8 LLRs of frame f (host memory, positive for a 0 bit);
 * out[f]: receives ceil(kldpc / 8) bytes of hard information bits, MSB first.
 * The frames are decoded together with the reference's semantics: they
 * iterate until all pass the syndrome check or max_iter is reached.  Returns
 * the iterations run, or -1 if some frame still fails (hard bits are written
 * either way), or if nframes > drx_ldpc_lanes().  Synchronous. */
int drx_ldpc_decode(drx_ldpc* d, const int8_t* const* llr, uint8_t* const* out, int nframes,
                    int max_iter);

/* ---- additions ---------------------------------------------------------- */

/* Message of the last failure in this thread ("" if none). */
const char* drx_ldpc_last_error(void);

/* Code geometry of a handle. */
typedef struct {
    int nldpc, kldpc, K, R, q;
    int edges;    /* links of the Tanner graph */
    int steps;    /* layer steps per iteration (wavefront levels) */
    int deg_max;  /* largest check degree */
    int levelled; /* some layer needs more than one step */
} drx_ldpc_info;
int drx_ldpc_get_info(const drx_ldpc* d, drx_ldpc_info* info);

/* The same geometry for a rate, computed on the host (no device needed);
 * kldpc is taken from the BCH table, or K for codes without one.
 * Returns 0, or -1 for an unknown rate. */
int drx_ldpc_code_info(int short_frame, const char* rate, drx_ldpc_info* info);

/* Stopping rule of the batch calls: DRX_STOP_FRAME stops every frame on its
 * own (its iteration count and flag are those of a one-frame
 * drx_ldpc_decode call); a value G > 0 stops groups of G consecutive
 * frames together, as a drx_ldpc_decode call with those G frames would. */
#define DRX_STOP_FRAME 0

/* Decode nframes frames already in device memory, asynchronously on
 * `stream`.  llr: frame f at llr + f * llr_stride (nldpc bytes used);
 * out: frame f at out + f * out_stride (ceil(kldpc/8) bytes); iters, ok:
 * nframes entries each, or NULL.  Returns 0 if the work was queued. */
int drx_ldpc_decode_device(drx_ldpc* d, const int8_t* llr, size_t llr_stride, uint8_t* out,
                           size_t out_stride, int32_t* iters, uint8_t* ok, int nframes,
                           int max_iter, int stop, void* stream);

/* No counterpart in the reference.  drx_ldpc_decode_device with per-frame
 * stopping for callers that must not allocate GPU memory on the decode path
 * (a real-time receiver thread, where cudaMalloc/cudaFree can stall on a
 * device-wide synchronisation; a program whose GPU memory belongs to
 * another allocator): the call allocates nothing.  Its scratch is a 16 MiB
 * array compiled into the library, held by every GPU that loads it until
 * exit.  It runs the kernel drx_ldpc_decode_device runs for the handle
 * (the frame-pair kernel, or the one-frame kernel where the handle is
 * pinned to it), on at most (16 MiB - 256) / slab CTAs, the slab being the
 * kernel's message scratch per CTA: 64 frame-pair CTAs for normal 3/5
 * (against 296 in the regular call), 233 for short 1/2; a code whose slab
 * would not fit is rejected with an error.  Large batches therefore decode
 * more slowly than through drx_ldpc_decode_device.  All calls share that
 * array: calls whose kernels overlap on the GPU race and must be
 * serialised by the caller.  The first call on a device looks up the
 * array's device address (set-up, which can load the library's device
 * code and allocate): make one call with nframes = 0 on every device at
 * initialisation, before any stream capture; it decodes nothing.  The
 * handle is made by drx_ldpc_new beforehand.  Returns 0 if the work was
 * queued. */
int drx_ldpc_decode_device_noalloc(drx_ldpc* d, const int8_t* llr, size_t llr_stride, uint8_t* out,
                                   size_t out_stride, int32_t* iters, uint8_t* ok, int nframes,
                                   int max_iter, void* stream);

/* The same with host buffers (contiguous rows), synchronous: stages through
 * pinned memory and returns 0 when the results are in place. */
int drx_ldpc_decode_host(drx_ldpc* d, const int8_t* llr, uint8_t* out, int32_t* iters,
                         uint8_t* ok, int nframes, int max_iter, int stop);

/* Seeded synthetic frames of the handle's code, in device memory: random
 * information bits (Philox4x32-10 keyed by seed and frame index), the DVB-S2
 * encoder, the bit interleaver and constellation of the MODCOD
 * (constellation "QPSK" / "8PSK" / "16APSK" / ..., const_rate the rate row
 * of that constellation table), complex AWGN at esn0_db and the max-log
 * demapper with the reference receiver's int8 scale (2 x LLR, saturated to
 * +-127, libdvbrx/src/demap.c:491-533).  Any of llr (int8 rows), llr_f16
 * (IEEE half rows of the unquantised values) and info (packed information
 * bits, kldpc bits MSB first) may be NULL.  Asynchronous on `stream`. */
int drx_channel_generate(drx_ldpc* d, const char* constellation, const char* const_rate, int nframes,
                         float esn0_db, unsigned long long seed, int8_t* llr, size_t llr_stride,
                         void* llr_f16, size_t llr_f16_stride, uint8_t* info, size_t info_stride,
                         void* stream);

/* Kernel of the per-frame batch calls: DRX_VARIANT_AUTO (the default) runs
 * the frame-pair kernel (two frames per CTA, 16x2 SIMD), which covers every
 * code; DRX_VARIANT_FRAME pins the one-frame kernel.  Both give identical
 * results.  Returns the
 * variant per-frame batches will now run (DRX_VARIANT_FRAME or
 * DRX_VARIANT_PAIR), or -1. */
#define DRX_VARIANT_AUTO 0
#define DRX_VARIANT_FRAME 1
#define DRX_VARIANT_PAIR 2
int drx_ldpc_set_variant(drx_ldpc* d, int variant);

/* New: how long a group barrier of this handle's group-stopping launches
 * (drx_ldpc_decode, and stop > 0) waits for the other CTAs of its team, in
 * polls about 200 ns apart; 0 restores the default (4,194,304 polls, about
 * a second).  A barrier that gives up ends its group's decode with the
 * frames flagged as failed and sets the device error word to 2
 * (drx_ldpc_device_error).  Returns 0, or -1. */
int drx_ldpc_set_wait_limit(drx_ldpc* d, int polls);

/* Testing hook: in this handle's later group-stopping launches, CTA `cta`
 * never arrives at its team's barriers, so that the other members' waits
 * run out (the time-out path of the group barrier); -1 turns it off.
 * Returns 0, or -1. */
int drx_ldpc_test_skip_vote(drx_ldpc* d, int cta);

/* Testing hook: after `after` more device allocations by this library (all
 * threads), the next one fails as an out-of-memory cudaMalloc would, once;
 * -1 turns it off.  The failing call reports the error as every other
 * allocation failure does (NULL from drx_ldpc_new, -1 from a decode call,
 * drx_ldpc_last_error()). */
void drx_test_fail_device_alloc(int after);

/* ---- mixed batches: several codes (MODCODs, normal and short) at once ---- */

typedef struct drx_ldpc_mix drx_ldpc_mix;

/* A set of ncodes codes (params[c], rates[c]); code index c refers to the
 * c-th.  NULL on failure (drx_ldpc_last_error()). */
drx_ldpc_mix* drx_ldpc_mix_new(int ncodes, const drx_fec_params* params, const char* const* rates);
void drx_ldpc_mix_free(drx_ldpc_mix* m);

/* Plan a device batch of nframes rows: row f holds a frame of code code[f]
 * (host array) at llr + f * llr_stride, its bits go to out + f * out_stride,
 * its iterations and flag to iters[f] and ok[f] (device; may be NULL).
 * Strides must fit the largest code of the set.  Per-frame stopping.  The
 * plan is captured as CUDA graphs, one per tiling, replayed by
 * drx_ldpc_mix_run on whatever the buffers hold at that time. */
int drx_ldpc_mix_plan(drx_ldpc_mix* m, int nframes, const int32_t* code, const int8_t* llr, size_t llr_stride,
                      uint8_t* out, size_t out_stride, int32_t* iters, uint8_t* ok, int max_iter);

/* No counterpart in the reference.  The learned table of code index
 * code_index (drx_ldpc_set_learned on that code's handle). */
int drx_ldpc_mix_set_learned(drx_ldpc_mix* m, int code_index, int iters, int nclass, const int8_t* class_of_degree,
                             const float* scale, const float* offset);

/* No counterpart in the reference.  As drx_ldpc_mix_plan, for the learned
 * decode with the plain decoder as fallback: every frame runs its code's
 * learned table (at most learned_iters iterations, in the planned tiling);
 * the rows whose syndrome still fails are then gathered on the device, in
 * processing order, and decoded again from their LLRs by the plain decoder
 * in one launch (at most plain_max_iter iterations; none if <= 0), all in
 * the same CUDA graph.  fallback (device, nframes bytes, or NULL): 1 for
 * the re-decoded rows.  Every code of the batch needs a learned table. */
int drx_ldpc_mix_plan_learned(drx_ldpc_mix* m, int nframes, const int32_t* code, const int8_t* llr,
                              size_t llr_stride, uint8_t* out, size_t out_stride, int32_t* iters, uint8_t* ok,
                              uint8_t* fallback, int learned_iters, int plain_max_iter);

/* Tilings of a mixed batch (identical results): one persistent launch over
 * all frames, one frame per CTA; one persistent launch per code with the
 * code's own kernel (two frames per CTA where the frame-pair kernel
 * applies) on concurrent graph branches; or one persistent launch over all
 * frames with two frames per CTA, each CTA running one code at a time with
 * that code's frame-pair kernel shape and moving to the code with the most
 * work left when its code runs out (plain plans whose codes are DVB-S2
 * codes).  drx_ldpc_mix_set_tiling returns -1 for a tiling the plan lacks. */
#define DRX_TILING_ONE_LAUNCH 1
#define DRX_TILING_PER_CODE 2
#define DRX_TILING_ONE_LAUNCH_PAIR 3
int drx_ldpc_mix_set_tiling(drx_ldpc_mix* m, int tiling);

/* Autotuner: decodes the planned batch with each tiling the plan has
 * (twice, after a warm-up), keeps the fastest and returns it; the times of
 * the first two tilings in ms if non-NULL (drx_ldpc_mix_tuned_ms gives
 * every tiling's).  Synchronous. */
int drx_ldpc_mix_tune(drx_ldpc_mix* m, void* stream, float* ms_one_launch, float* ms_per_code);

/* The autotuner's time of a tiling in ms, -1 if the plan lacks it. */
float drx_ldpc_mix_tuned_ms(const drx_ldpc_mix* m, int tiling);

/* Launch the plan's graph (the tuned or set tiling) on `stream`. */
int drx_ldpc_mix_run(drx_ldpc_mix* m, void* stream);

/* ---- learned (neural offset / scaled) min-sum: training -------------------
 *
 * The plain decoder's layered schedule with the check node's offset 1
 * replaced by mag = max(beta[t][k] * min(min_other, 127) - alpha[t][k], 0)
 * for iteration t and check-degree class k (class_of_degree[D], D = 0..32),
 * with the int8 decoder's saturations, in fp32 on the int8 scale (2 x LLR).
 * Loss: sum over iterations and information bits of the binary
 * cross-entropy softplus(-(1 - 2 b) P / 2) of the posterior P after each
 * iteration.  Parameters are FP16 (iters x nclass), inputs FP16 LLRs
 * (unquantised, 2 x LLR), targets the packed information bits.  The caller
 * owns all memory; nothing is allocated. */
size_t drx_learned_workspace_bytes(const drx_ldpc* d, int nframes, int iters, int train);

/* Forward over nframes frames; loss[t] (device, zeroed by the caller)
 * receives the BCE sum after iteration t; post (device, optional) the final
 * posteriors of the kldpc information bits.  With train != 0 the
 * workspace keeps one checkpoint per iteration for drx_learned_backward. */
int drx_learned_forward(drx_ldpc* d, int nframes, const void* llr_f16, size_t llr_stride, const uint8_t* bits,
                        size_t bits_stride, int iters, const void* beta_f16, const void* alpha_f16, int nclass,
                        const int8_t* class_of_degree, float* loss, float* post, void* workspace,
                        size_t workspace_bytes, int train, void* stream);

/* Backward of a training forward with the same arguments and workspace:
 * adds to dbeta and dalpha (device fp32, iters x nclass) the gradient of
 * loss_scale x (sum over t of w[t] x the BCE sum of iteration t), with
 * w = iter_weights (device float[iters]) or all ones if NULL.
 * loss_scratch: device float[iters] the re-run forward writes into. */
int drx_learned_backward(drx_ldpc* d, int nframes, const void* llr_f16, size_t llr_stride, const uint8_t* bits,
                         size_t bits_stride, int iters, const void* beta_f16, const void* alpha_f16, int nclass,
                         const int8_t* class_of_degree, float loss_scale, const float* iter_weights,
                         float* dbeta, float* dalpha, float* loss_scratch, void* workspace,
                         size_t workspace_bytes, void* stream);

/* ---- learned min-sum: int8 inference --------------------------------------
 *
 * No counterpart in the reference (its decoder has only the offset 1).
 * The trained scale and offset tables (iters x nclass floats, row t for
 * iteration t, as trained with drx_learned_*) are rounded to Q8 and the int8
 * decoders use, for a node of degree class k in iteration t (rows past the
 * last repeat it),
 *     mag = max((scale_q * m - offset_q + 128) >> 8, 0),  m = min(minimum, 127),
 * with scale_q = round(256 scale) in [0, 65535] and offset_q =
 * round(256 offset) in [-32768, 32767]; messages and posteriors stay int8
 * exactly as in the plain decoder.  Scale 1 and offset 1 give the plain
 * decoder bit for bit.  iters = 0 removes the table.  1 <= iters <= 32,
 * 1 <= nclass <= 8.  Synchronous; returns 0 or -1. */
int drx_ldpc_set_learned(drx_ldpc* d, int iters, int nclass, const int8_t* class_of_degree,
                         const float* scale, const float* offset);

/* The learned decode with the plain decoder as fallback, on device-resident
 * frames (arguments as drx_ldpc_decode_device, per-frame stopping): every
 * frame is decoded with the handle's learned table for at most
 * learned_iters iterations; with plain_max_iter > 0, the frames whose
 * syndrome still fails are decoded again from their LLRs by the plain
 * decoder (at most plain_max_iter iterations) and their bits, iterations
 * and flags replace the learned ones.  fallback (nframes bytes, or NULL)
 * receives 1 for the re-decoded frames.  The failing rows are gathered on
 * the device, so the call never waits for the GPU.  Returns 0 if the work
 * was queued. */
int drx_ldpc_decode_learned_device(drx_ldpc* d, const int8_t* llr, size_t llr_stride, uint8_t* out,
                                   size_t out_stride, int32_t* iters, uint8_t* ok, uint8_t* fallback,
                                   int nframes, int learned_iters, int plain_max_iter, void* stream);

/* The decoding schedule of a code, computed on the host: the number of
 * steps and the largest check degree; for every check (layer-order index
 * 360 i + j) its step (check_step[R]) and its links (links[R][deg_max]:
 * parity bit, previous parity bit or -1, information bits, -1 padding) as
 * codeword bit indexes (parity bit of check q j + i at K + q j + i).
 * Either array may be NULL. */
int drx_ldpc_schedule(int short_frame, const char* rate, int* nsteps, int* deg_max, int32_t* check_step,
                      int32_t* links);

/* ---- BCH outer code (reference libdvbrx/include/dvbrx/fec.h:27-37) ---------
 *
 * The DVB-S2 BCH decoder on the GPU, with the reference's results
 * (libdvbrx/src/bch.c:106-290): fed by the LDPC decoder's hard bits (kldpc =
 * nbch bits, MSB first; the first kbch bits are the BBFRAME). */
typedef struct drx_bch drx_bch;

/* Replaces drx_bch_new (fec.h:29, bch.c:106-172): the code of p (normal
 * frames over GF(2^16), short over GF(2^14), t from p).  NULL on failure. */
drx_bch* drx_bch_new(const drx_fec_params* p);

/* Replaces drx_bch_free (fec.h:30, bch.c:174-181); NULL-safe. */
void drx_bch_free(drx_bch* b);

/* Replaces drx_bch_decode (fec.h:31-37, bch.c:189-290): decode one codeword
 * in host memory in place.  Returns the number of corrected bits, or -1 if
 * it is uncorrectable (left untouched).  Synchronous. */
int drx_bch_decode(drx_bch* b, uint8_t* cw);

/* No counterpart in the reference (its decoder takes one word per call).
 * Decode nframes device-resident codewords in place (row f at cw + f *
 * stride) asynchronously on `stream`, straight after the LDPC decode of the
 * same rows: result[f] (device) receives what drx_bch_decode returns.
 * Returns 0 if the work was queued. */
int drx_bch_decode_device(drx_bch* b, uint8_t* cw, size_t stride, int32_t* result, int nframes, void* stream);

/* No counterpart in the reference (the transmitter side, for test and
 * benchmark frames): encode nframes device rows in place, the kbch message
 * bits of each row followed by its nbch - kbch parity bits.  Asynchronous. */
int drx_bch_encode_device(drx_bch* b, uint8_t* cw, size_t stride, int nframes, void* stream);

/* ---- the receiver's FEC stage on the GPU ---- */

/* New: the FEC chain on device rows, on one stream: LDPC decode of nframes
 * frames into cw (kldpc bits, MSB first, frame f at cw + f * cw_stride;
 * iters and ok as drx_ldpc_decode_device), then BCH decode of every
 * codeword in place, bch_result[f] = corrected bits or -1.  The BCH decode
 * runs whatever the LDPC outcome, as the reference's receivers do: the
 * DVB-T2 FEC path (libdvbrx/src/dvbt2.c:2386-2396, drx_ldpc_decode on
 * batches of drx_ldpc_lanes() blocks, so stop = 64 reproduces it, then
 * drx_bch_decode per block) and the DVB-S2 output thread
 * (libdvbrx/src/rxmt.c:547-552).  b must be the BCH code of d's FEC
 * parameters.  Asynchronous on `stream` (NULL: d's stream).  Returns 0 if
 * the work was queued. */
int drx_fec_decode_device(drx_ldpc* d, drx_bch* b, const int8_t* llr, size_t llr_stride, uint8_t* cw,
                          size_t cw_stride, int32_t* iters, uint8_t* ok, int32_t* bch_result, int nframes,
                          int max_iter, int stop, void* stream);

/* New: a receiver's frame queue in front of the GPU, replacing the LDPC
 * worker pool and output ordering of the reference's multi-threaded
 * receiver (libdvbrx/src/rxmt.c:214-275, 476-480, 514-536, 570-606).
 * Frames are pushed one at a time with the index of their code (codes
 * given at creation: params[c], rates[c]).  Each code has at most one open
 * batch and at most max_open batches are open (a frame of another code
 * sends the oldest, as batch_for does); a batch is sent when it holds
 * batch_frames frames, when it has been open longer than max_latency_ms
 * (0: no bound), on drx_rxq_flush, or when drx_rxq_pop waits for one of
 * its frames.  A sent batch is decoded on the GPU on its code's stream
 * (copy in, drx_fec_decode_device, copy out); stop 0 stops each frame on
 * its own, stop 1 decodes the batch as one group (the reference's
 * drx_ldpc_decode on the batch; batch_frames at most drx_ldpc_lanes()).  Batches of different codes overlap on the
 * GPU.  Frames leave in arrival order (sequence numbers 0, 1, 2, ...).  Like
 * a decoder handle, a queue is used from one host thread at a time. */
typedef struct drx_rxq drx_rxq;
drx_rxq* drx_rxq_new(int ncodes, const drx_fec_params* params, const char* const* rates, int batch_frames,
                     int max_open, int max_iter, int stop, int max_latency_ms);
void drx_rxq_free(drx_rxq* q);

/* Queue frame llr (host, nldpc int8 of code `code`); *fseq (may be NULL)
 * receives its sequence number.  The LLRs are copied before the call
 * returns.  Returns 0, or -1. */
int drx_rxq_push(drx_rxq* q, int code, const int8_t* llr, uint64_t* fseq);

/* Send every open batch.  Returns 0, or -1. */
int drx_rxq_flush(drx_rxq* q);

/* The next frame in arrival order, if its batch is done (wait = 0), or
 * after sending its batch if needed and waiting for it (wait = 1): its
 * sequence number and code, ceil(kldpc/8) bytes of BCH-corrected codeword
 * into cw (the first kbch bits are the BBFRAME), the LDPC iterations and
 * syndrome flag (the batch's, with stop 1) and the BCH result (corrected
 * bits or -1).  Any output pointer may be NULL.  Returns 1 if a frame was
 * returned, 0 if none is ready or the queue is empty, -1 on error. */
int drx_rxq_pop(drx_rxq* q, int wait, uint64_t* fseq, int* code, uint8_t* cw, int32_t* iters, int32_t* ok,
                int32_t* bch_result);

/* Frames pushed and not yet popped (-1 for NULL). */
int drx_rxq_pending(const drx_rxq* q);

/* ---- soft demapper (reference libdvbrx/src/demap.c:491-533) -------------
 *
 * The reference receiver's max-log demapper on the GPU, ahead of the LDPC
 * decoder: received symbols (interleaved float I/Q, unit average energy) to
 * int8 LLRs in codeword order, 2/n0 x (min distance, bit 1 - min distance,
 * bit 0) quantised as the reference does, the MODCOD's bit interleaver
 * applied.  Results equal drx_demap_frame of the reference's builds with
 * fused multiply-adds (AVX2, AVX-512).  Every DVB-S2 and S2X constellation
 * of the reference (QPSK to 256APSK, 128APSK with its padding bits).
 * Separate names from the reference's drx_demap_* (whose handle also serves
 * its hard-decision and noise-estimation calls): no counterpart to replace. */
typedef struct drx_demapper drx_demapper;

/* A demapper for a MODCOD ("8PSK", "3_5", normal or short frames); NULL for
 * an unknown one. */
drx_demapper* drx_demapper_new(const char* constellation, const char* rate, int short_frame);
void drx_demapper_free(drx_demapper* m);

/* Symbols per frame (the reference's drx_demap_symbols). */
int drx_demapper_symbols(const drx_demapper* m);

/* nframes device frames: sym + f * sym_stride (floats, 8-byte aligned) holds
 * frame f's symbols, n0[f] its noise variance per complex symbol (device);
 * llr + f * llr_stride receives its nldpc LLRs.  Asynchronous on `stream`. */
int drx_demapper_run(drx_demapper* m, const float* sym, size_t sym_stride, const float* n0, int8_t* llr,
                     size_t llr_stride, int nframes, void* stream);

/* One frame in host memory, synchronous (drx_demap_frame's arguments). */
int drx_demapper_frame(drx_demapper* m, const float* sym, float n0, int8_t* llr);

/* ---- baseband layer (reference libdvbrx/src/bb.c:46-101) ----------------
 *
 * No counterpart with these arguments in the reference (its calls take one
 * frame in host memory): device batches straight after the BCH decoder.
 * Stream NULL is the legacy default stream. */

/* Descramble nframes packed BBFRAMEs in place (frame f at frames + f *
 * stride, kbch_bytes long, <= 7274): XOR with the BB scrambling sequence,
 * as drx_bb_descramble (bb.c:62-67).  Asynchronous. */
int drx_bb_descramble_device(uint8_t* frames, size_t stride, int kbch_bytes, int nframes, void* stream);

/* Check the BBHEADER (first 10 bytes) of nframes descrambled frames:
 * status[f] (device) = 0 if drx_bbheader_parse (bb.c:69-101) accepts it in
 * normal mode, 1 if it accepts it in DVB-T2 High Efficiency Mode, -1 if it
 * rejects it.  Asynchronous. */
int drx_bbheader_check_device(const uint8_t* frames, size_t stride, int8_t* status, int nframes, void* stream);

/* Device error word of the handle: 0, or the code of a device-side fault
 * report (2: a group barrier timed out).  Cleared by the call. */
int drx_ldpc_device_error(drx_ldpc* d);

#ifdef __cplusplus
}
#endif

#endif /* DVBRX_B200_H */
