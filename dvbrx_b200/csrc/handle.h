/*
 * The decoder handle (drx_ldpc) and the host helpers shared by the C-ABI
 * files (capi.cu, mix.cu).
 */
#pragma once
#include <cuda_runtime.h>

#include <string>

#include "../../include/dvbrx_b200.h"
#include "codes.h"
#include "ldpc_device.h"

using drxg::Code;
using drxg::DevCode;

/* chunks of a pipelined host call, and their events (two per chunk + one) */
constexpr int kMaxChunks = 15;
constexpr int kChunkEvents = 2 * kMaxChunks + 1;

struct drx_ldpc {
    int device = 0;
    int sms = 0;
    Code code;
    drx_fec_params params{};
    int nbytes = 0;
    void* blob = nullptr; /* device: DevCode + tables */
    DevCode* dcode = nullptr;
    size_t smem = 0;
    int ctas_per_sm = 0;
    size_t pair_smem = 0;
    int pair_ctas_per_sm = 0; /* 0: the frame-pair kernel does not run this code */
    int pair_kid = -1;        /* its instantiation for this code */
    int variant = DRX_VARIANT_AUTO;
    int wait_limit = 0;     /* polls of a group barrier before a launch gives up (0: default) */
    int test_skip_vote = 0; /* testing: CTA test_skip_vote - 1 of group launches never votes */
    cudaStream_t stream = nullptr;
    /* scratch */
    void* msg = nullptr;
    size_t msg_cap = 0;
    unsigned* work = nullptr;
    unsigned* sync = nullptr;
    size_t sync_cap = 0;
    int* err = nullptr;
    /* learned check nodes: kLearnMaxIters rows of kLearnClasses words, then
     * the 33 degree classes; learn_iters rows in use (0: none) */
    uint32_t* learn = nullptr;
    int learn_iters = 0;
    /* fallback of the learned decode: failing rows (fb_cap + a count word)
     * and flags when the caller passes none */
    int32_t* fb_rows = nullptr;
    uint8_t* fb_ok = nullptr;
    size_t fb_cap = 0;
    /* pipelined host calls: two decode streams, one copy stream, chunk
     * events and frame counters, and a second message slab */
    cudaStream_t pipe[2] = {nullptr, nullptr};
    cudaStream_t copy = nullptr;
    cudaEvent_t chunk_ev[kChunkEvents] = {}; /* per chunk: copied in, results out; then the start */
    unsigned* chunk_work = nullptr;
    void* msg2 = nullptr;
    size_t msg2_cap = 0;
    /* staging of the host-pointer calls */
    int8_t* h_llr = nullptr;
    uint8_t* h_out = nullptr;
    int32_t* h_it = nullptr;
    uint8_t* h_ok = nullptr;
    int8_t* d_llr = nullptr;
    uint8_t* d_out = nullptr;
    int32_t* d_it = nullptr;
    uint8_t* d_ok = nullptr;
    size_t stage_frames = 0;
};

namespace drxg {

void set_error(const std::string& s);
bool cuda_check(cudaError_t e, const char* what);

/* True if the next device allocation of the library must fail (the
 * allocation-failure test hook, drx_test_fail_device_alloc). */
bool alloc_fails_now();

/* cudaMalloc through the library's test hook: every device allocation of
 * the library goes through here. */
template <class T>
cudaError_t dev_malloc(T** p, size_t n)
{
    if (alloc_fails_now()) {
        *p = nullptr;
        return cudaErrorMemoryAllocation;
    }
    return cudaMalloc((void**)p, n);
}

}  // namespace drxg
