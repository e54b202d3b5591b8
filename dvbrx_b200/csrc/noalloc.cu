/*
 * drx_ldpc_decode_device_noalloc: the plain decoder with its scratch memory
 * in a fixed array compiled into the library, for callers that must not
 * allocate GPU memory while they decode.
 *
 * Who cannot allocate: a receiver's real-time decode thread (the reference
 * runs its LDPC workers on live frames, libdvbrx/src/rxmt.c:514-536), where a
 * cudaMalloc or cudaFree can wait on a device-wide synchronisation for an
 * unbounded time and make the receiver drop samples; and programs whose GPU
 * memory belongs to another allocator (a framework's caching pool, a fixed
 * memory budget) that forbids allocations behind its back.  The regular
 * entry points grow the handle's scratch on demand, which allocates; this
 * one never does.  The handle itself is still made by drx_ldpc_new, at
 * set-up time.
 *
 * The scratch is g_scratch below: 16 MiB of device memory that every GPU
 * which loads the library holds until the process exits.  Bytes [0, 256)
 * hold the frame counter and an error word, cleared by every call; the rest
 * holds one message slab per CTA.  The call runs the kernel the regular
 * entry point runs for the handle: the frame-pair kernel (two frames per
 * CTA) where the handle uses it, its slab holding an 8- or 16-byte record
 * per check and, for the parity-out kernels of normal frames up to rate 4/5,
 * two bytes per parity bit; otherwise the one-frame kernel (R words of 4
 * bytes, 8 above check degree 16).  A call therefore runs at most
 * (16 MiB - 256) / slab CTAs: 64 frame-pair CTAs (128 frames at a time,
 * one CTA on each of 64 SMs) for normal 3/5, against the 296 CTAs (two on
 * every SM) of the regular call, so that large batches decode more slowly
 * than through drx_ldpc_decode_device; 233 frame-pair CTAs (of 296) for
 * short 1/2.
 * Every call shares the array and leaves its contents behind; calls whose
 * kernels overlap on the GPU (concurrent streams, or several host threads)
 * race on it and must be serialised by the caller.
 *
 * Host code cannot use the name g_scratch as a device address (in host code
 * it names a host-side stand-in): the device address comes from
 * cudaGetSymbolAddress, looked up once per device, with that device
 * current.  The first call made on a device does that set-up, which can
 * load this file's module and so allocate and synchronise: make one call
 * with nframes = 0 per device at initialisation, before any stream capture
 * and before the real-time path starts (it does the set-up and decodes
 * nothing).
 */
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>

#include "../../include/dvbrx_b200.h"
#include "codes.h"
#include "ldpc_device.h"

namespace {

constexpr size_t kScratchBytes = (size_t)16 << 20;
constexpr size_t kHeader = 256; /* frame counter, error word */
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_lock;
void* g_addr[kMaxDevices];

thread_local std::string g_noalloc_err;

/* Device address of g_scratch on the current device (set-up on first use). */
void* scratch_address(int dev)
{
    std::lock_guard<std::mutex> lock(g_lock);
    if (!g_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess) {
            g_noalloc_err = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
            return nullptr;
        }
        g_addr[dev] = p;
    }
    return g_addr[dev];
}

}  // namespace

/* Accessors of the handle, defined in capi.cu. */
namespace drxg {
const DevCode* handle_code(const drx_ldpc* d, int* R, int* dclass, int* N, int* nbytes, int* capacity,
                           size_t* smem, cudaStream_t* stream);
int handle_pair(const drx_ldpc* d, size_t* smem, int* capacity);
void handle_set_error(const char* msg);
}  // namespace drxg

extern "C" int drx_ldpc_decode_device_noalloc(drx_ldpc* d, const int8_t* llr, size_t llr_stride,
                                              uint8_t* out, size_t out_stride, int32_t* iters,
                                              uint8_t* ok, int nframes, int max_iter, void* stream)
{
    using namespace drxg;
    if (!d || (nframes > 0 && (!llr || !out))) {
        handle_set_error("NULL argument");
        return -1;
    }
    /* the per-device set-up first: a call with no frames does only that */
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        handle_set_error("drx_ldpc_decode_device_noalloc: no usable current device");
        return -1;
    }
    unsigned char* base = (unsigned char*)scratch_address(dev);
    if (!base) {
        handle_set_error(g_noalloc_err.c_str());
        return -1;
    }
    if (nframes <= 0)
        return 0;
    int R = 0, dclass = 0, N = 0, nbytes = 0, capacity = 0;
    size_t smem = 0;
    cudaStream_t own = nullptr;
    const DevCode* code = handle_code(d, &R, &dclass, &N, &nbytes, &capacity, &smem, &own);
    if (llr_stride < (size_t)N || out_stride < (size_t)nbytes) {
        handle_set_error("row stride below the frame size");
        return -1;
    }
    /* the frame-pair kernel where the regular entry point runs it */
    size_t pair_smem = 0;
    int pair_capacity = 0;
    const int kid = handle_pair(d, &pair_smem, &pair_capacity);
    const size_t slab = kid >= 0 ? decode_pair_msg_bytes(R, kid) : decode_msg_bytes(R, dclass);
    const size_t fit = (kScratchBytes - kHeader) / slab;
    if (fit < 1) {
        handle_set_error(("drx_ldpc_decode_device_noalloc: one CTA needs " + std::to_string(slab) +
                          " bytes of scratch, more than the " + std::to_string(kScratchBytes - kHeader) +
                          " the static array holds").c_str());
        return -1;
    }
    cudaStream_t s = stream ? (cudaStream_t)stream : own;
    /* the frame counter and the error word must start at zero */
    cudaError_t e = cudaMemsetAsync(base, 0, 8, s);
    if (e != cudaSuccess) {
        handle_set_error(cudaGetErrorString(e));
        return -1;
    }
    DecodeParams p{};
    p.code = code;
    p.llr = llr;
    p.llr_stride = llr_stride;
    p.out = out;
    p.out_stride = out_stride;
    p.iters = iters;
    p.ok = ok;
    p.nframes = nframes;
    p.max_iter = max_iter < 0 ? 0 : max_iter;
    p.group = 0;
    p.work = (unsigned*)base;
    p.err = (int*)(base + 4);
    p.msg = base + kHeader;
    p.msg_stride = slab;
    if (kid >= 0) {
        const int grid = (int)std::min<size_t>({ (size_t)(nframes + 1) / 2, (size_t)pair_capacity, fit });
        e = launch_decode_pair(p, kid, pair_smem, grid, s);
    } else {
        const int grid = (int)std::min<size_t>({ (size_t)nframes, (size_t)capacity, fit });
        e = launch_decode(p, dclass, smem, grid, s);
    }
    if (e != cudaSuccess) {
        handle_set_error(cudaGetErrorString(e));
        return -1;
    }
    return 0;
}
