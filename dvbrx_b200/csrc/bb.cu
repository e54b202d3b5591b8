/*
 * Baseband layer on the GPU, after the BCH decoder: BBFRAME descrambling and
 * the BBHEADER check (EN 302 307-1 5.1.6, 5.2.2), with the reference's
 * results (libdvbrx/src/bb.c:46-101: drx_bb_descramble, drx_bbheader_parse),
 * so that the device hands out BBFRAMEs ready for the TS reconstruction.
 *
 * The scrambling sequence (1 + x^14 + x^15, restarted on every BBFRAME) and
 * the CRC-8 table (0xD5) are generated from the standard into bb_tables.h
 * (dvbrx_b200/tables/gen_bb.py) and live in device memory.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "../../include/dvbrx_b200.h"
#include "bb_tables.h"
#include "handle.h"

namespace drxg {

constexpr int kBbThreads = 256;

/* frames[f][i] ^= prbs[i], i < kbytes; four bytes per thread, grid rows walk
 * the frames */
__global__ void __launch_bounds__(kBbThreads) k_bb_descramble(uint8_t* frames, size_t stride, int kbytes,
                                                             int nframes)
{
    for (int f = blockIdx.y; f < nframes; f += gridDim.y) {
        uint8_t* w = frames + (size_t)f * stride;
        const bool vec = (((uintptr_t)w) & 3) == 0;
        for (int i = 4 * (blockIdx.x * blockDim.x + threadIdx.x); i < kbytes; i += 4 * gridDim.x * blockDim.x) {
            if (vec && i + 4 <= kbytes) {
                const uint32_t p = (uint32_t)g_bb_prbs[i] | (uint32_t)g_bb_prbs[i + 1] << 8 |
                                   (uint32_t)g_bb_prbs[i + 2] << 16 | (uint32_t)g_bb_prbs[i + 3] << 24;
                *(uint32_t*)(w + i) ^= p;
            } else {
                for (int k = i; k < i + 4 && k < kbytes; k++)
                    w[k] ^= g_bb_prbs[k];
            }
        }
    }
}

/* BBHEADER of every frame: 0 valid, 1 valid in DVB-T2 High Efficiency Mode
 * (the CRC XOR 1, for a TS without ISSY), -1 invalid (bb.c:69-101) */
__global__ void __launch_bounds__(kBbThreads) k_bbheader(const uint8_t* frames, size_t stride, int8_t* status,
                                                        int nframes)
{
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nframes)
        return;
    const uint8_t* h = frames + (size_t)f * stride;
    uint8_t b[10];
#pragma unroll
    for (int k = 0; k < 10; k++)
        b[k] = h[k];
    uint8_t c = 0;
#pragma unroll
    for (int k = 0; k < 9; k++)
        c = g_bb_crc8[c ^ b[k]];
    int st = 0;
    if (c != b[9]) {
        if ((uint8_t)(c ^ 1) != b[9] || b[0] >> 6 != 3 || (b[0] & 0x08) || b[2] || b[3] || b[6])
            st = -1;
        else
            st = 1;
    }
    if (st >= 0) {
        const int dfl = b[4] << 8 | b[5], syncd = b[7] << 8 | b[8];
        if (dfl % 8 || dfl > DRXG_KBCH_MAX_BYTES * 8 - 80)
            st = -1;
        else if (b[0] >> 6 == 3 && (syncd > dfl || syncd % 8))
            st = -1;
    }
    status[f] = (int8_t)st;
}

}  // namespace drxg

using namespace drxg;

extern "C" {

int drx_bb_descramble_device(uint8_t* frames, size_t stride, int kbch_bytes, int nframes, void* stream)
{
    if (nframes <= 0)
        return 0;
    if (!frames || kbch_bytes < 0 || kbch_bytes > DRXG_KBCH_MAX_BYTES || stride < (size_t)kbch_bytes) {
        set_error("drx_bb_descramble_device: bad arguments");
        return -1;
    }
    const int gx = std::max(1, (kbch_bytes / 4 + kBbThreads - 1) / kBbThreads);
    const dim3 grid(gx, std::min(nframes, 4096));
    k_bb_descramble<<<grid, kBbThreads, 0, (cudaStream_t)stream>>>(frames, stride, kbch_bytes, nframes);
    return cuda_check(cudaGetLastError(), "descrambler launch") ? 0 : -1;
}

int drx_bbheader_check_device(const uint8_t* frames, size_t stride, int8_t* status, int nframes, void* stream)
{
    if (nframes <= 0)
        return 0;
    if (!frames || !status || stride < 10) {
        set_error("drx_bbheader_check_device: bad arguments");
        return -1;
    }
    k_bbheader<<<(nframes + kBbThreads - 1) / kBbThreads, kBbThreads, 0, (cudaStream_t)stream>>>(frames, stride,
                                                                                               status, nframes);
    return cuda_check(cudaGetLastError(), "BBHEADER check launch") ? 0 : -1;
}

}  // extern "C"
