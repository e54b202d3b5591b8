/*
 * Host side of the frame-pair decoder (kernels in ldpc_pair.cuh,
 * instantiated by ldpc_pair_k*.cu): the registry of instantiations, the
 * choice of kernel for a code, shared-memory and scratch sizes, launches.
 */
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "codes.h"
#include "ldpc_device.h"
#include "ldpc_pair.cuh"

namespace drxg {

static size_t a16h(size_t v) { return (v + 15) & ~(size_t)15; }

const PairKernel* pair_kernel_part0(int* n);
const PairKernel* pair_kernel_part1(int* n);
const PairKernel* pair_kernel_part2(int* n);
const PairKernel* pair_kernel_part3(int* n);
const PairKernel* pair_kernel_part4(int* n);
const PairKernel* pair_kernel_part5(int* n);

const PairKernel* pair_kernel_part(int part, int* n)
{
    switch (part) {
    case 0: return pair_kernel_part0(n);
    case 1: return pair_kernel_part1(n);
    case 2: return pair_kernel_part2(n);
    case 3: return pair_kernel_part3(n);
    case 4: return pair_kernel_part4(n);
    case 5: return pair_kernel_part5(n);
    }
    *n = 0;
    return nullptr;
}

/* Every instantiated kernel, the parts in order (the index is the kernel
 * id).  Pair kernels by information-link counts (A, B): every pair of the
 * DVB-S2, S2X and T2 codes, plus predicated kernels for the codes whose
 * layers have more than two different counts (degree bounds 7, 11, 14, 22,
 * 32); LS: late slots the kernel carries (two cover most levelled codes;
 * normal 4/5 and 9/10 need four, short 5/6 five, short 8/9 six); residency
 * mode 0 (one CTA per SM), and the two-CTA twins (modes 1 and 2) of the
 * kernels that fit 80 registers. */
static const std::vector<PairKernel>& kernels()
{
    static const std::vector<PairKernel> all = [] {
        std::vector<PairKernel> v;
        for (int k = 0; k < kPairKernelParts; k++) {
            int n = 0;
            const PairKernel* p = pair_kernel_part(k, &n);
            v.insert(v.end(), p, p + n);
        }
        return v;
    }();
    return all;
}

/* Dynamic shared memory of a pair kernel for a code: the posterior words
 * (every bit, or the information bits of a parity-out kernel and the last
 * parity layer), the link table, layer offsets and level steps */
size_t decode_pair_smem_bytes(int N, int K, int nent, int nsteps, int q, int kid)
{
    const bool po = kid >= 0 && kid < (int)kernels().size() && kernels()[kid].pm == 2;
    return a16h(2 * (size_t)(po ? K : N)) + (po ? a16h(2 * (size_t)kQCp) : 0) + a16h(sizeof(int2) * nent) +
           a16h(sizeof(uint16_t) * (q + 1)) + a16h(sizeof(uint32_t) * nsteps);
}

/* message slab of one CTA: one record per check, 8 or 16 bytes; a
 * parity-out kernel keeps the words of parity layers 0 .. q - 2 after them */
size_t decode_pair_msg_bytes(int R, int kid)
{
    if (kid < 0 || kid >= (int)kernels().size())
        return 0;
    const PairKernel& k = kernels()[kid];
    const int dm = k.gdm > 0 ? k.gdm : k.b + 2;
    const size_t rec = a16h((size_t)R * (dm > 16 ? sizeof(uint4) : sizeof(uint2)));
    return rec + (k.pm == 2 ? a16h(sizeof(uint16_t) * (size_t)(R - kQCp)) : 0);
}

bool pair_kernel_shape(int kid, int* a, int* b, int* gdm, int* ls, int* pm)
{
    if (kid < 0 || kid >= (int)kernels().size())
        return false;
    const PairKernel& k = kernels()[kid];
    *a = k.a;
    *b = k.b;
    *gdm = k.gdm;
    *ls = k.ls;
    *pm = k.pm;
    return true;
}

/* the twin of a mode-0 kernel in mode pm (1 or 2), -1 if it has none */
int pair_kernel_twin(int kid, int pm)
{
    if (kid < 0 || kid >= (int)kernels().size() || kernels()[kid].pm != 0)
        return -1;
    const PairKernel& k = kernels()[kid];
    for (int t = 0; t < (int)kernels().size(); t++) {
        const PairKernel& u = kernels()[t];
        if (u.pm == pm && u.a == k.a && u.b == k.b && u.gdm == k.gdm && u.ls == k.ls)
            return t;
    }
    return -1;
}

int pair_kernel_id(const Code& c)
{
    if (c.deg_max > 32 || !c.phased)
        return -1;
    /* late slots the code needs: link slots 2 .. 2 ls + 1 */
    int ls = 0;
    for (uint64_t m : c.lmeta) {
        const uint32_t b = (uint32_t)(((m >> 8) | (m >> 32)) & 0xFFFFFFull);
        while (b >> (2 * ls + 2))
            ls++;
    }
    if (ls > kLateSlotsMax)
        return -1;
    int lo = 1 << 30, hi = 0, other = 0;
    for (int i = 0; i < c.q; i++) {
        const int n = c.eoff[i + 1] - c.eoff[i];
        lo = n < lo ? n : lo;
        hi = n > hi ? n : hi;
    }
    for (int i = 0; i < c.q; i++) {
        const int n = c.eoff[i + 1] - c.eoff[i];
        other |= n != lo && n != hi;
    }
    if (!other)
        for (int k = 0; k < (int)kernels().size(); k++)
            if (kernels()[k].pm == 0 && kernels()[k].gdm == 0 && kernels()[k].a == lo &&
                kernels()[k].b == hi && kernels()[k].ls >= ls)
                return k;
    for (int k = 0; k < (int)kernels().size(); k++)
        if (kernels()[k].pm == 0 && kernels()[k].gdm >= c.deg_max && kernels()[k].ls >= ls)
            return k;
    return -1;
}

int decode_pair_ctas_per_sm(int kid, size_t smem)
{
    if (kid < 0 || kid >= (int)kernels().size())
        return 0;
    const void* k = kernels()[kid].fn;
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return 0;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, k, kernels()[kid].threads, smem) != cudaSuccess)
        return 0;
    return n;
}

cudaError_t launch_decode_pair(const DecodeParams& p, int kid, size_t smem, int grid, cudaStream_t stream)
{
    if (kid < 0 || kid >= (int)kernels().size())
        return cudaErrorInvalidValue;
    const void* k = kernels()[kid].fn;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess)
        return e;
    DecodeParams pc = p;
    void* args[] = { &pc };
    if (p.group > 0)
        return cudaLaunchCooperativeKernel(k, dim3(grid), dim3(kernels()[kid].threads), args, smem, stream);
    return cudaLaunchKernel(k, dim3(grid), dim3(kernels()[kid].threads), args, smem, stream);
}

}  // namespace drxg
