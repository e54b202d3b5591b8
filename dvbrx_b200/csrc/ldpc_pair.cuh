/*
 * Plain decoder, frame-pair variant (device code, included by the
 * ldpc_pair_k*.cu files, which instantiate the kernels in parts so that
 * they compile in parallel; ldpc_pair.cu holds the host side): the same arithmetic as ldpc_decode.cu
 * (bit-exact to libdvbrx/src/ldpc.c), two frames per CTA.
 *
 * SIMD within a register: every value of the decoder fits 16 bits, so each
 * 32-bit register carries the same quantity for two frames, lane A in the
 * low half and lane B in the high half, and every step of the check node is
 * a native 16x2 instruction on sm_100a (video min/max __vmins2/__vmaxs2,
 * DPX __viaddmax_s16x2 for the saturating add and |x|, the lane-wise __vadd2,
 * PRMT for sign masks and byte packing, an FP16 compare for the message
 * index).  One instruction stream decodes two frames.
 *
 * Shared memory holds both frames' posteriors interleaved: the 16-bit word
 * v holds the int8 posterior of variable v for lane A (low byte) and lane B
 * (high byte): K information bits, then R parity bits in layer order.
 *
 * A check node runs on one thread: 360 of the 384 threads hold the 360
 * checks of a layer, every link of a check in registers, no shuffles (two
 * threads per check, combining their minimums with a shuffle round, ran
 * 17-22 % slower on 3/5 and 18/30: twice the per-check set-up and finish
 * work for the same link work).  Levelled layers run in phases (layer_pair): the
 * wavefront levels carry only the links two checks of the layer share.  The
 * thread of a check stores its compressed messages for both frames in one
 * 8-byte record: per lane min0 (6 bits) | min1 << 6 | index << 12, then the
 * sign bits of lane A in the low half and of lane B in the high half.
 *
 * Frames stream through the two lanes independently: when a lane's frame
 * passes the syndrome check or reaches max_iter, its results are written
 * and the lane takes the next frame of the batch (its first iteration reads
 * zero messages), so a converged frame never waits for its neighbour.
 * Every DVB-S2, S2X and T2 code runs here (check degrees up to 30; message
 * records of 16 bytes above degree 16).
 */
#pragma once
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "codes.h"
#include "ldpc_device.h"

namespace drxg {

constexpr int kQCp = 360;
/* a kernel compiled for LS late slots reads late and writes early only owned
 * slots 1 .. LS of each thread (link slots 2 .. 2 LS + 1); two cover every
 * pair code but short 3/5 and 4/5, which take three */
constexpr int kLateSlotsMax = 6;

/* PRMT in its default mode: a selector nibble with bit 3 set replicates the
 * sign bit of the selected byte.  (__byte_perm keeps only the low 3 bits of
 * each nibble, so the sign-replicating forms need the instruction itself.) */
__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t sel)
{
    uint32_t d;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(a), "r"(b), "r"(sel));
    return d;
}
/* two int8 (low 16 bits) -> int16x2, sign-extended */
__device__ __forceinline__ uint32_t sx2(uint32_t b) { return prmt(b, 0, 0x9180); }
/* int16x2 in [-128, 127] -> two bytes (low 16 bits) */
__device__ __forceinline__ uint32_t pk2(uint32_t v) { return prmt(v, 0, 0x0020); }
/* 0xFFFF in each lane whose bit 15 is set */
__device__ __forceinline__ uint32_t lmask(uint32_t v) { return prmt(v, 0, 0xBB99); }
__device__ __forceinline__ uint32_t sel(uint32_t m, uint32_t a, uint32_t b) { return (m & a) | (~m & b); }
/* saturating int8 add in int16 lanes */
__device__ __forceinline__ uint32_t sadd(uint32_t a, uint32_t b)
{
    return __vmins2(__viaddmax_s16x2(a, b, 0xFF80FF80u), 0x007F007Fu);
}
/* lane-wise |x| = max(~x + 1, x): one LOP3 and one DPX add-max (a 16x2
 * subtract, __vsub2, has no single instruction: it costs three or four) */
__device__ __forceinline__ uint32_t abs2(uint32_t x) { return __viaddmax_s16x2(~x, 0x00010001u, x); }
/* lane-wise -x, the 16x2 add (__vadd2) being one instruction */
__device__ __forceinline__ uint32_t neg2(uint32_t x) { return __vadd2(~x, 0x00010001u); }
/* 16-bit shared-memory accesses at a 32-bit shared address */
__device__ __forceinline__ uint32_t lds16(uint32_t a)
{
    unsigned short v;
    asm volatile("ld.shared.u16 %0, [%1];" : "=h"(v) : "r"(a));
    return v;
}
__device__ __forceinline__ void sts16(uint32_t a, uint32_t v)
{
    asm volatile("st.shared.u16 [%0], %1;" ::"r"(a), "h"((unsigned short)v));
}
__device__ __forceinline__ uint32_t heq(uint32_t a, uint32_t b)
{
    return __heq2_mask(*(const __half2*)&a, *(const __half2*)&b);
}

/*
 * One check node (i, j) for both lanes, on one thread: link slots
 * k = 0 .. S-1.  Slot 0 is the parity bit, slot 1 the previous parity bit
 * (absent for (0, 0)), 2 + e information entry e of the layer.  DM is the
 * node degree (EXACT) or a bound on it (the degree is then a run-time
 * value).  The node state lives in registers across the phases of its layer
 * (see layer_pair).  Slot masks and the message index keep slot k at bit k.
 *
 * Minimums are taken over keys |x| * 32 + k (|x| <= 128, so a key fits 13
 * bits of a 16-bit lane): the smallest key gives min0 and the slot holding
 * it, the second smallest min1 (a tie between two slots at min0 puts min1 =
 * min0, and then which slot holds min0 changes no message).  The full
 * passes run every slot without branches: a slot that is not a link, or
 * whose bit an earlier check of the layer writes (read later, in its level),
 * enters the minimums with a key above every real one; stores are
 * predicated.
 *
 * Sign bits of a record: the 16 slots of a word in the byte layout
 * byte 0 = lane A even slots, byte 1 = lane A odd slots, byte 2 = lane B
 * even slots, byte 3 = lane B odd slots, slot 2s (2s + 1) at bit 7 - s of
 * its byte; shifted left by s, the word holds the signs of slots 2s and
 * 2s + 1 in the sign bits of its bytes, which one PRMT turns into lane
 * masks.
 */
/* A check's message record: 8 bytes up to degree 16 (per lane min0, min1
 * and a 4-bit index in one word, 16 sign bits per lane in the other); 16
 * bytes above (min0 and min1; sign bits of slots 0-15 and of slots 16-31;
 * the index, 16 bits per lane). */
template <bool WIDE>
using PairRec = typename std::conditional<WIDE, uint4, uint2>::type;

/* key of a slot that takes no part in the minimums */
constexpr uint32_t kKeyOff = 0x1FE01FE0u; /* 255 * 32 in both lanes */

/* the sign bits of slot k (k < 16) of both lanes in a record word */
__device__ __forceinline__ constexpr uint32_t sign_bits(int k)
{
    return (k & 1) ? (1u << (15 - (k >> 1))) | (1u << (31 - (k >> 1)))
                   : (1u << (7 - (k >> 1))) | (1u << (23 - (k >> 1)));
}
/* lane masks of slot k's sign bits in record word w (k < 16) */
__device__ __forceinline__ uint32_t sign_mask(uint32_t w, int k)
{
    return prmt(w << (k >> 1), 0, (k & 1) ? 0xBB99u : 0xAA88u);
}

/* The learned magnitudes of the current iteration (learned kernels): byte
 * 1024 h + 128 k + m = min(learned_mag(m, word of lane h's row and degree
 * class k), 255) for capped minimums m = 0..127.  A magnitude of 255 or more
 * saturates every posterior it meets and is capped at 32 in the record, so
 * the cap at 255 changes no result.  Rebuilt at the start of each learned
 * iteration (iterate_pair). */
static __shared__ uint8_t s_learn_lut[2 * kLearnClasses * 128];

/* the learned magnitudes of capped minimums c (both lanes, 0..127) from the
 * check's class table at index t of s_learn_lut (lane A; lane B at t + 1024) */
__device__ __forceinline__ uint32_t learned_lut(uint32_t c, uint32_t t)
{
    return (uint32_t)s_learn_lut[t + (c & 0xFFFFu)] | (uint32_t)s_learn_lut[t + 1024u + (c >> 16)] << 16;
}

/* WIDE: the kernel's records are 16 bytes (its degree bound is above 16).
 * PO: the parity posteriors (slots 0 and 1) are not in shared memory; the
 * layer loop hands their two-byte words in and takes the new ones back. */
template <int DM, bool EXACT, int LS, bool WIDE, bool PO>
struct PairCheckKey {
    static_assert(DM <= (WIDE ? 32 : 16), "degree above the record's slots");
    using Rec = PairRec<WIDE>;
    static constexpr bool kKeys = true;
    static constexpr int S = DM;
    /* slots that can be late or early: K0 .. K1 (link slots 2 .. 2 LS + 1) */
    static constexpr int K0 = 2;
    static constexpr int K1 = S - 1 < 2 * LS + 1 ? S - 1 : 2 * LS + 1;
    uint32_t addr[S]; /* shared-memory byte addresses of the owned links' posteriors */
    uint32_t x[S];
    uint32_t live, inm, outm; /* bit k: slot k is a link / is read late / is written early */
    uint32_t n0, n1, p0, p1, idxh, sgn, sgn1; /* old messages; sgn: sign bits of slots 0-15, sgn1: 16-31 */
    uint32_t min0, min1, sg;                  /* smallest keys, sign parity (bit 15 / 31) */
    uint32_t a0, a1, b0, b1, nidx;            /* outgoing message candidates (set by finish), index */
    uint32_t recw;                            /* the record's magnitude word (set by finish) */

    /* ent: the layer's entries (shared byte address of the link group's first
     * posterior word, -2a), cnt of them */
    __device__ __forceinline__ void setup(const int2* __restrict__ ent, int cnt, int K, int q, int i, int j,
                                          Rec rec, uint32_t fresh, unsigned long long meta, uint32_t sbase)
    {
        const int D = EXACT ? DM : cnt + 2;
        const int pc = K + kQCp * i + j;
        const int pp = i ? pc - kQCp : K + kQCp * (q - 1) + j - 1;
        uint32_t lv = (1u << D) - 1u;
        if ((i | j) == 0)
            lv &= ~2u;
        live = lv;
        inm = (uint32_t)(meta >> 8) & 0xFFFFFFu;
        outm = (uint32_t)(meta >> 32) & 0xFFFFFFu;
        const uint32_t tj = 2u * (uint32_t)j;
#pragma unroll
        for (int k = 0; k < S; k++) {
            if (k < 2) {
                addr[k] = PO ? 0u : sbase + 2u * (uint32_t)(k == 0 ? pc : pp);
            } else {
                /* a slot past the degree takes the last link's address: read, never used.
                 * Link of check j: word (j - a) mod 360 of the group, as min(u, u + 720)
                 * over unsigned byte offsets u = 2 j - 2 a */
                const int2 e = ent[min(k, D - 1) - 2];
                const uint32_t u = tj + (uint32_t)e.y;
                addr[k] = (uint32_t)e.x + __viaddmin_u32(u, 2u * kQCp, u);
            }
        }
        /* messages: zero for a lane in its first iteration */
        const uint32_t w0 = rec.x & ~fresh;
        sgn = rec.y & ~fresh;
        const uint32_t m0 = w0 & 0x003F003Fu, m1 = (w0 >> 6) & 0x003F003Fu;
        if constexpr (WIDE) {
            sgn1 = rec.z & ~fresh;
            idxh = (rec.w & ~fresh) | 0x64006400u; /* FP16 1024 + index */
        } else {
            sgn1 = 0;
            idxh = ((w0 >> 12) & 0x000F000Fu) | 0x64006400u; /* FP16 1024 + index */
        }
        /* minus the message: +m if it is negative, else -min(m, 31) */
        n0 = m0;
        n1 = m1;
        p0 = __viaddmax_s16x2(~m0, 0x00010001u, 0xFFE1FFE1u); /* max(-m, -31) */
        p1 = __viaddmax_s16x2(~m1, 0x00010001u, 0xFFE1FFE1u);
        min0 = min1 = kKeyOff;
        sg = 0;
    }

    /* minus the old message of slot k */
    __device__ __forceinline__ uint32_t unmsg(int k) const
    {
        const uint32_t im = heq(idxh, 0x64006400u + (uint32_t)k * 0x00010001u);
        const uint32_t sm = sign_mask(k < 16 ? sgn : sgn1, k & 15);
        return sel(sm, sel(im, n1, n0), sel(im, p1, p0));
    }

    /* the key of value v in slot k */
    static __device__ __forceinline__ uint32_t key(uint32_t v, int k)
    {
        return abs2(v) * 32u + (uint32_t)k * 0x00010001u;
    }

    __device__ __forceinline__ void fold(uint32_t kv)
    {
        min1 = __vmins2(min1, __vmaxs2(min0, kv));
        min0 = __vmins2(min0, kv);
    }

    /* every slot but the late ones, without branches; minimums folded
     * two slots at a time: min1 = second smallest of {min0, min1, a, b} =
     * min3(max(min0, min(a, b)), min1, max(a, b)).  LEV: the layer has late
     * slots; otherwise only the slots that can be absent are masked (the
     * previous parity of check (0, 0)). */
    template <bool LEV>
    __device__ __forceinline__ void read_all(const uint16_t* __restrict__ post, uint32_t r0, uint32_t r1)
    {
        const uint32_t excl = LEV ? (~live | inm) : ~live;
        /* slot k read: its value kept in x[k] (minus its old message for a
         * late slot), its key returned */
        auto slot = [&](int k) {
            const uint32_t m = unmsg(k);
            const uint32_t raw = PO && k < 2 ? (k == 0 ? r0 : r1) : lds16(addr[k]);
            const uint32_t v = sadd(sx2(raw), m);
            uint32_t kv = key(v, k);
            /* late slots are among K0 .. K1; past them only a non-link (inexact kernels) */
            const bool maybe_late = LEV && k >= K0 && k <= K1;
            if (maybe_late || !EXACT || k == 1) {
                /* excluded: not a link, or late (its sign and key are taken in read_late) */
                const bool ex = (excl >> k) & 1u;
                kv = ex ? kKeyOff : kv;
                sg ^= ex ? 0u : v;
            } else {
                sg ^= v;
            }
            if (maybe_late)
                x[k] = ((inm >> k) & 1u) ? m : v;
            else
                x[k] = v;
            return kv;
        };
#pragma unroll
        for (int k = 0; k + 1 < S; k += 2) {
            const uint32_t a = slot(k), b = slot(k + 1);
            const uint32_t lo = __vmins2(a, b), hi = __vmaxs2(a, b);
            min1 = __vimin3_s16x2(__vmaxs2(min0, lo), min1, hi);
            min0 = __vimin3_s16x2(min0, a, b);
        }
        if (S & 1)
            fold(slot(S - 1));
    }

    /* a thread that holds no check (t >= 360): valid addresses, no links, so
     * that it can run the warp-uniform level steps of its warp */
    __device__ __forceinline__ void idle(uint32_t sbase)
    {
#pragma unroll
        for (int k = 0; k < S; k++) {
            addr[k] = sbase;
            x[k] = 0;
        }
        live = inm = outm = 0;
        n0 = n1 = p0 = p1 = sgn = sgn1 = 0;
        idxh = 0x64006400u;
        min0 = min1 = kKeyOff;
        sg = a0 = a1 = b0 = b1 = nidx = recw = 0;
    }

    /* the late slots (their bits were written by earlier levels) of a check
     * in the current level (mine); other threads keep their state.  Shared
     * links come first in every layer (codes.cpp), so late and early slots
     * are among slots 2 .. KE */
    template <int KE>
    __device__ __forceinline__ void read_late(const uint16_t* __restrict__ post, bool mine)
    {
        const uint32_t im = mine ? inm : 0u;
#pragma unroll
        for (int k = K0; k <= KE; k++) {
            const bool in = (im >> k) & 1u;
            const uint32_t v = sadd(sx2(lds16(addr[k])), x[k]);
            x[k] = in ? v : x[k];
            sg ^= in ? v : 0u;
            fold(in ? key(v, k) : kKeyOff);
        }
    }

    /* the cap at 127 and offset 1, or the learned magnitudes of each lane's
     * iteration (lpA: the check's class table, learned_lut; lpB unused); the
     * outgoing candidates +-mn0, +-mn1 with the check's sign parity applied
     * (a0, a1 for a slot whose value is positive, b0 = -a0, b1 = -a1
     * otherwise) and the record's magnitudes.
     * Only threads with `take` keep the result: the level steps run it on
     * whole warps */
    __device__ __forceinline__ void finish(bool take, bool learned, uint32_t lpA, uint32_t lpB)
    {
        const uint32_t c0 = __vmins2((min0 >> 5) & 0x07FF07FFu, 0x007F007Fu);
        const uint32_t c1 = __vmins2((min1 >> 5) & 0x07FF07FFu, 0x007F007Fu);
        uint32_t m0, m1;
        if (learned) {
            m0 = learned_lut(c0, lpA);
            m1 = learned_lut(c1, lpA);
        } else {
            m0 = __viaddmax_s16x2(c0, 0xFFFFFFFFu, 0u);
            m1 = __viaddmax_s16x2(c1, 0xFFFFFFFFu, 0u);
        }
        if (take) {
            /* both signs of each candidate side by side (the level steps wait on this chain) */
            const uint32_t sm = lmask(sg), q0 = neg2(m0), q1 = neg2(m1);
            a0 = sel(sm, q0, m0);
            a1 = sel(sm, q1, m1);
            b0 = sel(sm, m0, q0);
            b1 = sel(sm, m1, q1);
            nidx = (min0 & 0x001F001Fu) | 0x64006400u; /* FP16 1024 + slot of min0 */
            /* per lane min0 (6 bits) | min1 << 6, magnitudes capped at 32 (| index << 12 below degree 17) */
            recw = __vmins2(m0, 0x00200020u) | (__vmins2(m1, 0x00200020u) << 6);
            if (!WIDE)
                recw |= (min0 & 0x000F000Fu) << 12;
        }
    }

    /* new posterior of slot k (two bytes) and the lane mask of its value's sign */
    __device__ __forceinline__ uint32_t update(int k, uint32_t& xm) const
    {
        const uint32_t v = x[k];
        xm = lmask(v);
        const uint32_t eq = heq(nidx, 0x64006400u + (uint32_t)k * 0x00010001u);
        const uint32_t o = sel(xm, sel(eq, b1, b0), sel(eq, a1, a0));
        return pk2(sadd(v, o));
    }

    /* posteriors that later levels of the layer read (checks of the current
     * level only) */
    template <int KE>
    __device__ __forceinline__ void write_early(uint16_t* __restrict__ post, bool mine) const
    {
        const uint32_t om = mine ? outm : 0u;
#pragma unroll
        for (int k = K0; k <= KE; k++) {
            uint32_t xm;
            const uint32_t nv = update(k, xm);
            if ((om >> k) & 1u)
                sts16(addr[k], nv);
        }
    }

    /* every other posterior (predicated stores) and the node's compressed
     * messages for both lanes: the slot holding min0 and one sign bit per
     * slot (the outgoing message's: the value's sign times the parity).
     * PO: the parity words go to o0 and o1. */
    __device__ __forceinline__ void write_rest(uint16_t* __restrict__ post, Rec* __restrict__ dst, uint32_t& o0,
                                               uint32_t& o1)
    {
        const uint32_t wm = live & ~outm;
        uint32_t nsg = 0, nsg1 = 0;
#pragma unroll
        for (int k = 0; k < S; k++) {
            uint32_t xm;
            const uint32_t nv = update(k, xm);
            if (PO && k < 2)
                (k == 0 ? o0 : o1) = nv;
            else if (EXACT && k > K1 && k != 1)
                sts16(addr[k], nv); /* every slot past K1 is a link written here */
            else if ((wm >> k) & 1u)
                sts16(addr[k], nv);
            if (k < 16)
                nsg |= xm & sign_bits(k);
            else
                nsg1 |= xm & sign_bits(k - 16);
        }
        /* the outgoing signs: each value's sign flipped where the parity is odd */
        const uint32_t pm = lmask(sg);
        nsg ^= pm;
        if constexpr (WIDE) {
            nsg1 ^= pm;
            __stcg(dst, make_uint4(recw, nsg, nsg1, nidx & 0x001F001Fu));
        } else {
            __stcg(dst, make_uint2(recw, nsg));
        }
    }
};

/*
 * The previous form of the check node (min form), kept for the kernels where
 * it measures faster (low check degrees, and levelled codes whose wavefront
 * steps wait on the check's finish): minimums over |x| itself, the index of
 * min0 found in the write pass (|x| > min0 per slot), sign bits of slot k
 * at bit k (lane A) and 16 + k (lane B), entries as (shared byte address of
 * the link for check 0 before the wrap, a).  Both forms give the reference's
 * results; a kernel uses one form throughout (its records, entries and
 * syndrome scan).
 */
template <int DM, bool EXACT, int LS, bool WIDE, bool PO>
struct PairCheckMin {
    static_assert(DM <= (WIDE ? 32 : 16), "degree above the record's slots");
    using Rec = PairRec<WIDE>;
    static constexpr bool kKeys = false;
    static constexpr int S = DM;
    /* slots that can be late or early: K0 .. K1 (link slots 2 .. 2 LS + 1) */
    static constexpr int K0 = 2;
    static constexpr int K1 = S - 1 < 2 * LS + 1 ? S - 1 : 2 * LS + 1;
    uint32_t addr[S]; /* shared-memory byte addresses of the owned links' posteriors */
    uint32_t x[S];
    uint32_t live, inm, outm; /* bit k: slot k is a link / is read late / is written early */
    uint32_t n0, n1, p0, p1, idxh, sgn, sgn1; /* sgn: sign bits of slots 0-15, sgn1: 16-31 */
    uint32_t min0, min1, sg, mn0, mn1;
    uint32_t m0p1, nmn0, nmn1; /* min0 + 1, -mn0, -mn1 (set by finish) */

    __device__ __forceinline__ void setup(const int2* __restrict__ ent, int cnt, int K, int q, int i, int j,
                                          Rec rec, uint32_t fresh, unsigned long long meta, uint32_t sbase)
    {
        const int D = EXACT ? DM : cnt + 2;
        const int pc = K + kQCp * i + j;
        const int pp = i ? pc - kQCp : K + kQCp * (q - 1) + j - 1;
        uint32_t lv = (1u << D) - 1u;
        if ((i | j) == 0)
            lv &= ~2u;
        live = lv;
        inm = (uint32_t)(meta >> 8) & 0xFFFFFFu;
        outm = (uint32_t)(meta >> 32) & 0xFFFFFFu;
#pragma unroll
        for (int k = 0; k < S; k++) {
            if (k < 2) {
                addr[k] = PO ? 0u : sbase + 2u * (uint32_t)(k == 0 ? pc : pp);
            } else {
                /* a slot past the degree takes the last link's address: read, never used */
                const int2 e = ent[min(k, D - 1) - 2];
                addr[k] = (uint32_t)e.x + 2u * (uint32_t)j + (j < e.y ? 2u * kQCp : 0u);
            }
        }
        /* messages: zero for a lane in its first iteration */
        const uint32_t w0 = rec.x & ~fresh;
        sgn = rec.y & ~fresh;
        const uint32_t m0 = w0 & 0x003F003Fu, m1 = (w0 >> 6) & 0x003F003Fu;
        if constexpr (WIDE) {
            sgn1 = rec.z & ~fresh;
            idxh = (rec.w & ~fresh) | 0x64006400u; /* FP16 1024 + index */
        } else {
            sgn1 = 0;
            idxh = ((w0 >> 12) & 0x000F000Fu) | 0x64006400u; /* FP16 1024 + index */
        }
        /* minus the message: +m if it is negative, else -min(m, 31) */
        n0 = m0;
        n1 = m1;
        p0 = __viaddmax_s16x2(~m0, 0x00010001u, 0xFFE1FFE1u); /* max(-m, -31) */
        p1 = __viaddmax_s16x2(~m1, 0x00010001u, 0xFFE1FFE1u);
        min0 = min1 = 0x00FF00FFu;
        sg = 0;
    }

    /* minus the old message of slot k */
    __device__ __forceinline__ uint32_t unmsg(int k) const
    {
        const uint32_t im = heq(idxh, 0x64006400u + (uint32_t)k * 0x00010001u);
        const uint32_t sm = lmask((k < 16 ? sgn : sgn1) << (15 - (k & 15)));
        return sel(sm, sel(im, n1, n0), sel(im, p1, p0));
    }

    __device__ __forceinline__ void fold(uint32_t v)
    {
        const uint32_t a = abs2(v);
        min1 = __vmins2(min1, __vmaxs2(min0, a));
        min0 = __vmins2(min0, a);
        sg ^= v;
    }

    /* every slot but the late ones, without branches; minimums folded
     * two slots at a time: min1 = second smallest of {min0, min1, a, b} =
     * min3(max(min0, min(a, b)), min1, max(a, b)).  LEV: the layer has late
     * slots; otherwise only the slots that can be absent are masked (the
     * previous parity of check (0, 0)). */
    template <bool LEV>
    __device__ __forceinline__ void read_all(const uint16_t* __restrict__ post, uint32_t r0, uint32_t r1)
    {
        const uint32_t excl = LEV ? (~live | inm) : ~live;
        uint32_t f[S];
#pragma unroll
        for (int k = 0; k < S; k++) {
            const uint32_t m = unmsg(k);
            const uint32_t raw = PO && k < 2 ? (k == 0 ? r0 : r1) : lds16(addr[k]);
            uint32_t v = sadd(sx2(raw), m);
            if (LEV || !EXACT || k == 1)
                v = ((excl >> k) & 1u) ? 0x00FF00FFu : v;
            f[k] = v;
            /* a late slot keeps minus its old message for read_late */
            x[k] = LEV && ((inm >> k) & 1u) ? m : v;
        }
#pragma unroll
        for (int k = 0; k + 1 < S; k += 2) {
            const uint32_t a = abs2(f[k]), b = abs2(f[k + 1]);
            const uint32_t lo = __vmins2(a, b), hi = __vmaxs2(a, b);
            min1 = __vimin3_s16x2(__vmaxs2(min0, lo), min1, hi);
            min0 = __vimin3_s16x2(min0, a, b);
            sg ^= f[k] ^ f[k + 1];
        }
        if (S & 1)
            fold(f[S - 1]);
    }

    /* a thread that holds no check (t >= 360): valid addresses, no links, so
     * that it can run the warp-uniform level steps of its warp */
    __device__ __forceinline__ void idle(uint32_t sbase)
    {
#pragma unroll
        for (int k = 0; k < S; k++) {
            addr[k] = sbase;
            x[k] = 0x00FF00FFu;
        }
        live = inm = outm = 0;
        n0 = n1 = p0 = p1 = sgn = sgn1 = 0;
        idxh = 0x64006400u;
        min0 = min1 = 0x00FF00FFu;
        sg = mn0 = mn1 = m0p1 = nmn0 = nmn1 = 0;
    }

    /* the late slots (their bits were written by earlier levels) of a check
     * in the current level (mine); other threads keep their state.  Shared
     * links come first in every layer (codes.cpp), so late and early slots
     * are among slots 2 .. KE */
    template <int KE>
    __device__ __forceinline__ void read_late(const uint16_t* __restrict__ post, bool mine)
    {
        const uint32_t im = mine ? inm : 0u;
#pragma unroll
        for (int k = K0; k <= KE; k++) {
            const bool in = (im >> k) & 1u;
            const uint32_t v = sadd(sx2(lds16(addr[k])), x[k]);
            x[k] = in ? v : x[k];
            fold(in ? v : 0x00FF00FFu);
        }
    }

    /* the cap at 127 and offset 1, or the learned magnitudes of each lane's
     * iteration (lpA: the check's class table, learned_lut; lpB unused).
     * Only threads with `take` keep the result: the level steps run it on
     * whole warps */
    __device__ __forceinline__ void finish(bool take, bool learned, uint32_t lpA, uint32_t lpB)
    {
        const uint32_t c1 = min1, c0 = min0;
        uint32_t m0, m1;
        if (learned) {
            m0 = learned_lut(__vmins2(c0, 0x007F007Fu), lpA);
            m1 = learned_lut(__vmins2(c1, 0x007F007Fu), lpA);
        } else {
            m0 = __viaddmax_s16x2(__vmins2(c0, 0x007F007Fu), 0xFFFFFFFFu, 0u);
            m1 = __viaddmax_s16x2(__vmins2(c1, 0x007F007Fu), 0xFFFFFFFFu, 0u);
        }
        if (take) {
            mn0 = m0;
            mn1 = m1;
            m0p1 = __vadd2(c0, 0x00010001u);
            nmn0 = neg2(m0);
            nmn1 = neg2(m1);
        }
    }

    /* new posterior of slot k (two bytes), and its masks: lanes where
     * |x| is above min0 (the slot does not hold the minimum) and lanes whose
     * outgoing message is negative */
    __device__ __forceinline__ uint32_t update(int k, uint32_t& above, uint32_t& neg) const
    {
        const uint32_t v = x[k];
        /* min0 - |x| = min(min0 + x, (min0 + 1) + ~x) < 0 */
        above = lmask(__viaddmin_s16x2(~v, m0p1, __vadd2(min0, v)));
        neg = lmask(sg ^ v);
        const uint32_t o = sel(neg, sel(above, nmn0, nmn1), sel(above, mn0, mn1));
        return pk2(sadd(v, o));
    }

    /* posteriors that later levels of the layer read (checks of the current
     * level only) */
    template <int KE>
    __device__ __forceinline__ void write_early(uint16_t* __restrict__ post, bool mine) const
    {
        const uint32_t om = mine ? outm : 0u;
#pragma unroll
        for (int k = K0; k <= KE; k++) {
            uint32_t above, neg;
            const uint32_t nv = update(k, above, neg);
            if ((om >> k) & 1u)
                sts16(addr[k], nv);
        }
    }

    /* every other posterior (predicated stores) and the node's compressed
     * messages for both lanes, stored by thread 0: the slot holding min0 and
     * one sign bit per slot.  PO: the parity words go to o0 and o1. */
    __device__ __forceinline__ void write_rest(uint16_t* __restrict__ post, Rec* __restrict__ dst, uint32_t& o0,
                                               uint32_t& o1)
    {
        const uint32_t wm = live & ~outm;
        uint32_t nidx = 0, nsg = 0, nsg1 = 0; /* nidx per lane: k + 1 of a slot holding min0, 0 if none */
#pragma unroll
        for (int k = 0; k < S; k++) {
            uint32_t above, neg;
            const uint32_t nv = update(k, above, neg);
            if (PO && k < 2)
                (k == 0 ? o0 : o1) = nv;
            else if ((wm >> k) & 1u)
                sts16(addr[k], nv);
            nidx = sel(above, nidx, (uint32_t)(k + 1) * 0x00010001u);
            if (k < 16)
                nsg |= neg & (0x00010001u << k);
            else
                nsg1 |= neg & (0x00010001u << (k - 16));
        }
        nidx = __viaddmax_s16x2(nidx, 0xFFFFFFFFu, 0u); /* slot number: max(nidx - 1, 0) */
        const uint32_t m0c = __vmins2(mn0, 0x00200020u), m1c = __vmins2(mn1, 0x00200020u);
        if constexpr (WIDE)
            __stcg(dst, make_uint4(m0c | (m1c << 6), nsg, nsg1, nidx));
        else
            __stcg(dst, make_uint2(m0c | (m1c << 6) | (nidx << 12), nsg));
    }
};


/* The form a kernel uses: the key form where it measured faster (normal
 * 1/2 and 3/5, whose layers have 5 and 9 information links and one pair of
 * shared links, and check degrees 22 and above), the min form elsewhere. */
__host__ __device__ constexpr bool pair_key_form(int a, int b, int gdm, int ls)
{
    return gdm == 0 && ((a == b && (a == 5 || a == 9) && ls == 2) || a >= 20);
}

template <int DM, bool EXACT, int LS, bool WIDE, bool PO, bool KEYS>
using PairCheck = typename std::conditional<KEYS, PairCheckKey<DM, EXACT, LS, WIDE, PO>,
                                            PairCheckMin<DM, EXACT, LS, WIDE, PO>>::type;

struct PairFrame {
    uint16_t* post;
    const int2* ent; /* (shared byte address of the link group's first word, -2 a) */
    const uint16_t* eoff;
    const uint32_t* steps;
    /* parity out of shared memory (PO kernels): the posterior word of
     * parity bit (i, j) is gpar[360 i + j] (global, this CTA's slab) for
     * i < q - 1 and wrap[j] (shared) for the last layer */
    uint16_t* gpar;
    uint16_t* wrap;
};

__device__ __forceinline__ size_t a16p(size_t v) { return (v + 15) & ~(size_t)15; }

template <bool PO, bool KEYS>
__device__ PairFrame stage_pair(const DevCode& c, char* smem, uint16_t* gpar)
{
    PairFrame f;
    f.post = (uint16_t*)smem;
    size_t off = a16p(2 * (size_t)(PO ? c.K : c.N));
    f.gpar = gpar;
    f.wrap = nullptr;
    if (PO) {
        f.wrap = (uint16_t*)(smem + off);
        off += a16p(2 * (size_t)kQCp);
    }
    int2* ent = (int2*)(smem + off);
    off += a16p(sizeof(int2) * c.nent);
    uint16_t* eoff = (uint16_t*)(smem + off);
    off += a16p(sizeof(uint16_t) * (c.q + 1));
    uint32_t* steps = (uint32_t*)(smem + off);
    /* entries (360 g - a, a) as, in the key form, (shared byte address of
     * group g's first posterior word, -2 a): the link of check j is word
     * (j - a) mod 360 of the group, at byte offset min(u, u + 720),
     * u = 2 j - 2 a unsigned; in the min form (shared byte address of the
     * link of check 0 before the wrap, a): x + 2 j, + 720 if j < a */
    const uint32_t sbase = (uint32_t)__cvta_generic_to_shared(f.post);
    for (int k = threadIdx.x; k < c.nent; k += blockDim.x) {
        const int2 e = c.ent[k];
        ent[k] = KEYS ? make_int2((int)(sbase + 2u * (uint32_t)(e.x + e.y)), -2 * e.y)
                      : make_int2((int)(sbase + 2u * (uint32_t)e.x), e.y);
    }
    for (int k = threadIdx.x; k <= c.q; k += blockDim.x)
        eoff[k] = c.eoff[k];
    for (int k = threadIdx.x; k < c.nsteps; k += blockDim.x)
        steps[k] = c.steps[k];
    f.ent = ent;
    f.eoff = eoff;
    f.steps = steps;
    return f;
}

/* Byte `h` of the posterior word of parity bit (ii, jj) */
template <bool PO>
__device__ __forceinline__ uint8_t* parity_byte(const DevCode& c, const PairFrame& fr, uint32_t ii, uint32_t jj, int h)
{
    if (!PO)
        return (uint8_t*)fr.post + 2 * (c.K + kQCp * ii + jj) + h;
    return ii + 1 < (uint32_t)c.q ? (uint8_t*)fr.gpar + 2 * (kQCp * ii + jj) + h : (uint8_t*)fr.wrap + 2 * jj + h;
}

/* Frame f's LLRs into byte `h` of every posterior word (f < 0: the all-zero
 * codeword at full confidence, which passes every check). */
template <bool PO>
__device__ void load_lane(const DevCode& c, const PairFrame& fr, const int8_t* __restrict__ src, int h)
{
    uint8_t* b = (uint8_t*)fr.post + h;
    const int t = threadIdx.x;
    if (!src) {
        for (int v = t; v < c.K; v += blockDim.x)
            b[2 * v] = 127;
        for (int k = t; k < c.R; k += blockDim.x)
            *parity_byte<PO>(c, fr, k / kQCp, k % kQCp, h) = 127;
        return;
    }
    if (((uintptr_t)src & 7) == 0) {
        const uint2* s8 = (const uint2*)src;
        for (int u = t; u < c.K / 8; u += blockDim.x) {
            const uint2 w = __ldcs(s8 + u);
#pragma unroll
            for (int r = 0; r < 8; r++)
                b[2 * (8 * u + r)] = (uint8_t)((r < 4 ? w.x : w.y) >> (8 * (r & 3)));
        }
        const uint32_t qm = 0xFFFFFFFFu / (uint32_t)c.q + 1u;
        for (int u = t; u < c.R / 8; u += blockDim.x) {
            const uint2 w = __ldcs(s8 + c.K / 8 + u);
#pragma unroll
            for (int r = 0; r < 8; r++) {
                const uint32_t k = 8u * u + r;
                const uint32_t jj = __umulhi(k, qm), ii = k - jj * c.q;
                *parity_byte<PO>(c, fr, ii, jj, h) = (uint8_t)((r < 4 ? w.x : w.y) >> (8 * (r & 3)));
            }
        }
    } else {
        for (int v = t; v < c.K; v += blockDim.x)
            b[2 * v] = (uint8_t)src[v];
        for (int k = t; k < c.R; k += blockDim.x)
            *parity_byte<PO>(c, fr, k % c.q, k / c.q, h) = (uint8_t)src[c.K + k];
    }
}

/* Syndrome of both lanes: bit h of the result set if lane h fails.  Thread
 * t checks column t % 360 of every other layer; the scan stops once both
 * lanes have failed.  The result is the OR over all layers, so the scan may
 * start anywhere: it starts at a layer where the previous scan found a
 * failure (srow[0], fixed during a scan; srow[1] collects a failing layer),
 * which a frame that still fails usually fails again. */
/* The posterior words of the two parity bits of check (i, j): its own and
 * the previous one (for check (0, 0), none: a positive stand-in) */
template <bool PO>
__device__ __forceinline__ void parity_words(const DevCode& c, const PairFrame& fr, int i, int j, uint32_t& pc,
                                             uint32_t& pp)
{
    if (PO) {
        pc = i + 1 < c.q ? fr.gpar[kQCp * i + j] : fr.wrap[j];
        pp = i ? fr.gpar[kQCp * (i - 1) + j] : (j ? fr.wrap[j - 1] : 0x0101u);
    } else {
        pc = fr.post[c.K + kQCp * i + j];
        pp = i ? fr.post[c.K + kQCp * (i - 1) + j] : (j ? fr.post[c.K + kQCp * (c.q - 1) + j - 1] : 0x0101u);
    }
}

template <bool PO, bool KEYS>
__device__ int syndrome_pair(const DevCode& c, const PairFrame& fr, volatile int* sflag, volatile int* srow)
{
    const int t = threadIdx.x;
    const int nh = blockDim.x / kQCp; /* threads per column */
    const int i0 = srow[0];
    int fail = 0;
    if (t < nh * kQCp) {
        const int j = t % kQCp, h0 = t / kQCp;
        /* parity words are loaded D rows ahead (global memory in PO kernels) */
        constexpr int D = 4;
        auto row = [&](int k) { return k + i0 < c.q ? k + i0 : k + i0 - c.q; };
        uint32_t bc[D], bp[D];
#pragma unroll
        for (int d = 0; d < D; d++) {
            bc[d] = bp[d] = 0;
            if (h0 + d * nh < c.q)
                parity_words<PO>(c, fr, row(h0 + d * nh), j, bc[d], bp[d]);
        }
        bool stop = false;
        for (int k0 = h0; k0 < c.q && !stop; k0 += D * nh) {
#pragma unroll
            for (int d = 0; d < D; d++) {
                const int k = k0 + d * nh;
                if (k >= c.q || *sflag == 3) {
                    stop = true;
                    break;
                }
                const int i = row(k);
                const uint32_t pc = sx2(bc[d]), pp = sx2(bp[d]);
                if (k + D * nh < c.q)
                    parity_words<PO>(c, fr, row(k + D * nh), j, bc[d], bp[d]);
                uint32_t par = pc ^ pp;
                uint32_t z = (__vadd2(pc, 0xFFFFFFFFu) & ~pc) | (__vadd2(pp, 0xFFFFFFFFu) & ~pp);
                const int e1 = fr.eoff[i + 1];
                for (int e = fr.eoff[i]; e < e1; e++) {
                    const int2 en = fr.ent[e];
                    uint32_t a;
                    if (KEYS) {
                        const uint32_t u = 2u * (uint32_t)j + (uint32_t)en.y;
                        a = (uint32_t)en.x + __viaddmin_u32(u, 2u * kQCp, u);
                    } else {
                        a = (uint32_t)en.x + 2u * (uint32_t)j + (j < en.y ? 2u * kQCp : 0u);
                    }
                    const uint32_t v = sx2(lds16(a));
                    par ^= v;
                    z |= __vadd2(v, 0xFFFFFFFFu) & ~v;
                }
                const uint32_t bad = (par | z);
                const int f = ((bad >> 15) & 1) | ((bad >> 30) & 2);
                if (f & ~fail) {
                    fail |= f;
                    atomicOr((int*)sflag, f);
                    srow[1] = i;
                }
            }
        }
    }
    __syncthreads();
    const int r = *sflag;
    if (t == 0)
        srow[0] = srow[1];
    __syncthreads();
    return r;
}

/*
 * Layer i of the phased schedule.  Every check reads its links that no
 * earlier check of the layer writes (a full-occupancy pass); then, level by
 * level, the checks of the level read their remaining links (written by
 * earlier levels), finish their minimums and write only the posteriors that
 * later checks of the layer read; a last full pass writes every other
 * posterior and the messages.  The reference's in-order semantics only
 * constrain the bits two checks of a layer share, so the wavefront levels
 * carry just those links.  Unlevelled layers take one pass.
 */
template <int DM, bool EXACT, int LS, bool WIDE, bool LEARNED, bool PO, bool KEYS>
__device__ __forceinline__ void layer_pair(const PairFrame& fr, const DevCode& c, int i, int cnt, int nlev,
                                           PairRec<WIDE> rec, unsigned long long meta, uint32_t fresh,
                                           PairRec<WIDE>* __restrict__ msg, int lA, int lB, uint32_t r0,
                                           uint32_t r1, uint32_t& o0, uint32_t& o1)
{
    const int t = threadIdx.x;
    const bool active = t < kQCp;
    const int j = t;
    /* the check's learned class table (an index into s_learn_lut) */
    auto lwords = [&](uint32_t& a, uint32_t& b) {
        a = b = 0;
        if (LEARNED)
            a = 128u * (uint32_t)s_learn_cls[(EXACT ? DM : cnt + 2) - ((i | j) == 0)];
    };
    using Ck = PairCheck<DM, EXACT, LS, WIDE, PO, KEYS>;
    Ck ck;
    if (active) {
        ck.setup(fr.ent + fr.eoff[i], cnt, c.K, c.q, i, j, rec, fresh, meta,
                 (uint32_t)__cvta_generic_to_shared(fr.post));
        if (nlev > 1)
            ck.template read_all<true>(fr.post, r0, r1);
        else
            ck.template read_all<false>(fr.post, r0, r1);
    } else {
        ck.idle((uint32_t)__cvta_generic_to_shared(fr.post));
    }
    if (nlev > 1) {
        /* a level step runs on every warp that holds a check of the level,
         * with all its lanes; the other checks keep their state.  KE: the
         * last slot that can be late or early in this warp (most
         * layers share one pair of links: link slots 2 and 3 only) */
        const int lev = active ? (int)(meta & 0xFF) : -1;
        uint32_t wa, wb; /* the check's learned words, read once for all its level steps */
        lwords(wa, wb);
        auto steps = [&](auto ke) {
            constexpr int KE = decltype(ke)::value;
            /* every level ends with a CTA barrier, the last one too: without
             * it the write pass of the other warps takes issue slots from the
             * last level's chain and the layer runs longer (measured), and
             * skipping the last level's early writes (it has none to store)
             * measured slower as well */
            for (int l = 0; l < nlev; l++) {
                const bool mine = lev == l;
                if (__any_sync(0xFFFFFFFFu, mine)) {
                    if (l > 0)
                        ck.template read_late<KE>(fr.post, mine);
                    ck.finish(mine, LEARNED, wa, wb);
                    ck.template write_early<KE>(fr.post, mine);
                }
                __syncthreads();
            }
        };
        constexpr int KS = Ck::K1 > 3 ? 3 : Ck::K1;
        const uint32_t lm = __reduce_or_sync(0xFFFFFFFFu, ck.inm | ck.outm);
        if (KS < Ck::K1 && (lm >> (KS + 1)) != 0)
            steps(std::integral_constant<int, Ck::K1>());
        else
            steps(std::integral_constant<int, KS>());
    } else if (active) {
        uint32_t wa, wb;
        lwords(wa, wb);
        ck.finish(true, LEARNED, wa, wb);
    }
    if (active)
        ck.write_rest(fr.post, msg + kQCp * i + j, o0, o1);
    __syncthreads();
}

/* One decoding iteration: the layers in order; each layer's messages and
 * level metadata are fetched one layer ahead.  The kernel is compiled for
 * the two information-link counts A <= B of its codes (exact-degree check
 * nodes), or, with GDM > 0, for any count up to GDM - 2 (predicated). */
template <int A, int B, int GDM, int LS, bool LEARNED, bool PO>
__device__ void iterate_pair(const DevCode& c, const PairFrame& fr, void* msgv, uint32_t fresh, int lA, int lB)
{
    constexpr bool WIDE = (GDM > 0 ? GDM : B + 2) > 16;
    using Rec = PairRec<WIDE>;
    Rec* __restrict__ msg = (Rec*)msgv;
    const int t = threadIdx.x;
    const int j = t;
    const bool active = t < kQCp;
    Rec rn{};
    unsigned long long mn = 0;
    /* PO: the words of parity bits (i, j) and (i + 1, j) for layers i and
     * i + 1 (loaded two layers ahead), and of (i - 1, j), which the previous
     * layer of this thread wrote */
    uint32_t pnext = 0, pnext2 = 0, carry = 0;
    if (LEARNED) {
        /* this iteration's learned magnitudes: lane A's row lA, lane B's lB */
        for (int e = t; e < 2 * kLearnClasses * 128; e += blockDim.x) {
            const int h = e / (kLearnClasses * 128), k = (e / 128) % kLearnClasses;
            s_learn_lut[e] = (uint8_t)min(learned_mag(e % 128, s_learn_tab[(h ? lB : lA) + k]), 255);
        }
        __syncthreads();
    }
    if (active) {
        rn = __ldcg(msg + j);
        mn = __ldg(c.lmeta + j);
        if (PO && c.q > 1)
            pnext = fr.gpar[j];
        if (PO && c.q > 2)
            pnext2 = fr.gpar[kQCp + j];
    }
    for (int i = 0; i < c.q; i++) {
        const Rec rec = rn;
        const unsigned long long meta = mn;
        uint32_t r0 = 0, r1 = 0, o0 = 0, o1 = 0;
        if (active && i + 1 < c.q) {
            rn = __ldcg(msg + kQCp * (i + 1) + j);
            mn = __ldg(c.lmeta + kQCp * (i + 1) + j);
        }
        if (PO && active) {
            r0 = i + 1 < c.q ? pnext : fr.wrap[j];
            pnext = pnext2;
            if (i + 3 < c.q)
                pnext2 = fr.gpar[kQCp * (i + 2) + j];
            r1 = i ? carry : (j ? fr.wrap[j - 1] : 0u);
        }
        const int cnt = fr.eoff[i + 1] - fr.eoff[i];
        const int nlev = c.nlev[i];
        if (GDM > 0)
            layer_pair<(GDM > 0 ? GDM : 2), false, LS, WIDE, LEARNED, PO, pair_key_form(A, B, GDM, LS)>(fr, c, i, cnt, nlev, rec, meta, fresh, msg,
                                                                           lA, lB, r0, r1, o0, o1);
        else if (A == B || cnt == A)
            layer_pair<A + 2, true, LS, WIDE, LEARNED, PO, pair_key_form(A, B, GDM, LS)>(fr, c, i, cnt, nlev, rec, meta, fresh, msg, lA, lB, r0, r1,
                                                           o0, o1);
        else
            layer_pair<B + 2, true, LS, WIDE, LEARNED, PO, pair_key_form(A, B, GDM, LS)>(fr, c, i, cnt, nlev, rec, meta, fresh, msg, lA, lB, r0, r1,
                                                           o0, o1);
        /* (i - 1, j) is final for this iteration; (i, j) goes to the next
         * layer, or, for the last layer, to the check (0, j + 1) */
        if (PO && active) {
            if (i)
                fr.gpar[kQCp * (i - 1) + j] = (uint16_t)o1;
            else if (j)
                fr.wrap[j - 1] = (uint16_t)o1;
            if (i + 1 < c.q)
                carry = o0;
            else
                fr.wrap[j] = (uint16_t)o0;
        }
    }
    if (PO)
        __syncthreads(); /* the last layer's wrap words before the syndrome reads them */
}

static __device__ void store_lane(const DevCode& c, const PairFrame& fr, int h, uint8_t* __restrict__ dst)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int8_t* b = (const int8_t*)fr.post + h;
    const int nchunks = (c.kldpc + 31) / 32;
    for (int ch = warp; ch < nchunks; ch += nw) {
        const int v = ch * 32 + lane;
        const int x = v < c.kldpc ? b[2 * v] : 0;
        const unsigned m = __ballot_sync(0xFFFFFFFFu, x < 0);
        const unsigned rr = __byte_perm(__brev(m), 0, 0x0123);
        if (lane < 4 && 4 * ch + lane < c.nbytes)
            dst[4 * ch + lane] = (uint8_t)(rr >> (8 * lane));
    }
}

/* Group barrier of a team of M co-resident CTAs (a cooperative launch):
 * returns 1 if no member saw a failing frame, 0 if one did, -1 if the
 * barrier gave up after `limit` polls (the device error word is set to 2).
 * skip: this CTA does not arrive (a test of the time-out) and returns -1. */
static __device__ int pair_team_vote(unsigned* slot, int M, bool fail, int* err, int limit, bool skip)
{
    __shared__ int s_res;
    if (threadIdx.x == 0) {
        unsigned* arrive = slot;
        unsigned* fails = slot + 1;
        int res = 0;
        if (skip) {
            res = -1;
        } else {
            if (fail)
                atomicAdd(fails, 1u);
            __threadfence();
            atomicAdd(arrive, 1u);
            int spins = 0;
            while (*(volatile unsigned*)arrive < (unsigned)M) {
                if (++spins > limit) {
                    atomicExch(err, 2);
                    res = -1;
                    break;
                }
                __nanosleep(200);
            }
            __threadfence();
            if (res == 0)
                res = *(volatile unsigned*)fails == 0 ? 1 : 0;
        }
        s_res = res;
    }
    __syncthreads();
    const int r = s_res;
    __syncthreads();
    return r;
}

/* Lane state of a frame-pair CTA (shared memory): the frame and iteration
 * of each lane, the syndrome flags, the lanes to reload, the syndrome
 * scan's start rows. */
struct PairLanes {
    int frame[2], iter[2], flag, reload, row[2];
};

/* Per-frame stopping: frames stream through the two lanes independently.
 * A lane whose frame passes the syndrome check or reaches max_iter writes
 * its results and takes the next frame of the batch (the counter p.work;
 * work item k is row p.rows[k], or k), so a converged frame never waits for
 * its neighbour.  The CTA's tables are staged (fr) and its lane state
 * initialised (frames -1, both lanes to reload, flag 0, rows 0). */
template <int A, int B, int GDM, int LS, bool PO>
__device__ __forceinline__ void stream_frames(const DecodeParams& p, const DevCode& c, const PairFrame& fr, void* msg,
                                              int lT, int nframes, PairLanes& st)
{
    int* s_frame = st.frame;
    int* s_iter = st.iter;
    int& s_flag = st.flag;
    int& s_reload = st.reload;
    int* s_row = st.row;
    const int t = threadIdx.x;
    uint32_t fresh = 0;
    for (;;) {
        /* lanes that need a frame take the next one of the batch */
        const int reload = s_reload;
        if (reload) {
            if (t == 0) {
                for (int h = 0; h < 2; h++)
                    if (reload & (1 << h)) {
                        const int f = (int)atomicAdd(p.work, 1u);
                        s_frame[h] = f < nframes ? f : -1;
                        s_iter[h] = 0;
                    }
            }
            __syncthreads();
            for (int h = 0; h < 2; h++)
                if (reload & (1 << h)) {
                    const int f = s_frame[h];
                    const int row = f < 0 ? 0 : p.rows ? p.rows[f] : f;
                    load_lane<PO>(c, fr, f >= 0 ? p.llr + (size_t)row * p.llr_stride : nullptr, h);
                    fresh |= 0xFFFFu << (16 * h);
                }
            if (t == 0)
                s_reload = 0;
            __syncthreads();
        }
        if (s_frame[0] < 0 && s_frame[1] < 0)
            break;
        const int fail = syndrome_pair<PO, pair_key_form(A, B, GDM, LS)>(c, fr, &s_flag, s_row);
        /* lanes whose frame is done: results out, refill */
        int done = 0;
        for (int h = 0; h < 2; h++) {
            const int f = s_frame[h];
            if (f >= 0 && (!((fail >> h) & 1) || s_iter[h] >= p.max_iter)) {
                const int row = p.rows ? p.rows[f] : f;
                store_lane(c, fr, h, p.out + (size_t)row * p.out_stride);
                if (t == 0) {
                    if (p.iters)
                        p.iters[row] = s_iter[h];
                    if (p.ok)
                        p.ok[row] = (fail >> h) & 1 ? 0 : 1;
                }
                done |= 1 << h;
            }
        }
        __syncthreads();
        if (t == 0) {
            s_flag = 0;
            s_reload = done;
        }
        __syncthreads();
        if (done)
            continue; /* reload, then check the new frames first */
        if (lT)
            iterate_pair<A, B, GDM, LS, true, PO>(c, fr, msg, fresh, learn_row(s_iter[0], lT),
                                                  learn_row(s_iter[1], lT));
        else
            iterate_pair<A, B, GDM, LS, false, PO>(c, fr, msg, fresh, -1, -1);
        fresh = 0;
        if (t == 0) {
            s_iter[0]++;
            s_iter[1]++;
        }
        __syncthreads();
    }
}

/* PM: 0 one resident CTA per SM; 1 two (80 registers), for codes whose
 * posteriors leave room for two (short frames); 2 two, with the parity
 * posteriors out of shared memory (PO: normal frames up to rate 4/5) */
template <int A, int B, int GDM, int LS, int PM>
__global__ void __launch_bounds__(384, PM ? 2 : 1) k_decode_pair(DecodeParams p)
{
    constexpr bool PO = PM == 2;
    extern __shared__ __align__(16) char smem[];
    __shared__ int s_lanes[sizeof(PairLanes) / sizeof(int)];
    int* s_frame = ((PairLanes*)s_lanes)->frame;
    int& s_flag = ((PairLanes*)s_lanes)->flag;
    int& s_reload = ((PairLanes*)s_lanes)->reload;
    int* s_row = ((PairLanes*)s_lanes)->row;
    const DevCode c = *p.code;
    constexpr bool WIDE = (GDM > 0 ? GDM : B + 2) > 16;
    void* msg = (char*)p.msg + (size_t)blockIdx.x * p.msg_stride;
    /* the parity words follow the message records in this CTA's slab */
    uint16_t* gpar = (uint16_t*)((char*)msg + (((size_t)c.R * (WIDE ? 16 : 8) + 15) & ~(size_t)15));
    const PairFrame fr = stage_pair<PO, pair_key_form(A, B, GDM, LS)>(c, smem, gpar);
    const int lT = stage_learn(p.learn, p.learn_class, p.learn_iters);
    const int nframes = p.nframes_dev ? *p.nframes_dev : p.nframes;
    const int t = threadIdx.x;
    if (t == 0) {
        s_frame[0] = s_frame[1] = -1;
        s_flag = 0;
        s_reload = 3;
        s_row[0] = s_row[1] = 0;
    }
    __syncthreads();
    if (p.group > 0) {
        /* group stopping (the reference's batch semantics): the G frames of a
         * group run on a team of M = ceil(G / 2) CTAs, two frames each, and
         * stop together at the first syndrome that every frame passes */
        const int G = p.group, M = (G + 1) / 2;
        const int team = blockIdx.x / M, member = blockIdx.x % M;
        const int ngroups = (p.nframes + G - 1) / G;
        const int per = p.max_iter + 1, per_team = (ngroups + p.nteams - 1) / p.nteams;
        for (int g = team, k = 0; g < ngroups; g += p.nteams, k++) {
            unsigned* sync = p.team_sync + 2 * (size_t)per * ((size_t)team * per_team + k);
            const int end = min((g + 1) * G, p.nframes);
            int fr2[2];
            for (int h = 0; h < 2; h++) {
                const int f = g * G + 2 * member + h;
                fr2[h] = f < end ? f : -1;
                const int row = fr2[h] < 0 ? 0 : p.rows ? p.rows[fr2[h]] : fr2[h];
                load_lane<PO>(c, fr, fr2[h] >= 0 ? p.llr + (size_t)row * p.llr_stride : nullptr, h);
            }
            __syncthreads();
            uint32_t gfresh = 0xFFFFFFFFu;
            int it = 0;
            bool ok = true;
            for (;;) {
                const int fail = syndrome_pair<PO, pair_key_form(A, B, GDM, LS)>(c, fr, &s_flag, s_row);
                if (t == 0)
                    s_flag = 0; /* read again only after later barriers */
                const int v = pair_team_vote(sync + 2 * it, M, fail != 0, p.err,
                                             p.wait_limit > 0 ? p.wait_limit : kDefaultWaitLimit,
                                             (int)blockIdx.x + 1 == p.skip_vote);
                ok = v == 1;
                if (v < 0 || ok || it >= p.max_iter)
                    break;
                iterate_pair<A, B, GDM, LS, false, PO>(c, fr, msg, gfresh, -1, -1);
                gfresh = 0;
                it++;
            }
            for (int h = 0; h < 2; h++)
                if (fr2[h] >= 0) {
                    const int row = p.rows ? p.rows[fr2[h]] : fr2[h];
                    store_lane(c, fr, h, p.out + (size_t)row * p.out_stride);
                    if (t == 0) {
                        if (p.iters)
                            p.iters[row] = it;
                        if (p.ok)
                            p.ok[row] = ok ? 1 : 0;
                    }
                }
            __syncthreads();
        }
        return;
    }
    PairLanes& st = *(PairLanes*)s_lanes;
    stream_frames<A, B, GDM, LS, PO>(p, c, fr, msg, lT, nframes, st);
}

/* Pair kernels by information-link counts (A, B): every pair of the DVB-S2,
 * S2X and T2 codes, plus predicated kernels for the codes whose layers have
 * more than two different counts (degree bounds 7, 11, 14, 22, 32).  LS:
 * late slots the kernel carries (two cover most levelled codes; normal 4/5
 * and 9/10 need four, short 5/6 five, short 8/9 six). */
struct PairKernel {
    int a, b, gdm, ls, pm, threads;
    const void* fn;
};


/* The instantiated kernels, in parts (part k in ldpc_pair_k<k>.cu):
 * pair_kernel_part(k, &n) returns part k and its n entries. */
const PairKernel* pair_kernel_part(int part, int* n);
constexpr int kPairKernelParts = 6;

/* launch bounds of a residency mode: 1 CTA per SM (mode 0) or two */
#define DRXG_PAIR_KERNEL(a, b, gdm, ls, pm) { a, b, gdm, ls, pm, 384, (const void*)k_decode_pair<a, b, gdm, ls, pm> }

}  // namespace drxg
