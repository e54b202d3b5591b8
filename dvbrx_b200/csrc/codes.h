/*
 * Host-side LDPC code compiler: turns a DVB-S2 / S2X / T2 parity-address
 * table into the layer form the GPU decoder walks.
 *
 * The reference (libdvbrx/src/ldpc.c:199-260) expands every table into an
 * R x CNL list of information-bit indexes in layer order.  Here the
 * quasi-cyclic structure is kept instead: a table address x = q*a + i feeds,
 * for every check j of layer i, information bit 360*g + ((j - a) mod 360) of
 * column group g.  One layer is therefore a short list of (g, a) pairs, and
 * the address of every link is computed on the fly from the check index.
 *
 * The reference walks the 360 checks of a layer in order j = 0..359
 * (ldpc.c:465-482).  Two checks of the same layer that share an information
 * bit (which happens in every DVB-S2 table, in none of the S2X ones) must
 * therefore run in j order.  The compiler levels each layer: level(j) =
 * 1 + max level of the earlier checks sharing a bit with j; checks of one
 * level are independent and run in parallel, levels run in order.  The
 * result is a list of "steps" (layer, first position, count) and, for
 * levelled layers, the permutation position -> check index.
 */
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

namespace drxg {

constexpr int QC = 360; /* columns of a quasi-cyclic group */

struct Code {
    int table = -1;         /* index into cg_tables */
    std::string table_name; /* e.g. "DVB_S2_TABLE_B5" */
    int N = 0, K = 0, R = 0, q = 0;
    int cnt_max = 0;   /* most information links of a check */
    int cnt_min = 0;   /* fewest information links of a layer */
    int deg_max = 0;   /* cnt_max + 2 parity links */
    int dclass = 0;    /* kernel class: degree_class(deg_max) */
    int edges = 0;     /* links of the whole Tanner graph */
    int nlevels = 0;   /* steps per iteration */
    bool levelled = false;
    bool phased = true; /* lmeta holds every check's late and early slots */
    /* per layer i: entries eoff[i] .. eoff[i+1]-1, each a pair
     * (360*g - a, a): check j of the layer links information bit
     * 360*g - a + j, plus 360 if j < a */
    std::vector<int32_t> ent;
    std::vector<uint16_t> eoff;
    /* step = layer | start << 8 | count << 17 | permuted << 26 */
    std::vector<uint32_t> steps;
    /* q * 360 check indexes by position (identity for unlevelled layers) */
    std::vector<uint16_t> perm;
    /* per layer: number of wavefront levels */
    std::vector<uint8_t> nlev;
    /* per check j of layer i (index 360 i + j), for the phased schedule:
     * bits 0-7 its level, bits 8-31 the link slots it reads after an earlier
     * check of the layer wrote them ("in"), bits 32-55 the slots a later
     * check of the layer reads after it ("out").  Slot 0 = parity, 1 =
     * previous parity, 2 + e = information entry e of the layer. */
    std::vector<uint64_t> lmeta;
    /* accumulator addresses of the standard table, for the encoder:
     * per information bit group g, addr[aoff[g] .. aoff[g+1]-1] */
    std::vector<uint16_t> addr;
    std::vector<uint32_t> aoff;
};

/* Kernel classes by largest check degree: each class's kernel is compiled
 * for degrees up to kClassDeg[class] only, so that its register budget fits
 * the codes it runs. */
constexpr int kNumClasses = 6;
constexpr int kClassDeg[kNumClasses] = { 7, 11, 14, 18, 22, 32 };
/* smallest information-link count of a layer in the codes of each class
 * (the frame-pair kernel instantiates link counts kClassCntLo .. max) */
constexpr int kClassCntLo[kNumClasses] = { 1, 5, 7, 12, 14, 25 };
int degree_class(int deg_max);

/* Rate string -> table index (cg_rates_normal / cg_rates_short), or -1.
 * Mirrors find_table(), libdvbrx/src/ldpc.c:188-197. */
int find_table(int short_frame, const char* rate);

/* Compile table `table`; false if the table violates an assumption of the
 * GPU layout (reported through `err`). */
bool compile_code(int table, Code* out, std::string* err);

}  // namespace drxg
