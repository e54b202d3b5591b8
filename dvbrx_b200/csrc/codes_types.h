/*
 * Row types of the generated code tables (codes_gen.h).  Plain C so that the
 * product library and the oracle restatement read the same data.
 */
#pragma once
#include <stdint.h>

/* One LDPC parity-check table of EN 302 307 / EN 302 755: N, K and the
 * 360-bit column groups as runs of (addresses per group, groups), then the
 * parity-accumulator addresses of the first bit of every group. */
struct cg_table {
    const char* name;
    int N, K, nruns;
    const uint16_t* runs; /* nruns pairs: addresses per group, number of groups */
    const uint16_t* addr;
};

/* Rate string (gr-dvbs2rx naming, e.g. "3_5", "13_45", "2_3_t2") -> table. */
struct cg_rate {
    const char* rate;
    int table;
};

/* Rate string -> BCH parameters (kbch, nbch = kldpc, t). */
struct cg_fec {
    const char* rate;
    int kbch, nbch, t;
};

/* Constellation of a PLS code: bits per symbol, bit-interleaver column order
 * (-1: no interleaver) and the points by bit label, MSB first. */
struct cg_const {
    int pls;
    const char* name;
    const char* rate;
    int short_frame, bits;
    int order[8];
    float points[512];
};
