/*
 * A C caller of the LDPC decoder through the reference's own public API
 * (libdvbrx/include/dvbrx/ldpc.h:14-36, fec.h:13-25) and nothing else: the
 * program a receiver built against libdvbrx would be, relinked against
 * libdvbrx_b200.so.  It decodes a file of frames in batches of
 * drx_ldpc_lanes() frames, through per-frame pointer arrays sized for the
 * callers' MAX_LANES of 64 (the loop of libdvbrx/tests/test_ldpc.c:78-94 and
 * libdvbrx/src/rx.c:132).
 *
 *   dropin_caller <short 0|1> <rate> <max_iter> <llr file> <out file>
 *
 * llr file: nframes * nldpc int8 LLRs.  out file: nframes * ceil(kldpc/8)
 * bytes of hard bits, then one int32 per batch (drx_ldpc_decode's return
 * value).  Exit status 0 on success, 2 if drx_fec_lookup or drx_ldpc_new
 * fails (no device: the library fails loudly), 1 on a usage or I/O error.
 *
 * Compiled with -DUSE_B200_HEADER against include/dvbrx_b200.h, otherwise
 * against the reference's headers (dvbrx/fec.h, dvbrx/ldpc.h).
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

#ifdef USE_B200_HEADER
#include "dvbrx_b200.h"
#else
#include "dvbrx/fec.h"
#include "dvbrx/ldpc.h"
#endif

#define MAX_LANES 64

int main(int argc, char** argv)
{
    if (argc != 6) {
        fprintf(stderr, "usage: %s short rate max_iter llr_file out_file\n", argv[0]);
        return 1;
    }
    const int short_frame = atoi(argv[1]), max_iter = atoi(argv[3]);
    drx_fec_params p;
    if (drx_fec_lookup(short_frame, argv[2], &p) != 0) {
        fprintf(stderr, "drx_fec_lookup(%s) failed\n", argv[2]);
        return 2;
    }
    FILE* f = fopen(argv[4], "rb");
    if (!f)
        return 1;
    fseek(f, 0, SEEK_END);
    const long bytes = ftell(f);
    fseek(f, 0, SEEK_SET);
    const int nf = (int)(bytes / p.nldpc);
    int8_t* llr = malloc((size_t)bytes);
    if (!llr || fread(llr, 1, (size_t)bytes, f) != (size_t)bytes)
        return 1;
    fclose(f);

    drx_ldpc* d = drx_ldpc_new(&p, argv[2]);
    if (!d) {
        fprintf(stderr, "drx_ldpc_new(%s) failed\n", argv[2]);
        return 2;
    }
    const int lanes = drx_ldpc_lanes();
    if (lanes < 1 || lanes > MAX_LANES) {
        fprintf(stderr, "drx_ldpc_lanes() = %d, outside 1..%d\n", lanes, MAX_LANES);
        return 1;
    }
    const size_t nb = (size_t)(p.kldpc + 7) / 8;
    const int nbatch = (nf + lanes - 1) / lanes;
    uint8_t* out = calloc((size_t)nf, nb);
    int32_t* ret = calloc((size_t)(nbatch > 0 ? nbatch : 1), sizeof(int32_t));
    for (int f0 = 0, b = 0; f0 < nf; f0 += lanes, b++) {
        const int n = nf - f0 < lanes ? nf - f0 : lanes;
        const int8_t* in[MAX_LANES];
        uint8_t* o[MAX_LANES];
        for (int k = 0; k < n; k++) {
            in[k] = llr + (size_t)(f0 + k) * p.nldpc;
            o[k] = out + (size_t)(f0 + k) * nb;
        }
        ret[b] = drx_ldpc_decode(d, in, o, n, max_iter);
    }
    drx_ldpc_free(d);

    f = fopen(argv[5], "wb");
    if (!f || fwrite(out, nb, (size_t)nf, f) != (size_t)nf || fwrite(ret, sizeof(int32_t), (size_t)nbatch, f) != (size_t)nbatch)
        return 1;
    fclose(f);
    free(llr);
    free(out);
    free(ret);
    return 0;
}
