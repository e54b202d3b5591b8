/*
 * ORACLE — test infrastructure only.  Nothing in the product links, loads or
 * calls this file; only tests/, __graft_entry__.smoke() and bench.py's
 * cpu_baseline leg use it, and only as the checker.
 *
 * A scalar (one frame at a time) C restatement of the reference LDPC decoder,
 * libdvbrx/src/ldpc.c (dvbrx 0.1.3): layered offset min-sum (offset 1) on
 * saturating int8 values, check-to-variable messages clamped to [-32, 31],
 * syndrome check before every iteration.  The reference runs one frame per
 * SIMD byte lane; here every lane operation is written out on plain ints, so
 * the decisions, iteration counts and syndrome flags are those of the
 * reference for the same input bytes.  Parity is pinned by the tests against
 * the reference compiled from its own sources (oracle/_ref) and against the
 * committed golden fixtures (tests/golden/).
 *
 * Also here: the DVB-S2 systematic encoder (accumulator rule), which the
 * reference does not ship (its test vectors come from GNU Radio gr-dtv,
 * tests/txvectors.py:22); its correctness is checked by the reference decoder
 * converging in 0 iterations on every encoded word.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "codes_gen.h"

#define M 360
#define MAX_DEG 32

typedef struct orc_code {
    int N, K, R, q, CNL, kldpc;
    int comp;      /* the reference stores this code's messages compressed */
    uint16_t* pos; /* R * CNL information-bit indexes, layer order */
    uint8_t* cnc;  /* information links of every check of layer i, i < q */
} orc_code;

static int find_rate(int short_frame, const char* rate)
{
    const struct cg_rate* map = short_frame ? cg_rates_short : cg_rates_normal;
    const int n = short_frame ? (int)(sizeof(cg_rates_short) / sizeof(*cg_rates_short))
                              : (int)(sizeof(cg_rates_normal) / sizeof(*cg_rates_normal));
    for (int i = 0; i < n; i++)
        if (!strcmp(map[i].rate, rate))
            return map[i].table;
    return -1;
}

/* libdvbrx/src/bch.c:25-41 */
int orc_fec_lookup(int short_frame, const char* rate, int* nldpc, int* kldpc, int* kbch, int* t)
{
    const struct cg_fec* rows = short_frame ? cg_fec_short : cg_fec_normal;
    const int n = short_frame ? (int)(sizeof(cg_fec_short) / sizeof(*cg_fec_short))
                              : (int)(sizeof(cg_fec_normal) / sizeof(*cg_fec_normal));
    for (int i = 0; i < n; i++)
        if (!strcmp(rows[i].rate, rate)) {
            *nldpc = short_frame ? 16200 : 64800;
            *kldpc = rows[i].nbch;
            *kbch = rows[i].kbch;
            *t = rows[i].t;
            return 0;
        }
    return -1;
}

/* libdvbrx/src/ldpc.c:199-260: group walk, accumulator addresses
 * (x + m q) mod R, then check q*j + i moved to layer position M*i + j. */
orc_code* orc_new(int short_frame, const char* rate, int kldpc)
{
    const int ti = find_rate(short_frame, rate);
    if (ti < 0)
        return NULL;
    const struct cg_table* t = &cg_tables[ti];
    orc_code* d = calloc(1, sizeof(*d));
    d->N = t->N;
    d->K = t->K;
    d->R = t->N - t->K;
    d->q = d->R / M;
    d->kldpc = kldpc;
    /* check degree = information links + 2 parity links */
    int cnl = 0;
    {
        uint8_t* c = calloc(d->R, 1);
        const uint16_t* a = t->addr;
        for (int r = 0; r < t->nruns; r++)
            for (int g = 0; g < t->runs[2 * r + 1]; g++, a += t->runs[2 * r])
                for (int n = 0; n < t->runs[2 * r]; n++)
                    c[a[n] % d->q]++; /* layer a % q gains one link per check */
        for (int i = 0; i < d->q; i++)
            cnl = c[i] > cnl ? c[i] : cnl;
        free(c);
    }
    d->CNL = cnl;
    d->comp = d->CNL + 2 >= 9; /* COMP_MIN_DEG, ldpc.c:170-172,223 */
    uint16_t* pos = calloc((size_t)d->R * d->CNL, sizeof(uint16_t));
    d->pos = malloc(sizeof(uint16_t) * (size_t)d->R * d->CNL);
    d->cnc = calloc(d->R, 1);
    const uint16_t* row = t->addr;
    int j = 0;
    for (int r = 0; r < t->nruns; r++) {
        const int deg = t->runs[2 * r];
        for (int g = 0; g < t->runs[2 * r + 1]; g++, row += deg)
            for (int m = 0; m < M; m++, j++)
                for (int n = 0; n < deg; n++) {
                    const int acc = (row[n] + m * d->q) % d->R;
                    pos[d->CNL * acc + d->cnc[acc]++] = (uint16_t)j;
                }
    }
    for (int i = 0; i < d->q; i++)
        for (int jj = 0; jj < M; jj++)
            memcpy(d->pos + (size_t)d->CNL * (M * i + jj), pos + (size_t)d->CNL * (d->q * jj + i),
                   sizeof(uint16_t) * d->CNL);
    free(pos);
    return d;
}

void orc_free(orc_code* d)
{
    if (!d)
        return;
    free(d->pos);
    free(d->cnc);
    free(d);
}

int orc_n(const orc_code* d) { return d->N; }
int orc_k(const orc_code* d) { return d->K; }
int orc_q(const orc_code* d) { return d->q; }
int orc_cnl(const orc_code* d) { return d->CNL; }
int orc_comp(const orc_code* d) { return d->comp; }

/* ldpc.c:277-284 */
static inline int prev_parity(const orc_code* d, int i, int j)
{
    if (i)
        return M * (i - 1) + j;
    if (j)
        return j + (d->q - 1) * M - 1;
    return -1;
}

static inline int sat8(int x) { return x > 127 ? 127 : x < -128 ? -128 : x; }
/* v_sign(a, b), ldpc.c:50-54: a if b > 0, -a if b < 0, 0 if b == 0 */
static inline int vsign(int a, int b) { return b > 0 ? a : b < 0 ? -a : 0; }

/* ldpc.c:286-305: 1 if some check node is not satisfied; a posterior of
 * exactly 0 fails the check. */
static int bad(const orc_code* d, const int8_t* data, const int8_t* pty)
{
    for (int i = 0; i < d->q; i++) {
        const int cnt = d->cnc[i];
        for (int j = 0; j < M; j++) {
            const int cn = M * i + j;
            int cnv = vsign(1, pty[cn]);
            const int pp = prev_parity(d, i, j);
            if (pp >= 0)
                cnv = vsign(cnv, pty[pp]);
            const uint16_t* p = d->pos + (size_t)d->CNL * cn;
            for (int c = 0; c < cnt; c++)
                cnv = vsign(cnv, data[p[c]]);
            if (cnv <= 0)
                return 1;
        }
    }
    return 0;
}

/* ldpc.c:321-362 (check_node), one lane.  v[c] are the node's posteriors in
 * link order (information links, then the parity node, then the previous
 * parity node), bl its messages.  The compressed variant (ldpc.c:386-462)
 * stores the same clamped messages in another layout, so one restatement
 * serves both. */
/* Learned magnitude of this project's learned decoder (not in the
 * reference): word = scale_q | offset_q << 16 (Q8), m capped at 127. */
static inline int learned_mag(int m, uint32_t w)
{
    const int r = ((int)(w & 0xFFFFu) * m - ((int32_t)w >> 16) + 128) >> 8;
    return r > 0 ? r : 0;
}

static void check_node(int8_t* const* v, int8_t* bl, int deg, int first, const uint32_t* lw)
{
    int x[MAX_DEG];
    int min0 = 255, min1 = 255, signs = 0;
    for (int c = 0; c < deg; c++) {
        x[c] = first ? *v[c] : sat8(*v[c] - bl[c]);
        const int a = x[c] < 0 ? -x[c] : x[c]; /* |x| as uint8: -128 -> 128 */
        const int mx = min0 > a ? min0 : a;
        min1 = min1 < mx ? min1 : mx;
        min0 = min0 < a ? min0 : a;
        signs ^= x[c];
    }
    /* offset 1 and the cap at 127 once per node (ldpc.c:350-353) */
    int mn0 = (min0 < 127 ? min0 : 127) - 1 > 0 ? (min0 < 127 ? min0 : 127) - 1 : 0;
    int mn1 = (min1 < 127 ? min1 : 127) - 1 > 0 ? (min1 < 127 ? min1 : 127) - 1 : 0;
    if (lw) { /* the learned rule replaces offset 1 (scale_q >= 0: mn1 >= mn0 still) */
        mn0 = learned_mag(min0 < 127 ? min0 : 127, *lw);
        mn1 = learned_mag(min1 < 127 ? min1 : 127, *lw);
    }
    for (int c = 0; c < deg; c++) {
        const int a = x[c] < 0 ? -x[c] : x[c];
        const int mag = a == min0 ? (mn0 > mn1 ? mn0 : mn1) : mn0;
        /* sign of (signs ^ x) | 127: never zero (ldpc.c:341) */
        const int o = ((signs ^ x[c]) < 0) ? -mag : mag;
        *v[c] = (int8_t)sat8(x[c] + o);                    /* posterior: unclamped o */
        bl[c] = (int8_t)(o < -32 ? -32 : o > 31 ? 31 : o); /* message: clamped */
    }
}

/* One decoder state (one frame): posteriors, layer-ordered parity
 * posteriors and messages (R * (CNL + 2), link order). */
typedef struct {
    int8_t* data;
    int8_t* pty;
    int8_t* bl;
} lane;

static void lane_load(const orc_code* d, lane* l, const int8_t* llr)
{
    memcpy(l->data, llr, d->N);
    for (int i = 0; i < d->q; i++) /* ldpc.c:624-626 */
        for (int j = 0; j < M; j++)
            l->pty[M * i + j] = l->data[d->K + d->q * j + i];
}

/* ldpc.c:465-517: layers in order, checks j = 0..359 in order.  lrow /
 * lcls: a learned table row and the class of each degree, or NULL. */
static void update(const orc_code* d, lane* l, int first, const uint32_t* lrow, const int8_t* lcls)
{
    int8_t* v[MAX_DEG];
    for (int i = 0; i < d->q; i++) {
        const int cnt = d->cnc[i];
        for (int j = 0; j < M; j++) {
            const int cn = M * i + j;
            const uint16_t* p = d->pos + (size_t)d->CNL * cn;
            for (int c = 0; c < cnt; c++)
                v[c] = l->data + p[c];
            v[cnt] = l->pty + cn;
            const int pp = prev_parity(d, i, j);
            int deg = cnt + 1;
            if (pp >= 0)
                v[deg++] = l->pty + pp;
            check_node(v, l->bl + (size_t)(d->CNL + 2) * cn, deg, first, lrow ? lrow + lcls[deg] : NULL);
        }
    }
}

/* ldpc.c:581-612: bit = posterior < 0, kldpc bits packed MSB first. */
static void lane_store(const orc_code* d, const lane* l, uint8_t* out)
{
    const int nbytes = (d->kldpc + 7) / 8;
    memset(out, 0, nbytes);
    for (int b = 0; b < d->kldpc; b++)
        if (l->data[b] < 0)
            out[b >> 3] |= (uint8_t)(0x80 >> (b & 7));
}

static int lane_alloc(const orc_code* d, lane* l)
{
    l->data = malloc(d->N);
    l->pty = malloc(d->R);
    l->bl = malloc((size_t)d->R * (d->CNL + 2));
    return l->data && l->pty && l->bl;
}

static void lane_release(lane* l)
{
    free(l->data);
    free(l->pty);
    free(l->bl);
}

/*
 * Reference semantics for a batch of n frames decoded together
 * (ldpc.c:614-638): iterate while some frame fails the syndrome and
 * it < max_iter; every frame runs the same number of iterations.  Returns
 * the iterations run if all frames pass, else -1.
 */
int orc_decode_group(const orc_code* d, const int8_t* const* llr, uint8_t* const* out, int n,
                     int max_iter)
{
    if (n <= 0)
        return 0;
    lane* l = calloc(n, sizeof(lane));
    for (int f = 0; f < n; f++) {
        if (!lane_alloc(d, &l[f]))
            return -2;
        lane_load(d, &l[f], llr[f]);
    }
    int it = 0, ok;
    for (;;) {
        ok = 1;
        for (int f = 0; f < n && ok; f++)
            ok = !bad(d, l[f].data, l[f].pty);
        if (ok || it >= max_iter)
            break;
        for (int f = 0; f < n; f++)
            update(d, &l[f], it == 0, NULL, NULL);
        it++;
    }
    for (int f = 0; f < n; f++) {
        lane_store(d, &l[f], out[f]);
        lane_release(&l[f]);
    }
    free(l);
    return ok ? it : -1;
}

/*
 * One frame on its own: the reference called with nframes = 1 (the other
 * lanes carry the all-zero codeword, ldpc.c:550-551, which satisfies every
 * check).  *iters receives the iterations run; returns 1 if the syndrome
 * passed, 0 if not after max_iter iterations.
 */
int orc_decode_frame(const orc_code* d, const int8_t* llr, uint8_t* out, int max_iter, int* iters)
{
    const int8_t* in[1] = { llr };
    uint8_t* o[1] = { out };
    const int r = orc_decode_group(d, in, o, 1, max_iter);
    *iters = r < 0 ? max_iter : r;
    return r >= 0;
}

/* Many frames, each decoded on its own (contiguous buffers). */
void orc_decode_frames(const orc_code* d, const int8_t* llr, uint8_t* out, int32_t* iters,
                       uint8_t* ok, int nframes, int max_iter)
{
    const int nbytes = (d->kldpc + 7) / 8;
    for (int f = 0; f < nframes; f++) {
        int it;
        ok[f] = (uint8_t)orc_decode_frame(d, llr + (size_t)f * d->N, out + (size_t)f * nbytes,
                                          max_iter, &it);
        iters[f] = it;
    }
}

/*
 * This project's learned decoder at int8 (not in the reference): the same
 * schedule with the node magnitude of learned_mag from row min(it, T - 1)
 * of tab (8 words per row, one per degree class; cls[deg] is the class of a
 * node of degree deg).  One frame, per-frame stopping; returns 1 if the
 * syndrome passed.
 */
int orc_decode_frame_learned(const orc_code* d, const int8_t* llr, uint8_t* out, int max_iter, int* iters,
                             const uint32_t* tab, int T, const int8_t* cls)
{
    lane l;
    if (!lane_alloc(d, &l))
        return -2;
    lane_load(d, &l, llr);
    int it = 0, ok;
    for (;;) {
        ok = !bad(d, l.data, l.pty);
        if (ok || it >= max_iter)
            break;
        update(d, &l, it == 0, tab + 8 * (it < T ? it : T - 1), cls);
        it++;
    }
    lane_store(d, &l, out);
    lane_release(&l);
    *iters = it;
    return ok;
}

/*
 * Systematic DVB-S2 encoder (EN 302 307-1 5.3.2): information bit m of
 * 360-bit group g is added into parity accumulators (x + m q) mod R for the
 * group's addresses x, then p_k ^= p_{k-1}.  info: K bytes of 0/1; cw: N
 * bytes of 0/1 (information bits, then parity bits).
 */
void orc_encode(const orc_code* d, const uint8_t* info, uint8_t* cw)
{
    memcpy(cw, info, d->K);
    uint8_t* p = cw + d->K;
    memset(p, 0, d->R);
    /* the layer-ordered pos table holds, for check q*j + i at M*i + j, the
     * information bits that accumulator sums: the same walk as the
     * standard's accumulator rule, over the code the decoder decodes */
    for (int i = 0; i < d->q; i++)
        for (int j = 0; j < M; j++) {
            const uint16_t* pp = d->pos + (size_t)d->CNL * (M * i + j);
            int s = 0;
            for (int c = 0; c < d->cnc[i]; c++)
                s ^= info[pp[c]];
            p[d->q * j + i] = (uint8_t)s;
        }
    for (int k = 1; k < d->R; k++)
        p[k] ^= p[k - 1];
}

/*
 * DVB-S2 BCH encoder (EN 302 307-1 5.3.1), for building test codewords: the
 * generator g(x) is the product of the minimal polynomials of alpha^(2i+1),
 * i < t, over GF(2^16) (normal frames, primitive x^16+x^5+x^3+x^2+1) or
 * GF(2^14) (short frames, x^14+x^5+x^3+x+1); the codeword is the kbch
 * message bits followed by the nbch - kbch bits of m(x) x^(nbch-kbch) mod
 * g(x), packed MSB first.  Checked by the reference's own decoder
 * (bch.c:189-290) finding no error in every encoded word.
 */
static int bch_gpoly(int short_frame, int t, uint8_t* g)
{
    const int m = short_frame ? 14 : 16, q = (1 << m) - 1;
    const unsigned prim = short_frame ? 0x402B : 0x1002D;
    uint16_t* ex = malloc(sizeof(uint16_t) * 2 * q);
    int* lg = malloc(sizeof(int) * (q + 1));
    unsigned x = 1;
    for (int i = 0; i < q; i++) {
        ex[i] = ex[i + q] = (uint16_t)x;
        lg[x] = i;
        x <<= 1;
        if (x >> m)
            x ^= prim;
    }
    int dg = 0;
    g[0] = 1;
    for (int i = 1; i < 2 * t; i += 2) {
        /* minimal polynomial of alpha^i: product of (x + alpha^e), e over i's cyclotomic coset */
        uint16_t p[40] = { 1 };
        int dp = 0, e = i % q;
        do {
            const uint16_t beta = ex[e];
            for (int k = dp + 1; k > 0; k--)
                p[k] = p[k - 1] ^ (p[k] && beta ? ex[lg[p[k]] + lg[beta]] : 0);
            p[0] = p[0] && beta ? ex[lg[p[0]] + lg[beta]] : 0;
            dp++;
            e = (2 * e) % q;
        } while (e != i % q);
        uint8_t r[200] = { 0 };
        for (int a = 0; a <= dg; a++)
            if (g[a])
                for (int b = 0; b <= dp; b++)
                    r[a + b] ^= (uint8_t)(p[b] & 1);
        dg += dp;
        memcpy(g, r, dg + 1);
    }
    free(ex);
    free(lg);
    return dg;
}

int orc_bch_encode(int short_frame, int t, int kbch, int nbch, const uint8_t* msg, uint8_t* cw)
{
    uint8_t g[200];
    const int W = bch_gpoly(short_frame, t, g);
    if (W != nbch - kbch)
        return -1;
    uint8_t* rem = calloc(W + 1, 1); /* rem[k]: coefficient of x^k */
    for (int b = 0; b < kbch; b++) {
        const int bit = (msg[b >> 3] >> (7 - (b & 7))) & 1;
        const int top = rem[W - 1] ^ bit;
        for (int k = W - 1; k > 0; k--)
            rem[k] = rem[k - 1] ^ (top & g[k]);
        rem[0] = (uint8_t)(top & g[0]);
    }
    memset(cw, 0, (nbch + 7) / 8);
    for (int b = 0; b < kbch; b++)
        if ((msg[b >> 3] >> (7 - (b & 7))) & 1)
            cw[b >> 3] |= (uint8_t)(0x80 >> (b & 7));
    for (int k = 0; k < W; k++) { /* parity bits, highest degree first */
        const int b = kbch + (W - 1 - k);
        if (rem[k])
            cw[b >> 3] |= (uint8_t)(0x80 >> (b & 7));
    }
    free(rem);
    return W;
}
