/*
 * ORACLE — test and benchmark infrastructure only; never linked into the
 * product library.
 *
 * Host-thread drivers of the reference decoder (libdvbrx/src/ldpc.c, built
 * from its own sources into oracle/_ref/libref_<isa>.so with every drx_*
 * export renamed ref_*).  This file is compiled into the same shared object
 * and calls the reference only through its public API
 * (libdvbrx/include/dvbrx/ldpc.h:14-36, fec.h:25).
 *
 *   refx_decode_frames_mt  each frame on its own (one drx_ldpc_decode call
 *                          with nframes = 1): hard bits, iterations, flags.
 *                          This is the per-frame oracle: the other lanes are
 *                          padded with 127 and pass every check
 *                          (ldpc.c:550-551, 614-638).
 *   refx_decode_groups_mt  consecutive groups of G frames, one call each:
 *                          hard bits and the call's return value (the
 *                          reference's batch semantics).
 *   refx_bench             the reference's production mode
 *                          (libdvbrx/src/rxmt.c:514-536): persistent worker
 *                          threads, each with its own handle, decoding
 *                          batches of `lanes` frames with drx_ldpc_decode;
 *                          timed steps separated by barriers, CLOCK_MONOTONIC
 *                          as tests/test_ldpc.c:22-27 does.
 *
 * Every function spreads its work over `threads` POSIX threads, each with
 * its own decoder handle (a reference handle is not thread-safe).
 */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

typedef struct {
    int short_frame, nldpc, kldpc, kbch, t;
} refx_fec;

/* the reference's API, renamed at build time (oracle/Makefile) */
int ref_ldpc_lanes(void);
void* ref_ldpc_new(const refx_fec* p, const char* rate);
void ref_ldpc_free(void* d);
int ref_ldpc_decode(void* d, const int8_t* const* llr, uint8_t* const* out, int nframes, int max_iter);

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

/* ---------------------------------------------------------------------- */
/* per-frame and per-group decodes over a work counter                     */
/* ---------------------------------------------------------------------- */

typedef struct {
    const refx_fec* p;
    const char* rate;
    const int8_t* llr;
    size_t llr_stride;
    uint8_t* out;
    size_t out_stride;
    int32_t* iters;   /* per frame (frames mode) */
    uint8_t* ok;      /* per frame (frames mode) */
    int32_t* rets;    /* per group (groups mode) */
    int nframes, max_iter, group;
    int next;         /* work counter (atomic) */
    int failed;       /* a handle could not be made */
} refx_job;

static void* frames_worker(void* arg)
{
    refx_job* j = (refx_job*)arg;
    void* d = ref_ldpc_new(j->p, j->rate);
    if (!d) {
        __atomic_store_n(&j->failed, 1, __ATOMIC_RELAXED);
        return NULL;
    }
    for (;;) {
        const int f = __atomic_fetch_add(&j->next, 1, __ATOMIC_RELAXED);
        if (f >= j->nframes)
            break;
        const int8_t* in = j->llr + (size_t)f * j->llr_stride;
        uint8_t* o = j->out + (size_t)f * j->out_stride;
        const int r = ref_ldpc_decode(d, &in, &o, 1, j->max_iter);
        j->iters[f] = r < 0 ? j->max_iter : r;
        j->ok[f] = r >= 0 ? 1 : 0;
    }
    ref_ldpc_free(d);
    return NULL;
}

static void* groups_worker(void* arg)
{
    refx_job* j = (refx_job*)arg;
    void* d = ref_ldpc_new(j->p, j->rate);
    if (!d) {
        __atomic_store_n(&j->failed, 1, __ATOMIC_RELAXED);
        return NULL;
    }
    const int G = j->group;
    const int ngroups = (j->nframes + G - 1) / G;
    const int8_t** in = (const int8_t**)malloc(sizeof(*in) * (size_t)G);
    uint8_t** o = (uint8_t**)malloc(sizeof(*o) * (size_t)G);
    for (;;) {
        const int g = __atomic_fetch_add(&j->next, 1, __ATOMIC_RELAXED);
        if (g >= ngroups)
            break;
        const int f0 = g * G, n = j->nframes - f0 < G ? j->nframes - f0 : G;
        for (int f = 0; f < n; f++) {
            in[f] = j->llr + (size_t)(f0 + f) * j->llr_stride;
            o[f] = j->out + (size_t)(f0 + f) * j->out_stride;
        }
        j->rets[g] = ref_ldpc_decode(d, in, o, n, j->max_iter);
    }
    free(in);
    free(o);
    ref_ldpc_free(d);
    return NULL;
}

static int run_job(refx_job* j, void* (*fn)(void*), int threads)
{
    if (threads < 1)
        threads = 1;
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)threads);
    int started = 0;
    for (int t = 0; t < threads; t++)
        if (pthread_create(&th[t], NULL, fn, j) == 0)
            started++;
        else
            break;
    if (started == 0) /* no thread at all: run on the caller's */
        fn(j);
    for (int t = 0; t < started; t++)
        pthread_join(th[t], NULL);
    free(th);
    return j->failed ? -1 : 0;
}

int refx_decode_frames_mt(const refx_fec* p, const char* rate, const int8_t* llr, size_t llr_stride, int nframes,
                          int max_iter, uint8_t* out, size_t out_stride, int32_t* iters, uint8_t* ok, int threads)
{
    refx_job j;
    memset(&j, 0, sizeof(j));
    j.p = p;
    j.rate = rate;
    j.llr = llr;
    j.llr_stride = llr_stride;
    j.out = out;
    j.out_stride = out_stride;
    j.iters = iters;
    j.ok = ok;
    j.nframes = nframes;
    j.max_iter = max_iter;
    return run_job(&j, frames_worker, threads);
}

int refx_decode_groups_mt(const refx_fec* p, const char* rate, const int8_t* llr, size_t llr_stride, int nframes,
                          int group, int max_iter, uint8_t* out, size_t out_stride, int32_t* rets, int threads)
{
    if (group < 1 || group > ref_ldpc_lanes())
        return -1;
    refx_job j;
    memset(&j, 0, sizeof(j));
    j.p = p;
    j.rate = rate;
    j.llr = llr;
    j.llr_stride = llr_stride;
    j.out = out;
    j.out_stride = out_stride;
    j.rets = rets;
    j.nframes = nframes;
    j.group = group;
    j.max_iter = max_iter;
    return run_job(&j, groups_worker, threads);
}

/* ---------------------------------------------------------------------- */
/* production-mode throughput: persistent workers, timed steps             */
/* ---------------------------------------------------------------------- */

typedef struct {
    const refx_fec* p;
    const char* rate;
    const int8_t* pool;  /* npool frames of pool_stride bytes */
    size_t pool_stride;
    int npool;
    int max_iter;
    int lanes;           /* frames per drx_ldpc_decode call */
    int steps;           /* warm-up + timed */
    int calls_per_step;  /* calls of the whole pool of threads in one step */
    double seconds;      /* > 0: one open-ended step of this length instead */
    pthread_barrier_t bar;
    pthread_mutex_t gate_lock;
    pthread_cond_t gate_cv;
    int gate;            /* 0 closed, 1 go, -1 abort (a worker did not start) */
    int failed;
    long long calls_done;
    double* step_s;      /* steps entries (thread 0 writes) */
    int call_next;       /* call counter, re-based by thread 0 between steps */
    volatile int stop;   /* open-ended step: time is up */
} refx_bench_job;

typedef struct {
    refx_bench_job* b;
    int id;
} refx_bench_arg;

static void* bench_worker(void* arg)
{
    refx_bench_arg* a = (refx_bench_arg*)arg;
    refx_bench_job* b = a->b;
    pthread_mutex_lock(&b->gate_lock);
    while (b->gate == 0)
        pthread_cond_wait(&b->gate_cv, &b->gate_lock);
    const int go = b->gate > 0;
    pthread_mutex_unlock(&b->gate_lock);
    if (!go)
        return NULL; /* another worker could not start: the barrier would never open */
    const size_t nb = (size_t)((b->p->kldpc + 7) / 8);
    void* d = ref_ldpc_new(b->p, b->rate);
    if (!d)
        __atomic_store_n(&b->failed, 1, __ATOMIC_RELAXED);
    const int8_t** in = (const int8_t**)malloc(sizeof(*in) * (size_t)b->lanes);
    uint8_t* obuf = (uint8_t*)malloc((size_t)b->lanes * nb);
    uint8_t** o = (uint8_t**)malloc(sizeof(*o) * (size_t)b->lanes);
    for (int f = 0; f < b->lanes; f++)
        o[f] = obuf + (size_t)f * nb;
    long long mine = 0;
    const int nsteps = b->seconds > 0 ? 1 : b->steps;
    for (int s = 0; s < nsteps; s++) {
        double t0 = 0;
        pthread_barrier_wait(&b->bar); /* every worker ready */
        if (a->id == 0)
            t0 = now_s();
        pthread_barrier_wait(&b->bar);
        for (;;) {
            if (b->seconds > 0 && b->stop)
                break;
            const int k = __atomic_fetch_add(&b->call_next, 1, __ATOMIC_RELAXED);
            if (b->seconds <= 0 && k >= (s + 1) * b->calls_per_step)
                break;
            if (d) {
                /* call k decodes `lanes` consecutive frames of the pool */
                const int f0 = (int)(((long long)k * b->lanes) % (b->npool - b->lanes + 1));
                for (int f = 0; f < b->lanes; f++)
                    in[f] = b->pool + (size_t)(f0 + f) * b->pool_stride;
                ref_ldpc_decode(d, in, o, b->lanes, b->max_iter);
            }
            mine++;
            if (b->seconds > 0 && a->id == 0 && now_s() - t0 >= b->seconds)
                b->stop = 1;
        }
        pthread_barrier_wait(&b->bar); /* every worker done */
        if (a->id == 0) {
            b->step_s[s] = now_s() - t0;
            b->call_next = (s + 1) * b->calls_per_step; /* workers ran past the step's last call */
        }
    }
    __atomic_fetch_add(&b->calls_done, mine, __ATOMIC_RELAXED);
    free(in);
    free(o);
    free(obuf);
    if (d)
        ref_ldpc_free(d);
    return NULL;
}

/*
 * Production-mode run.  With seconds > 0: one step of about that length
 * (every worker decoding calls until the time is up).  Otherwise `steps`
 * steps of `calls_per_step` calls each, shared by the workers.  step_s
 * receives each step's wall time (CLOCK_MONOTONIC, between barriers);
 * *calls receives the number of drx_ldpc_decode calls made.  Returns 0, or
 * -1 if a handle could not be made or a thread could not start.
 */
int refx_bench(const refx_fec* p, const char* rate, const int8_t* pool, size_t pool_stride, int npool, int max_iter,
               int lanes, int threads, int steps, int calls_per_step, double seconds, double* step_s,
               long long* calls)
{
    if (lanes < 1 || lanes > ref_ldpc_lanes() || npool < lanes || threads < 1)
        return -1;
    refx_bench_job b;
    memset(&b, 0, sizeof(b));
    b.p = p;
    b.rate = rate;
    b.pool = pool;
    b.pool_stride = pool_stride;
    b.npool = npool;
    b.max_iter = max_iter;
    b.lanes = lanes;
    b.steps = steps < 1 ? 1 : steps;
    b.calls_per_step = calls_per_step < 1 ? 1 : calls_per_step;
    b.seconds = seconds;
    b.step_s = step_s;
    if (pthread_barrier_init(&b.bar, NULL, (unsigned)threads) != 0)
        return -1;
    pthread_mutex_init(&b.gate_lock, NULL);
    pthread_cond_init(&b.gate_cv, NULL);
    pthread_t* th = (pthread_t*)malloc(sizeof(pthread_t) * (size_t)threads);
    refx_bench_arg* args = (refx_bench_arg*)malloc(sizeof(refx_bench_arg) * (size_t)threads);
    int started = 0;
    for (int t = 0; t < threads; t++) {
        args[t].b = &b;
        args[t].id = t;
        if (pthread_create(&th[t], NULL, bench_worker, &args[t]) != 0)
            break;
        started++;
    }
    pthread_mutex_lock(&b.gate_lock);
    b.gate = started == threads ? 1 : -1;
    pthread_cond_broadcast(&b.gate_cv);
    pthread_mutex_unlock(&b.gate_lock);
    for (int t = 0; t < started; t++)
        pthread_join(th[t], NULL);
    if (started != threads)
        b.failed = 1;
    pthread_barrier_destroy(&b.bar);
    pthread_mutex_destroy(&b.gate_lock);
    pthread_cond_destroy(&b.gate_cv);
    free(th);
    free(args);
    if (calls)
        *calls = b.calls_done;
    return b.failed ? -1 : 0;
}
